// mlp.h -- the barostat screening network's layout and launchers (k_mlp.cu).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

namespace mdb {

constexpr int kMlpIn = 16;       // input features (padded with zeros)
constexpr int kMlpHidden = 64;   // units per hidden layer
constexpr int kMlpBatch = 128;   // training minibatch

// Parameter layout (FP32 master and BF16 copy alike): W1[H][In], b1[H],
// W2[H][H], b2[H], w3[H], b3.
constexpr int kMlpOffB1 = kMlpHidden * kMlpIn;
constexpr int kMlpOffW2 = kMlpOffB1 + kMlpHidden;
constexpr int kMlpOffB2 = kMlpOffW2 + kMlpHidden * kMlpHidden;
constexpr int kMlpOffW3 = kMlpOffB2 + kMlpHidden;
constexpr int kMlpOffB3 = kMlpOffW3 + kMlpHidden;
constexpr int kMlpParams = kMlpOffB3 + 1;

struct MlpDev {
  float* w;              // FP32 master weights
  float* m;              // Adam first moment
  float* v;              // Adam second moment
  __nv_bfloat16* w_bf16; // the weights the kernels compute with
  int* step_count;       // Adam's t
  float lr, beta1, beta2, eps;
};

int mlp_epoch_smem_bytes();
void launch_mlp_forward(const __nv_bfloat16* w, const float* x, int n, float* y, cudaStream_t st);
cudaError_t launch_mlp_epoch(const MlpDev& m, const float* x, const float* target, int n, int perm_a, int perm_c,
                             float* grads, float* loss, cudaStream_t st);
void mlp_init_weights(uint32_t seed, float* w);
cudaError_t mlp_upload_weights(const MlpDev& m, const float* w, cudaStream_t st);
cudaError_t mlp_train(const MlpDev& m, const float* x, const float* t, int n, int epochs, uint32_t seed,
                      float* loss_dev, std::vector<double>* epoch_loss, cudaStream_t st);

}  // namespace mdb
