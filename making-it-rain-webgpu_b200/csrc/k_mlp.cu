// k_mlp.cu -- the barostat's screening network: a 3-layer perceptron
// (inputs -> 64 tanh -> 64 tanh -> 1), BF16 weights, FP32 accumulation,
// trained on the device by its own forward/backward/Adam kernel.
//
// No reference counterpart: the reference's Monte Carlo barostat
// (src/reference/barostat.ts:210) evaluates the exact energy for every
// proposal.  Here the network predicts the potential-energy change of a
// volume move from the current energy components, virial, box and the move's
// dlnV, and serves as the first stage of a delayed-acceptance test
// (Christen & Fox 2005); the exact PME energy still decides the second stage.
//
// Sizes are tiny (a 128-sample minibatch is 1.2 MFLOP per layer), so the
// contractions run on the FP32 pipe out of shared memory: at this size tensor
// core tiles would be almost all padding and launch latency dominates.
// Every reduction over samples runs in a fixed order, with no atomics, so
// training is bit-reproducible.
#include <cmath>
#include <numeric>
#include <vector>

#include "../../include/mdb.h"
#include "device_state.h"
#include "mlp.h"

namespace mdb {
namespace {

constexpr int kT = 256;  // threads of the one training CTA

struct Smem {
  float w1[kMlpHidden * kMlpIn], b1[kMlpHidden];
  float w2[kMlpHidden * kMlpHidden], b2[kMlpHidden];
  float w3[kMlpHidden], b3;
};

__device__ __forceinline__ void load_weights(Smem& s, const __nv_bfloat16* w) {
  for (int i = threadIdx.x; i < kMlpParams; i += blockDim.x) {
    const float v = __bfloat162float(w[i]);
    if (i < kMlpOffB1) s.w1[i] = v;
    else if (i < kMlpOffW2) s.b1[i - kMlpOffB1] = v;
    else if (i < kMlpOffB2) s.w2[i - kMlpOffW2] = v;
    else if (i < kMlpOffW3) s.b2[i - kMlpOffB2] = v;
    else if (i < kMlpOffB3) s.w3[i - kMlpOffW3] = v;
    else s.b3 = v;
  }
}

// Forward for one sample held by one thread (inference).
__global__ void __launch_bounds__(128) k_mlp_forward(const __nv_bfloat16* w, const float* x, int n, float* y) {
  __shared__ Smem s;
  load_weights(s, w);
  __syncthreads();
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < n; b += gridDim.x * blockDim.x) {
    float in[kMlpIn], h1[kMlpHidden];
#pragma unroll
    for (int k = 0; k < kMlpIn; ++k) in[k] = x[b * kMlpIn + k];
#pragma unroll 4
    for (int j = 0; j < kMlpHidden; ++j) {
      float a = s.b1[j];
#pragma unroll
      for (int k = 0; k < kMlpIn; ++k) a = fmaf(s.w1[j * kMlpIn + k], in[k], a);
      h1[j] = tanhf(a);
    }
    float out = s.b3;
    for (int j = 0; j < kMlpHidden; ++j) {
      float a = s.b2[j];
#pragma unroll 8
      for (int i = 0; i < kMlpHidden; ++i) a = fmaf(s.w2[j * kMlpHidden + i], h1[i], a);
      out = fmaf(s.w3[j], tanhf(a), out);
    }
    y[b] = out;
  }
}

// One epoch of minibatch Adam on the mean squared error, in one CTA.
// Sample order: p(i) = (perm_a * i + perm_c) mod n (perm_a coprime to n).
// With `grads` non-null the kernel stops after the first minibatch and writes
// that minibatch's gradient (the FP32 master layout) and loss instead of
// updating: the gradient check.
__global__ void __launch_bounds__(kT) k_mlp_epoch(MlpDev m, const float* x, const float* target, int n,
                                                   int perm_a, int perm_c, float* grads, float* loss_out) {
  extern __shared__ float dyn[];
  __shared__ Smem s;
  float* X = dyn;                                  // [B][In]
  float* H1 = X + kMlpBatch * kMlpIn;              // [B][H]
  float* H2 = H1 + kMlpBatch * kMlpHidden;         // [B][H]
  float* D2 = H2 + kMlpBatch * kMlpHidden;         // [B][H]  dL/d(pre-activation 2)
  float* D1 = D2 + kMlpBatch * kMlpHidden;         // [B][H]  dL/d(pre-activation 1)
  float* DY = D1 + kMlpBatch * kMlpHidden;         // [B]
  float* G = DY + kMlpBatch;                       // [params] gradient of this minibatch
  __shared__ float red[kT / 32];
  const int tid = threadIdx.x;
  int adam_step = *m.step_count;  // Adam's t, carried across epochs
  load_weights(s, m.w_bf16);
  __syncthreads();
  for (int start = 0; start < n; start += kMlpBatch) {
    const int B = min(kMlpBatch, n - start);
    for (int i = tid; i < B * kMlpIn; i += kT) {
      const int b = i / kMlpIn, k = i - b * kMlpIn;
      const int row = static_cast<int>((static_cast<long long>(perm_a) * (start + b) + perm_c) % n);
      X[i] = x[row * kMlpIn + k];
    }
    __syncthreads();
    // ---- forward
    for (int i = tid; i < B * kMlpHidden; i += kT) {
      const int b = i / kMlpHidden, j = i - b * kMlpHidden;
      float a = s.b1[j];
#pragma unroll
      for (int k = 0; k < kMlpIn; ++k) a = fmaf(s.w1[j * kMlpIn + k], X[b * kMlpIn + k], a);
      H1[i] = tanhf(a);
    }
    __syncthreads();
    for (int i = tid; i < B * kMlpHidden; i += kT) {
      const int b = i / kMlpHidden, j = i - b * kMlpHidden;
      float a = s.b2[j];
#pragma unroll 8
      for (int k = 0; k < kMlpHidden; ++k) a = fmaf(s.w2[j * kMlpHidden + k], H1[b * kMlpHidden + k], a);
      H2[i] = tanhf(a);
    }
    __syncthreads();
    float part = 0.f;
    for (int b = tid; b < B; b += kT) {
      float y = s.b3;
      for (int j = 0; j < kMlpHidden; ++j) y = fmaf(s.w3[j], H2[b * kMlpHidden + j], y);
      const int row = static_cast<int>((static_cast<long long>(perm_a) * (start + b) + perm_c) % n);
      const float e = y - target[row];
      DY[b] = 2.f * e / B;
      part += e * e;
    }
    __syncthreads();
    // ---- backward: deltas
    for (int i = tid; i < B * kMlpHidden; i += kT) {
      const int b = i / kMlpHidden, j = i - b * kMlpHidden;
      const float h = H2[i];
      D2[i] = DY[b] * s.w3[j] * (1.f - h * h);
    }
    __syncthreads();
    for (int i = tid; i < B * kMlpHidden; i += kT) {
      const int b = i / kMlpHidden, k = i - b * kMlpHidden;
      float a = 0.f;
      for (int j = 0; j < kMlpHidden; ++j) a = fmaf(s.w2[j * kMlpHidden + k], D2[b * kMlpHidden + j], a);
      const float h = H1[i];
      D1[i] = a * (1.f - h * h);
    }
    __syncthreads();
    // ---- gradients, each a fixed-order sum over the minibatch
    for (int p = tid; p < kMlpParams; p += kT) {
      float g = 0.f;
      if (p < kMlpOffB1) {
        const int j = p / kMlpIn, k = p - j * kMlpIn;
        for (int b = 0; b < B; ++b) g = fmaf(D1[b * kMlpHidden + j], X[b * kMlpIn + k], g);
      } else if (p < kMlpOffW2) {
        const int j = p - kMlpOffB1;
        for (int b = 0; b < B; ++b) g += D1[b * kMlpHidden + j];
      } else if (p < kMlpOffB2) {
        const int q = p - kMlpOffW2, j = q / kMlpHidden, k = q - j * kMlpHidden;
        for (int b = 0; b < B; ++b) g = fmaf(D2[b * kMlpHidden + j], H1[b * kMlpHidden + k], g);
      } else if (p < kMlpOffW3) {
        const int j = p - kMlpOffB2;
        for (int b = 0; b < B; ++b) g += D2[b * kMlpHidden + j];
      } else if (p < kMlpOffB3) {
        const int j = p - kMlpOffW3;
        for (int b = 0; b < B; ++b) g = fmaf(DY[b], H2[b * kMlpHidden + j], g);
      } else {
        for (int b = 0; b < B; ++b) g += DY[b];
      }
      G[p] = g;
    }
    // minibatch loss (mean squared error), fixed-order
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
    if ((tid & 31) == 0) red[tid >> 5] = part;
    __syncthreads();
    if (grads) {
      for (int p = tid; p < kMlpParams; p += kT) grads[p] = G[p];
      if (tid == 0) {
        float l = 0.f;
        for (int w = 0; w < kT / 32; ++w) l += red[w];
        *loss_out = l / B;
      }
      return;
    }
    if (tid == 0 && loss_out) {
      float l = 0.f;
      for (int w = 0; w < kT / 32; ++w) l += red[w];
      loss_out[start / kMlpBatch] = l / B;
    }
    // ---- Adam on the FP32 master weights, then the BF16 copy and the smem weights
    ++adam_step;
    const float c1 = 1.f - powf(m.beta1, float(adam_step)), c2 = 1.f - powf(m.beta2, float(adam_step));
    for (int p = tid; p < kMlpParams; p += kT) {
      const float g = G[p];
      const float mm = m.beta1 * m.m[p] + (1.f - m.beta1) * g;
      const float vv = m.beta2 * m.v[p] + (1.f - m.beta2) * g * g;
      m.m[p] = mm;
      m.v[p] = vv;
      const float w = m.w[p] - m.lr * (mm / c1) / (sqrtf(vv / c2) + m.eps);
      m.w[p] = w;
      const __nv_bfloat16 wb = __float2bfloat16_rn(w);
      m.w_bf16[p] = wb;
    }
    __syncthreads();
    load_weights(s, m.w_bf16);
    __syncthreads();
  }
  if (tid == 0) *m.step_count = adam_step;
}

}  // namespace

int mlp_epoch_smem_bytes() {
  return int(sizeof(float)) * (kMlpBatch * kMlpIn + 4 * kMlpBatch * kMlpHidden + kMlpBatch + kMlpParams);
}

void launch_mlp_forward(const __nv_bfloat16* w, const float* x, int n, float* y, cudaStream_t st) {
  const int blocks = std::max(1, std::min((n + 127) / 128, 148));
  k_mlp_forward<<<blocks, 128, 0, st>>>(w, x, n, y);
}

cudaError_t launch_mlp_epoch(const MlpDev& m, const float* x, const float* target, int n, int perm_a, int perm_c,
                             float* grads, float* loss, cudaStream_t st) {
  const int smem = mlp_epoch_smem_bytes();
  cudaError_t err = cudaFuncSetAttribute(k_mlp_epoch, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (err != cudaSuccess) return err;
  k_mlp_epoch<<<1, kT, smem, st>>>(m, x, target, n, perm_a, perm_c, grads, loss);
  return cudaGetLastError();
}

// Seeded Glorot-uniform weights (splitmix64 stream), zero biases, rounded to
// BF16 like every weight the kernels see.
void mlp_init_weights(uint32_t seed, float* w) {
  uint64_t state = 0x9e3779b97f4a7c15ull ^ seed;
  auto uniform = [&]() {
    state += 0x9e3779b97f4a7c15ull;
    uint64_t z = state;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    z ^= z >> 31;
    return double(z >> 11) * 0x1.0p-53;
  };
  for (int i = 0; i < kMlpParams; ++i) w[i] = 0.f;
  auto glorot = [&](int off, int fan_in, int fan_out, int count) {
    const double lim = std::sqrt(6.0 / (fan_in + fan_out));
    for (int i = 0; i < count; ++i) w[off + i] = float(lim * (2 * uniform() - 1));
  };
  glorot(0, kMlpIn, kMlpHidden, kMlpHidden * kMlpIn);
  glorot(kMlpOffW2, kMlpHidden, kMlpHidden, kMlpHidden * kMlpHidden);
  glorot(kMlpOffW3, kMlpHidden, 1, kMlpHidden);
  for (int i = 0; i < kMlpParams; ++i) w[i] = __bfloat162float(__float2bfloat16_rn(w[i]));
}

cudaError_t mlp_upload_weights(const MlpDev& m, const float* w, cudaStream_t st) {
  std::vector<__nv_bfloat16> wb(kMlpParams);
  for (int i = 0; i < kMlpParams; ++i) wb[i] = __float2bfloat16_rn(w[i]);
  cudaError_t err = cudaMemcpyAsync(m.w, w, sizeof(float) * kMlpParams, cudaMemcpyHostToDevice, st);
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(m.w_bf16, wb.data(), sizeof(__nv_bfloat16) * kMlpParams, cudaMemcpyHostToDevice, st);
  if (err == cudaSuccess) err = cudaStreamSynchronize(st);
  return err;
}

// Fresh Adam state, then `epochs` epochs over (x, t) on the device.  The
// sample order of epoch e is a multiplicative permutation with a prime
// coprime to n.  `epoch_loss` (may be null) receives each epoch's mean
// minibatch loss.
cudaError_t mlp_train(const MlpDev& m, const float* x, const float* t, int n, int epochs, uint32_t seed,
                      float* loss_dev, std::vector<double>* epoch_loss, cudaStream_t st) {
  std::vector<float> w(kMlpParams), zeros(kMlpParams, 0.f);
  mlp_init_weights(seed, w.data());
  cudaError_t err = mlp_upload_weights(m, w.data(), st);
  const int zero = 0;
  if (err == cudaSuccess) err = cudaMemcpy(m.m, zeros.data(), sizeof(float) * kMlpParams, cudaMemcpyHostToDevice);
  if (err == cudaSuccess) err = cudaMemcpy(m.v, zeros.data(), sizeof(float) * kMlpParams, cudaMemcpyHostToDevice);
  if (err == cudaSuccess) err = cudaMemcpy(m.step_count, &zero, sizeof(int), cudaMemcpyHostToDevice);
  static const int kPrimes[] = {7919, 104729, 15485863, 32452843, 49979687};
  const int batches = (n + kMlpBatch - 1) / kMlpBatch;
  std::vector<float> losses(batches);
  for (int ep = 0; ep < epochs && err == cudaSuccess; ++ep) {
    long long a = kPrimes[ep % 5];
    while (std::gcd(a, static_cast<long long>(n)) != 1) a += 2;
    err = launch_mlp_epoch(m, x, t, n, static_cast<int>(a % n == 0 ? 1 : a % n), (ep * 97) % n, nullptr, loss_dev, st);
    if (err == cudaSuccess && epoch_loss) {
      err = cudaMemcpyAsync(losses.data(), loss_dev, sizeof(float) * batches, cudaMemcpyDeviceToHost, st);
      if (err == cudaSuccess) err = cudaStreamSynchronize(st);
      double l = 0;
      for (float v : losses) l += v;
      epoch_loss->push_back(l / batches);
    }
  }
  return err == cudaSuccess ? cudaStreamSynchronize(st) : err;
}

}  // namespace mdb

// ---- diagnostic entry points (allocate; used by the tests) -------------------
namespace {

struct MlpScratch {
  mdb::MlpDev m{};
  float *x = nullptr, *t = nullptr, *y = nullptr, *g = nullptr, *loss = nullptr;
  ~MlpScratch() {
    for (void* p : {(void*)m.w, (void*)m.m, (void*)m.v, (void*)m.w_bf16, (void*)m.step_count, (void*)x, (void*)t,
                    (void*)y, (void*)g, (void*)loss})
      if (p) cudaFree(p);
  }
  cudaError_t alloc(int n) {
    cudaError_t err = cudaSuccess;
    auto get = [&](void** p, size_t bytes) {
      if (err == cudaSuccess) err = cudaMalloc(p, std::max<size_t>(bytes, 16));
    };
    get((void**)&m.w, sizeof(float) * mdb::kMlpParams);
    get((void**)&m.m, sizeof(float) * mdb::kMlpParams);
    get((void**)&m.v, sizeof(float) * mdb::kMlpParams);
    get((void**)&m.w_bf16, sizeof(__nv_bfloat16) * mdb::kMlpParams);
    get((void**)&m.step_count, sizeof(int));
    get((void**)&x, sizeof(float) * size_t(n) * mdb::kMlpIn);
    get((void**)&t, sizeof(float) * size_t(n));
    get((void**)&y, sizeof(float) * size_t(n));
    get((void**)&g, sizeof(float) * mdb::kMlpParams);
    get((void**)&loss, sizeof(float) * (size_t(n) / mdb::kMlpBatch + 2));
    m.lr = 2e-3f;
    m.beta1 = 0.9f;
    m.beta2 = 0.999f;
    m.eps = 1e-8f;
    return err;
  }
};

}  // namespace

extern "C" int mdb_mlp_gradient(const float* params, const float* x, const float* t, int32_t n, float* grad,
                                float* loss) {
  if (!params || !x || !t || !grad || !loss || n <= 0) return MDB_ERR_INVALID_ARGUMENT;
  MlpScratch s;
  if (s.alloc(n) != cudaSuccess) return MDB_ERR_DEVICE;
  if (mdb::mlp_upload_weights(s.m, params, nullptr) != cudaSuccess) return MDB_ERR_DEVICE;
  if (cudaMemcpy(s.x, x, sizeof(float) * size_t(n) * mdb::kMlpIn, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(s.t, t, sizeof(float) * size_t(n), cudaMemcpyHostToDevice) != cudaSuccess)
    return MDB_ERR_DEVICE;
  if (mdb::launch_mlp_epoch(s.m, s.x, s.t, n, 1, 0, s.g, s.loss, nullptr) != cudaSuccess) return MDB_ERR_DEVICE;
  if (cudaMemcpy(grad, s.g, sizeof(float) * mdb::kMlpParams, cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(loss, s.loss, sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
    return MDB_ERR_DEVICE;
  return MDB_OK;
}

extern "C" int mdb_mlp_fit(const float* x, const float* t, int32_t n, int32_t epochs, uint32_t seed,
                           float* params, float* epoch_loss) {
  if (!x || !t || !params || n < mdb::kMlpBatch || epochs <= 0) return MDB_ERR_INVALID_ARGUMENT;
  MlpScratch s;
  if (s.alloc(n) != cudaSuccess) return MDB_ERR_DEVICE;
  if (cudaMemcpy(s.x, x, sizeof(float) * size_t(n) * mdb::kMlpIn, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(s.t, t, sizeof(float) * size_t(n), cudaMemcpyHostToDevice) != cudaSuccess)
    return MDB_ERR_DEVICE;
  std::vector<double> losses;
  if (mdb::mlp_train(s.m, s.x, s.t, n, epochs, seed, s.loss, epoch_loss ? &losses : nullptr, nullptr) !=
      cudaSuccess)
    return MDB_ERR_DEVICE;
  if (cudaMemcpy(params, s.m.w, sizeof(float) * mdb::kMlpParams, cudaMemcpyDeviceToHost) != cudaSuccess)
    return MDB_ERR_DEVICE;
  if (epoch_loss)
    for (size_t k = 0; k < losses.size(); ++k) epoch_loss[k] = float(losses[k]);
  return MDB_OK;
}

extern "C" int mdb_mlp_predict(const float* params, const float* x, int32_t n, float* y) {
  if (!params || !x || !y || n <= 0) return MDB_ERR_INVALID_ARGUMENT;
  MlpScratch s;
  if (s.alloc(n) != cudaSuccess) return MDB_ERR_DEVICE;
  if (mdb::mlp_upload_weights(s.m, params, nullptr) != cudaSuccess) return MDB_ERR_DEVICE;
  if (cudaMemcpy(s.x, x, sizeof(float) * size_t(n) * mdb::kMlpIn, cudaMemcpyHostToDevice) != cudaSuccess)
    return MDB_ERR_DEVICE;
  mdb::launch_mlp_forward(s.m.w_bf16, s.x, n, s.y, nullptr);
  if (cudaMemcpy(y, s.y, sizeof(float) * size_t(n), cudaMemcpyDeviceToHost) != cudaSuccess) return MDB_ERR_DEVICE;
  return MDB_OK;
}
