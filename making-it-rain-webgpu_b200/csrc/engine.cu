// engine.cu -- the host runtime behind include/mdb.h.
//
// Owns every device table (labelled, so destroy() can report what it frees,
// src/gpu/allocator.ts:69), three streams, and the captured CUDA graphs that
// replace the reference's per-step command-buffer encoding
// (src/gpu/loop.ts:715-751).  One step is
//
//   list kernels (return at once unless a rebuild was asked for)
//   wrap
//   fork:  nonbonded tiles (s0) | listed terms (s2) | PME chain (s1)
//   join:  fused integrator (s0)
//
// and `max_batch` such steps are captured once and replayed.  Nothing on this
// path runs on the CPU: the host only uploads inputs, replays graphs, and
// reads results back.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <map>
#include <memory>
#include <numeric>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/mdb.h"
#include "barostat_rules.h"
#include "device_state.h"
#include "mlp.h"
#include "prep.h"

namespace mdb {
void set_pme_smem(int z, int y, int x, int plane);
}

using namespace mdb;

namespace {

constexpr double kCellWidth = 0.25;  // nm, fractional cells of the spatial sort
constexpr int kDefaultCluster = 8;   // atoms per cluster of the tile list
constexpr double kDefaultInnerSkin = -1.0;  // nm; <= 0: no inner list unless a tuning asks for one
// Starting capacity of the dense tile list, per cluster: about 1.7 times the
// mean row of water at a 0.5 nm skin (~230 tiles for 8-atom clusters) and
// twice that at a 0.2 nm skin (~90 for 32).  A list that needs more stops the
// integrator and is grown and rebuilt by the host (grow_tile_list).
int row_cap_for(int cluster) { return cluster == 8 ? 384 : 192; }
// the exact stage switches the screening network off once its running RMS
// error exceeds this many kT (the plain barostat takes over)
constexpr double kSurrogateMaxRmsKT = 1.5;
constexpr int kPlaneSmemLimit = 200 * 1024;  // bytes: two complex Ky x Kz planes per CTA

struct Allocation {
  std::string label;
  void* ptr;
  size_t bytes;
};

// The barostat's screening network for one system (no reference counterpart).
struct Surrogate {
  int target = 0;                 // exact attempts to learn from before screening; 0 = off
  bool active = false;            // trained: proposals go through the two-stage test
  bool disabled = false;          // the exact stage found it too inaccurate: plain barostat
  std::vector<float> feats;       // raw features of every exact attempt, kMlpIn each
  std::vector<double> delta_u;    // exact change minus its first-order term, per atom, kJ/mol
  std::vector<double> dlnv;       // the move of each attempt
  double mu[kMlpIn] = {}, sd[kMlpIn] = {}, mu_t = 0, sd_t = 1;
  double err2 = 0;                // running mean square of (predicted - exact) change
  int64_t checked = 0;
  MlpDev dev{};
  float* x = nullptr;             // device: normalised training inputs, then inference inputs
  float* t = nullptr;             // device: normalised targets
  float* y = nullptr;             // device: inference outputs
  float* loss = nullptr;          // device: per-minibatch losses of the last epoch
  float* xi = nullptr;            // device: inference inputs, two rows per system
  float* yi = nullptr;            // device: inference outputs
  double final_loss = 0;
  double fit_ms = 0;              // device time of the fits so far (one CTA: the epochs run in sequence)
};

struct BarostatState {
  double volume_scale = 0;
  int64_t attempts = 0, accepted = 0, step = 0, draw = 0;
  int64_t screened = 0, exact = 0;
  int window_attempts = 0, window_accepted = 0;
};

}  // namespace

struct mdb_engine {
  int device = 0;
  mdb_run_options opt{};
  RunDev run{};
  std::vector<HostSystem> hs;
  std::vector<SysDev> sd;
  std::vector<BarostatState> baro;
  // the barostats' screening network, one for every system of the engine:
  // it learns from the pooled exact attempts of all of them
  Surrogate net;
  Dev d{};
  std::vector<Allocation> allocs;
  cudaStream_t s0 = nullptr, s1 = nullptr, s2 = nullptr;
  cudaEvent_t fork = nullptr, listed = nullptr, join1 = nullptr, join2 = nullptr, t0 = nullptr, t1 = nullptr;
  std::map<int64_t, cudaGraphExec_t> graphs;
  int64_t step = 0;
  std::string error;
  int n_mesh_items = 0;
  std::vector<int> fft_x_sys;  // system of each x-pass work item
  bool coop_list = false;      // the list kernels run as one cooperative launch
  int cluster = 8;                 // atoms per cluster of the tile list (8 or 32), per engine
  bool prune = true;               // rebuilds drop tiles with no pair inside cutoff + skin
  std::vector<double> skin;        // per system, nm
  std::vector<int> mol_first, mol_count;  // per system: its molecules in d.mol_off
  double* mol_partials = nullptr;          // 9 per block of the molecular-offset kernel, systems one after another
  std::vector<int> mol_part_off;           // per system: its first block in mol_partials
  std::vector<double> sort_cell;   // per system, nm
  std::vector<double> inner_skin;  // per system, nm; <= 0: that system's inner list is its outer list
  int64_t list_grown = 0;          // times an overflowing list was grown and rebuilt
  unsigned char* active = nullptr;  // device: per system, whether an evaluation computes it
  std::vector<std::array<double, 9>> box_at_rebuild;  // per system: the box when a box change last asked for a rebuild
};

namespace {

int fail(mdb_engine* e, int status, const std::string& message) {
  if (e) e->error = message;
  return status;
}

#define CUDA_TRY(e, call)                                                                        \
  do {                                                                                           \
    cudaError_t err_ = (call);                                                                   \
    if (err_ != cudaSuccess) {                                                                   \
      return fail(e, MDB_ERR_DEVICE, std::string(#call) + ": " + cudaGetErrorString(err_));      \
    }                                                                                            \
  } while (0)

template <typename T>
int alloc(mdb_engine* e, const char* label, T*& out, size_t count) {
  out = nullptr;
  const size_t bytes = std::max<size_t>(1, count) * sizeof(T);
  void* p = nullptr;
  cudaError_t err = cudaMalloc(&p, bytes);
  if (err != cudaSuccess) return fail(e, MDB_ERR_DEVICE, std::string("cudaMalloc ") + label + ": " + cudaGetErrorString(err));
  err = cudaMemset(p, 0, bytes);
  if (err != cudaSuccess) {
    cudaFree(p);
    return fail(e, MDB_ERR_DEVICE, std::string("cudaMemset ") + label + ": " + cudaGetErrorString(err));
  }
  e->allocs.push_back({label, p, bytes});
  out = static_cast<T*>(p);
  return MDB_OK;
}

template <typename T>
int upload(mdb_engine* e, const char* label, T*& out, const std::vector<T>& host) {
  int st = alloc(e, label, out, host.size());
  if (st) return st;
  if (!host.empty()) CUDA_TRY(e, cudaMemcpy(out, host.data(), host.size() * sizeof(T), cudaMemcpyHostToDevice));
  return MDB_OK;
}

// Free one of the engine's allocations and forget it.
void release(mdb_engine* e, void* ptr) {
  if (!ptr) return;
  for (size_t k = 0; k < e->allocs.size(); ++k)
    if (e->allocs[k].ptr == ptr) {
      cudaFree(ptr);
      e->allocs.erase(e->allocs.begin() + long(k));
      return;
    }
}

// The tile-list arrays, sized by the systems' tile capacities (tile_cap):
// tiles, their interaction-mask words (C * C / 32 a tile), shifts and
// survival flags for the fill pass's raw list and for the list the pair
// kernel reads, and the inner list's copies.
int alloc_tile_list(mdb_engine* e) {
  Dev& d = e->d;
  const size_t n = size_t(d.tile_cap_total), words = size_t(e->cluster * e->cluster / 32);
  int st = MDB_OK;
  if ((st = alloc(e, "tiles", d.tiles, n))) return st;
  if ((st = alloc(e, "tile masks", d.masks, n * words))) return st;
  if ((st = alloc(e, "tile image shifts", d.tile_shift, n))) return st;
  if ((st = alloc(e, "raw tiles", d.raw_tiles, n))) return st;
  if ((st = alloc(e, "raw tile masks", d.raw_masks, n * words))) return st;
  if ((st = alloc(e, "raw tile shifts", d.raw_shift, n))) return st;
  if ((st = alloc(e, "tile survives", d.tile_alive, n))) return st;
  if (d.inner) {
    if ((st = alloc(e, "inner tiles", d.in_tiles, n))) return st;
    if ((st = alloc(e, "inner tile masks", d.in_masks, n * words))) return st;
    if ((st = alloc(e, "inner tile shifts", d.in_shift, n))) return st;
  }
  return MDB_OK;
}

long long to_fixed_host(double x) { return std::llround(x * 4294967296.0); }

// Position of a cell along the 3D Hilbert curve of side 2^bits: Skilling's
// axes-to-transpose conversion ("Programming the Hilbert curve", AIP Conf.
// Proc. 707, 381, 2004), then the transposed bits interleaved.
uint64_t hilbert_index(uint32_t x, uint32_t y, uint32_t z, int bits) {
  uint32_t X[3] = {x, y, z};
  const uint32_t M = 1u << (bits - 1);
  for (uint32_t Q = M; Q > 1; Q >>= 1) {
    const uint32_t P = Q - 1;
    for (int i = 0; i < 3; ++i) {
      if (X[i] & Q) {
        X[0] ^= P;
      } else {
        const uint32_t t = (X[0] ^ X[i]) & P;
        X[0] ^= t;
        X[i] ^= t;
      }
    }
  }
  for (int i = 1; i < 3; ++i) X[i] ^= X[i - 1];
  uint32_t t = 0;
  for (uint32_t Q = M; Q > 1; Q >>= 1)
    if (X[2] & Q) t ^= Q - 1;
  for (int i = 0; i < 3; ++i) X[i] ^= t;
  uint64_t h = 0;
  for (int b = bits - 1; b >= 0; --b)
    for (int i = 0; i < 3; ++i) h = (h << 1) | ((X[i] >> b) & 1u);
  return h;
}

// Hilbert order of the fractional cells: consecutive cells are neighbours, so
// 32 consecutive slots form a compact cluster and its bounding box is small.
std::vector<int> cell_order_map(const int* dim) {
  const int n = dim[0] * dim[1] * dim[2];
  int bits = 1;
  while ((1 << bits) < std::max({dim[0], dim[1], dim[2]})) ++bits;
  std::vector<std::pair<uint64_t, int>> keys(n);
  for (int x = 0; x < dim[0]; ++x)
    for (int y = 0; y < dim[1]; ++y)
      for (int z = 0; z < dim[2]; ++z) {
        const int id = (x * dim[1] + y) * dim[2] + z;
        keys[id] = {hilbert_index(uint32_t(x), uint32_t(y), uint32_t(z), bits), id};
      }
  std::sort(keys.begin(), keys.end());
  std::vector<int> map(n);
  for (int r = 0; r < n; ++r) map[keys[r].second] = r;
  return map;
}

// Every box-dependent field of one system's device constants.
void fill_box(const HostSystem& h, SysDev& S, bool keep_shift) {
  const double* B = h.box.data();
  double M[9];
  inverse_box(B, M);
  for (int i = 0; i < 9; ++i) {
    S.box_f[i] = float(B[i]);
    S.inv_f[i] = float(M[i]);
    S.box_fx[i] = to_fixed_host(B[i]);
    S.inv_fx[i] = to_fixed_host(M[i]);
  }
  S.triclinic = (B[3] != 0 || B[6] != 0 || B[7] != 0) ? 1 : 0;
  double widths[3];
  perpendicular_widths(B, widths);
  S.min_width = float(std::min({widths[0], widths[1], widths[2]}));
  // cells narrower than cutoff + list radius + 1 nm flag most tiles per-pair
  S.prune_per_pair = S.min_width < std::sqrt(S.cut2) + std::sqrt(S.list2) + 1.0f ? 1 : 0;
  // Pair coordinates: the folded extent plus one box stays below 2^31.
  const double ext = std::max({B[0] + std::fabs(B[3]) + std::fabs(B[6]), B[4] + std::fabs(B[7]), B[8]});
  int shift = int(std::floor(std::log2(std::ldexp(1.0, 30) / ext)));
  shift = std::min(shift, 30);
  if (!keep_shift || shift < S.pc_shift) S.pc_shift = shift;
  const double sc = std::ldexp(1.0, S.pc_shift);
  S.pc_inv = float(1.0 / sc);
  S.cut2u = float(std::ldexp(double(S.cut2), 2 * S.pc_shift));  // exact: a power-of-two scaling
  for (int i = 0; i < 9; ++i) S.pc_box[i] = int(std::llround(B[i] * sc));
  for (int k = 0; k < 3; ++k) {
    S.pc_half[k] = S.pc_box[k * 4] / 2;
    S.pc_inv_diag[k] = float(1.0 / S.pc_box[k * 4]);
  }
  // PME: u = r . (K o M)
  const int* K = h.grid.data();
  const double um[6] = {K[0] * M[0], K[0] * M[3], K[0] * M[6], K[1] * M[4], K[1] * M[7], K[2] * M[8]};
  for (int i = 0; i < 6; ++i) S.umat[i] = to_fixed_host(um[i]);
  for (int v = 0; v < 3; ++v)
    for (int u = 0; u < 3; ++u) S.umat_f[v * 3 + u] = float(K[u] * M[v * 3 + u]);
  const double vol = box_volume(B);
  S.pme_pref = float(kOne4PiEps0 * 2 * 3.14159265358979323846 / vol);
}

int request_rebuild(mdb_engine* e, int s);

int check_device_status(mdb_engine* e) {
  cudaError_t err = cudaStreamSynchronize(e->s0);
  if (err != cudaSuccess) return fail(e, MDB_ERR_DEVICE, std::string("device: ") + cudaGetErrorString(err));
  std::vector<int> flags(e->d.S), shake(e->d.S);
  CUDA_TRY(e, cudaMemcpy(flags.data(), e->d.err, sizeof(int) * e->d.S, cudaMemcpyDeviceToHost));
  int any = 0;
  for (int f : flags) any |= f;
  if (any & kErrTileCapacity) return fail(e, MDB_ERR_CAPACITY, "the cluster-pair tile list ran out of room");
  if (any & kErrTimeout) {
    // the list kernel's grid barrier gave up: its count holds the blocks that
    // arrived; clear it and the bit so the next list build starts afresh
    CUDA_TRY(e, cudaMemset(e->d.list_barrier, 0, 2 * sizeof(unsigned int)));
    for (int& f : flags) f &= ~kErrTimeout;
    CUDA_TRY(e, cudaMemcpy(e->d.err, flags.data(), sizeof(int) * e->d.S, cudaMemcpyHostToDevice));
    request_rebuild(e, -1);
    return fail(e, MDB_ERR_TIMEOUT, "a bounded device wait gave up");
  }
  if (any & kErrRange) return fail(e, MDB_ERR_RANGE, "a value left the fixed-point range: the run diverged");
  return MDB_OK;
}

// Sort, wrap and tile list: one cooperative launch when the device can, else
// the phase kernels one by one.
void list_kernels(mdb_engine* e, cudaStream_t st) {
  if (!(e->coop_list && launch_list(e->d, st))) {
    launch_rebuild_sort(e->d, st);
    launch_wrap(e->d, st);
    launch_rebuild_tiles(e->d, st);
  }
  launch_inner_prune(e->d, st);
}

// One step on three streams: the PME spread and transforms fork off at the
// start and run on a high-priority stream beside the list kernels (which
// return at once unless a rebuild or a prune is due); the gather and the
// listed terms, which write forces by slot, wait for the list; the pair kernel
// follows the list; all join before the integrator.
void launch_step(mdb_engine* e) {
  const Dev& d = e->d;
  cudaEventRecord(e->fork, e->s0);
  cudaStreamWaitEvent(e->s1, e->fork, 0);
  launch_pme_spread(d, e->s1);
  launch_pme_fft(d, false, e->s1);
  list_kernels(e, e->s0);
  cudaEventRecord(e->listed, e->s0);
  cudaStreamWaitEvent(e->s1, e->listed, 0);
  cudaStreamWaitEvent(e->s2, e->listed, 0);
  launch_pme_gather(d, e->s1);
  launch_listed(d, false, e->s2);
  launch_nonbonded(d, false, e->s0);
  cudaEventRecord(e->join1, e->s1);
  cudaEventRecord(e->join2, e->s2);
  cudaStreamWaitEvent(e->s0, e->join1, 0);
  cudaStreamWaitEvent(e->s0, e->join2, 0);
  launch_integrate(d, e->s0);
}

int run_steps(mdb_engine* e, int64_t steps) {
  if (steps <= 0) return MDB_OK;
  if (e->opt.flags & MDB_FLAG_NO_GRAPH) {
    for (int64_t k = 0; k < steps; ++k) launch_step(e);
    CUDA_TRY(e, cudaGetLastError());
  } else {
    auto it = e->graphs.find(steps);
    if (it == e->graphs.end()) {
      cudaGraph_t g = nullptr;
      CUDA_TRY(e, cudaStreamBeginCapture(e->s0, cudaStreamCaptureModeThreadLocal));
      for (int64_t k = 0; k < steps; ++k) launch_step(e);
      CUDA_TRY(e, cudaStreamEndCapture(e->s0, &g));
      cudaGraphExec_t exec = nullptr;
      // keep the captured streams' priorities (PME and listed above the pair kernel)
      CUDA_TRY(e, cudaGraphInstantiate(&exec, g, cudaGraphInstantiateFlagUseNodePriority));
      cudaGraphDestroy(g);
      it = e->graphs.emplace(steps, exec).first;
    }
    CUDA_TRY(e, cudaGraphLaunch(it->second, e->s0));
  }
  e->step += steps;
  return MDB_OK;
}

int request_rebuild(mdb_engine* e, int s) {
  std::vector<int> now(e->d.S, 0);
  CUDA_TRY(e, cudaMemcpy(now.data(), e->d.rebuild_now, sizeof(int) * e->d.S, cudaMemcpyDeviceToHost));
  if (s < 0) std::fill(now.begin(), now.end(), 1);
  else now[s] = 1;
  const int one = 1;
  CUDA_TRY(e, cudaMemcpy(e->d.rebuild_now, now.data(), sizeof(int) * e->d.S, cudaMemcpyHostToDevice));
  CUDA_TRY(e, cudaMemcpy(e->d.any_rebuild, &one, sizeof(int), cudaMemcpyHostToDevice));
  return MDB_OK;
}

// A list that needed more tiles than its system's capacity stopped the
// integrator (the halt word) at the step whose rebuild overflowed.  Grow every
// such system's capacity to half again what it needed (at least double),
// reallocate the list, drop the captured graphs (they hold the old arrays),
// clear the halt and the capacity bits, and ask for a rebuild of every system.
int grow_tile_list(mdb_engine* e) {
  Dev& d = e->d;
  CUDA_TRY(e, cudaStreamSynchronize(e->s0));
  CUDA_TRY(e, cudaStreamSynchronize(e->s1));
  CUDA_TRY(e, cudaStreamSynchronize(e->s2));
  std::vector<int> need(d.S), err(d.S);
  CUDA_TRY(e, cudaMemcpy(need.data(), d.tile_need, sizeof(int) * d.S, cudaMemcpyDeviceToHost));
  CUDA_TRY(e, cudaMemcpy(err.data(), d.err, sizeof(int) * d.S, cudaMemcpyDeviceToHost));
  long long total = 0;
  for (int s = 0; s < d.S; ++s) {
    SysDev& S = e->sd[s];
    const long long most = (long long)S.n_blocks * (S.n_blocks + 1) / 2;
    if (need[s] > S.tile_cap)
      S.tile_cap = int(std::min<long long>(most, std::max<long long>(need[s] + need[s] / 2, 2ll * S.tile_cap)));
    S.tile_off = int(total);
    total += S.tile_cap;
    err[s] &= ~kErrTileCapacity;
  }
  if (total > std::numeric_limits<int>::max()) return fail(e, MDB_ERR_CAPACITY, "the tile list cannot grow further");
  for (auto& g : e->graphs) cudaGraphExecDestroy(g.second);
  e->graphs.clear();
  for (void* p : {(void*)d.tiles, (void*)d.masks, (void*)d.tile_shift, (void*)d.raw_tiles, (void*)d.raw_masks,
                  (void*)d.raw_shift, (void*)d.tile_alive, (void*)d.in_tiles, (void*)d.in_masks, (void*)d.in_shift})
    release(e, p);
  d.tile_cap_total = int(total);
  if (const int st = alloc_tile_list(e)) return st;
  CUDA_TRY(e, cudaMemcpy(const_cast<SysDev*>(d.sys), e->sd.data(), sizeof(SysDev) * d.S, cudaMemcpyHostToDevice));
  CUDA_TRY(e, cudaMemcpy(d.err, err.data(), sizeof(int) * d.S, cudaMemcpyHostToDevice));
  CUDA_TRY(e, cudaMemset(d.halt, 0, sizeof(int)));
  e->list_grown += 1;
  return request_rebuild(e, -1);
}

// Whether a list overflowed (the integrator has stopped): one 4-byte read.
int list_halted(mdb_engine* e, bool* halted) {
  int h = 0;
  CUDA_TRY(e, cudaMemcpyAsync(&h, e->d.halt, sizeof(int), cudaMemcpyDeviceToHost, e->s0));
  CUDA_TRY(e, cudaStreamSynchronize(e->s0));
  *halted = h != 0;
  return MDB_OK;
}

int build_engine(mdb_engine* e, int n, const mdb_system_desc* systems, const mdb_state_desc* states,
                 const mdb_run_options* options) {
  e->opt = *options;
  if (e->opt.max_batch <= 0) e->opt.max_batch = 100;
  if (!(e->opt.time_step > 0)) return fail(e, MDB_ERR_INVALID_ARGUMENT, "time_step must be positive");
  const double default_skin = e->opt.verlet_skin < 0 ? 0.15 : e->opt.verlet_skin;
  e->skin.assign(n, default_skin);
  e->sort_cell.assign(n, kCellWidth);
  e->inner_skin.assign(n, kDefaultInnerSkin);
  e->cluster = kDefaultCluster;
  if (e->opt.tuning) {
    bool shape_set = false, prune_set = false;
    for (int s = 0; s < n; ++s) {
      if (e->opt.tuning[s].verlet_skin > 0) e->skin[s] = e->opt.tuning[s].verlet_skin;
      if (e->opt.tuning[s].sort_cell > 0) e->sort_cell[s] = e->opt.tuning[s].sort_cell;
      if (e->opt.tuning[s].inner_skin != 0) e->inner_skin[s] = e->opt.tuning[s].inner_skin;
      const int shape = e->opt.tuning[s].tile_atoms;
      if (shape != 0 && shape != 8 && shape != 32)
        return fail(e, MDB_ERR_INVALID_ARGUMENT, "tile_atoms must be 8 or 32");
      if (shape && !shape_set) {  // one tile shape per engine: the first system's that names one
        e->cluster = shape;
        shape_set = true;
      }
      const int prune = e->opt.tuning[s].prune_tiles;
      if (prune < 0 || prune > 2) return fail(e, MDB_ERR_INVALID_ARGUMENT, "prune_tiles must be 0, 1 or 2");
      if (prune && !prune_set) {
        e->prune = prune == 1;
        prune_set = true;
      }
    }
    e->opt.tuning = nullptr;  // the caller's array is not kept
  }
  // the systems are checked on the host first, so a caller learns what is
  // wrong with its input (the reference's named errors) on any machine
  e->hs.resize(n);
  for (int s = 0; s < n; ++s) {
    std::string msg;
    const int st = prepare_system(systems[s], states[s], e->opt, e->hs[s], msg);
    if (st) return fail(e, st, n > 1 ? "system " + std::to_string(s) + ": " + msg : msg);
  }
  e->box_at_rebuild.resize(n);
  for (int s = 0; s < n; ++s) e->box_at_rebuild[s] = e->hs[s].box;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
    return fail(e, MDB_ERR_NO_DEVICE, "no CUDA device is visible");
  e->device = e->opt.device;
  CUDA_TRY(e, cudaSetDevice(e->device));
  // run options (integrate.ts:170 packStepParams)
  RunDev& R = e->run;
  R.dt = float(e->opt.time_step);
  R.velocity_scale = float(std::exp(-e->opt.time_step * e->opt.friction));
  R.noise_scale = float(std::sqrt(1.0 - std::exp(-2.0 * e->opt.time_step * e->opt.friction)));
  R.kt = float(kBoltzmann * e->opt.temperature);
  R.tolerance = float(e->opt.constraint_tolerance > 0 ? e->opt.constraint_tolerance : 1e-6);
  R.seed = e->opt.seed;
  R.integrator = e->opt.integrator;
  R.draw_noise = (R.noise_scale > 0 && e->opt.integrator == MDB_INTEGRATOR_LFMIDDLE) ? 1 : 0;
  R.always_rebuild = (e->opt.flags & MDB_FLAG_ALWAYS_REBUILD) ? 1 : 0;

  // ---- layout ----
  e->sd.resize(n);
  e->baro.resize(n);
  std::vector<long long> px, py, pz;
  std::vector<float> vx, vy, vz, invm;
  std::vector<int> atom_sys, slot_sys, block_sys, cell_sys, cell_map;
  std::vector<float4> prm_atom;
  std::vector<int2> excl;
  std::vector<int> excl_sys;
  std::vector<BondDev> bonds;
  std::vector<AngleDev> angles;
  std::vector<TorsionDev> torsions;
  std::vector<ExceptionDev> exceptions;
  std::vector<RestraintDev> restraints;
  std::vector<float> moduli;
  std::vector<float2> twiddles;
  std::vector<FftWork> wz, wy, wx;
  std::vector<UnitDev> units;
  std::vector<int> iblk_sys, iblk_unit0, iblk_nunit, iblk_atom0, iblk_natom, iatom;
  int atoms = 0, slots = 0, blocks = 0, cells = 0, tiles = 0, units_n = 0, iblk = 0;
  long long grid_pts = 0, cgrid_pts = 0;
  int smem_z = 0, smem_y = 0, smem_x = 0, smem_p = 0;
  std::vector<FftWork> wp;
  const float sq = float(std::sqrt(kOne4PiEps0));
  for (int s = 0; s < n; ++s) {
    HostSystem& h = e->hs[s];
    SysDev& S = e->sd[s];
    std::memset(&S, 0, sizeof(S));
    S.n_atoms = h.n;
    S.atom_off = atoms;
    S.n_slots = (h.n + 31) / 32 * 32;
    // clusters of the tile list; trailing ones may be empty so that cluster I
    // of every system starts at slot I * cluster (their bounding boxes are
    // inverted, so no tile ever includes them)
    S.n_blocks = S.n_slots / e->cluster;
    S.slot_off = slots;
    S.block_off = blocks;
    double widths[3];
    perpendicular_widths(h.box.data(), widths);
    for (int k = 0; k < 3; ++k) S.cdim[k] = std::max(1, int(std::floor(widths[k] / e->sort_cell[s])));
    S.n_cells = S.cdim[0] * S.cdim[1] * S.cdim[2];
    S.cell_off = cells;
    const long long all_pairs = (long long)S.n_blocks * (S.n_blocks + 1) / 2;
    const long long row_cap = e->opt.tile_row_capacity > 0 ? e->opt.tile_row_capacity : row_cap_for(e->cluster);
    S.tile_cap = int(std::min<long long>(all_pairs, (long long)S.n_blocks * row_cap));
    S.tile_off = tiles;
    S.energy_base = s * kECount;
    S.cut2 = float(h.cutoff * h.cutoff);
    const double skin = e->skin[s];
    S.list2 = float((h.cutoff + skin) * (h.cutoff + skin));
    S.half_skin2 = float(0.25 * skin * skin);
    // a system without an inner skin keeps every outer tile and is never re-pruned
    const double inner = e->inner_skin[s] > 0 ? std::min(e->inner_skin[s], skin) : skin;
    S.inner2 = float((h.cutoff + inner) * (h.cutoff + inner));
    S.half_inner2 = e->inner_skin[s] > 0 ? float(0.25 * inner * inner) : 3.0e38f;
    S.alpha = float(h.alpha);
    S.alpha_2_sqrtpi = float(h.alpha * 2.0 / std::sqrt(3.14159265358979323846));
    S.gauss_scale = float(-h.alpha * h.alpha / std::log(2.0));
    S.exp_scale = float(-1.0 / (4 * h.alpha * h.alpha));
    S.com_freq = h.com_frequency;
    S.total_mass = h.total_mass;
    for (int k = 0; k < 3; ++k) S.grid[k] = h.grid[k];
    S.kzh = h.grid[2] / 2 + 1;
    S.grid_off = grid_pts;
    S.cgrid_off = cgrid_pts;
    S.pc_shift = 0;
    fill_box(h, S, false);
    grid_pts += (long long)h.grid[0] * h.grid[1] * h.grid[2];
    cgrid_pts += (long long)h.grid[0] * h.grid[1] * S.kzh;
    S.mod_off = int(moduli.size());
    for (int k = 0; k < 3; ++k)
      for (double m : bspline_moduli(h.grid[k])) moduli.push_back(float(m));
    for (int k = 0; k < 3; ++k) {
      plan_radices(h.grid[k], S.radices[k], &S.nradix[k]);
      S.tw_off[k] = int(twiddles.size());
      for (int j = 0; j < h.grid[k]; ++j) {
        const double a = -2 * 3.14159265358979323846 * j / h.grid[k];
        twiddles.push_back(make_float2(float(std::cos(a)), float(std::sin(a))));
      }
    }
    // FFT work items
    const int Kx = h.grid[0], Ky = h.grid[1], Kz = h.grid[2];
    // lines per z-pass CTA: at most 2048 points in shared memory, and enough
    // CTAs (about two per SM) that a small mesh still fills the device
    const int lines = std::max(1, std::min(2048 / Kz, (Kx * Ky + 295) / 296));
    for (int l = 0; l < Kx * Ky; l += lines) wz.push_back({s, l, 0, std::min(lines, Kx * Ky - l)});
    smem_z = std::max(smem_z, 2 * lines * Kz * int(sizeof(float2)));
    for (int x = 0; x < Kx; ++x)
      for (int k = 0; k < S.kzh; k += kFftTile) wy.push_back({s, x, k, std::min(kFftTile, S.kzh - k)});
    smem_y = std::max(smem_y, 2 * kFftTile * Ky * int(sizeof(float2)));
    for (int y = 0; y < Ky; ++y)
      for (int k = 0; k < S.kzh; k += kFftTile) {
        wx.push_back({s, y, k, std::min(kFftTile, S.kzh - k)});
        e->fft_x_sys.push_back(s);
      }
    smem_x = std::max(smem_x, (2 * kFftTile + 1) * Kx * int(sizeof(float2)));  // two tiles of lines, twiddles
    for (int x = 0; x < Kx; ++x) wp.push_back({s, x, 0, 1});
    smem_p = std::max(smem_p, (2 * Ky * Kz + Ky + Kz) * int(sizeof(float2)));  // two planes, twiddles

    // atoms
    const double* pos = states[s].positions;
    const double* vel = states[s].velocities;
    for (int a = 0; a < h.n; ++a) {
      px.push_back(to_fixed_host(pos[3 * a]));
      py.push_back(to_fixed_host(pos[3 * a + 1]));
      pz.push_back(to_fixed_host(pos[3 * a + 2]));
      vx.push_back(vel ? float(vel[3 * a]) : 0.f);
      vy.push_back(vel ? float(vel[3 * a + 1]) : 0.f);
      vz.push_back(vel ? float(vel[3 * a + 2]) : 0.f);
      invm.push_back(h.mass[a] == 0 ? 0.f : float(1.0 / h.mass[a]));
      atom_sys.push_back(s);
      prm_atom.push_back(make_float4(float(h.charge[a]) * sq, float(0.5 * h.sigma[a]),
                                     float(std::sqrt(24.0 * h.epsilon[a])), float(h.charge[a])));
    }
    for (int k = 0; k < S.n_slots; ++k) slot_sys.push_back(s);
    for (int k = 0; k < S.n_blocks; ++k) block_sys.push_back(s);
    for (int k = 0; k < S.n_cells; ++k) cell_sys.push_back(s);
    const std::vector<int> mm = cell_order_map(S.cdim);
    cell_map.insert(cell_map.end(), mm.begin(), mm.end());

    // listed terms, global indices
    const int off = atoms;
    for (auto b : h.bonds) { b.a += off; b.b += off; b.sys = s; bonds.push_back(b); }
    for (auto a : h.angles) { a.a += off; a.b += off; a.c += off; a.sys = s; angles.push_back(a); }
    for (auto t : h.torsions) { t.a += off; t.b += off; t.c += off; t.d += off; t.sys = s; torsions.push_back(t); }
    for (size_t k = 0; k < h.ep1.size(); ++k) {
      ExceptionDev x;
      x.a = h.ep1[k] + off;
      x.b = h.ep2[k] + off;
      x.sys = s;
      x.qq_particles = float(kOne4PiEps0 * h.charge[h.ep1[k]] * h.charge[h.ep2[k]]);
      x.qq_own = float(kOne4PiEps0 * h.eqq[k]);
      x.sigma = float(h.esig[k]);
      x.eps4 = float(4 * h.eeps[k]);
      exceptions.push_back(x);
      excl.push_back(make_int2(h.ep1[k] + off, h.ep2[k] + off));
      excl_sys.push_back(s);
    }
    for (size_t k = 0; k < h.rparticle.size(); ++k)
      restraints.push_back({h.rparticle[k] + off, s, float(h.rk[k]), to_fixed_host(h.rx0[k]),
                            to_fixed_host(h.ry0[k]), to_fixed_host(h.rz0[k])});

    // integration units: SETTLE waters, SHAKE clusters, free atoms
    std::vector<UnitDev> su;
    for (const auto& w : h.settle) {
      UnitDev u{};
      u.kind = kUnitSettle;
      u.sys = s;
      u.na = 3;
      u.nc = 0;
      u.atom[0] = w.central + off;
      u.atom[1] = w.first + off;
      u.atom[2] = w.second + off;
      u.dist[0] = w.d1;
      u.dist[1] = w.d2;
      su.push_back(u);
    }
    for (const auto& cl : h.shake) {
      UnitDev u{};
      u.kind = kUnitShake;
      u.sys = s;
      u.na = int(cl.atoms.size());
      u.nc = int(cl.constraints.size());
      for (int k = 0; k < u.na; ++k) u.atom[k] = cl.atoms[k] + off;
      for (int k = 0; k < u.nc; ++k) {
        const int c = cl.constraints[k];
        u.ci[k] = (unsigned char)(std::find(cl.atoms.begin(), cl.atoms.end(), h.cp1[c]) - cl.atoms.begin());
        u.cj[k] = (unsigned char)(std::find(cl.atoms.begin(), cl.atoms.end(), h.cp2[c]) - cl.atoms.begin());
        u.dist[k] = float(h.cdist[c]);
      }
      // An X-H_n star (one atom in every constraint, nc = na - 1 <= 3) is
      // reordered to centre first and spoke c at position c + 1.
      if (u.nc >= 1 && u.nc <= 3 && u.na == u.nc + 1) {
        for (int centre : {int(u.ci[0]), int(u.cj[0])}) {
          bool star = true;
          for (int k = 0; k < u.nc; ++k) star &= u.ci[k] == centre || u.cj[k] == centre;
          if (!star) continue;
          int atom[kMaxClusterAtoms];
          atom[0] = u.atom[centre];
          for (int k = 0; k < u.nc; ++k) {
            atom[k + 1] = u.atom[u.ci[k] == centre ? u.cj[k] : u.ci[k]];
            u.ci[k] = 0;
            u.cj[k] = (unsigned char)(k + 1);
          }
          for (int k = 0; k < u.na; ++k) u.atom[k] = atom[k];
          u.kind = kUnitStar;
          break;
        }
      }
      su.push_back(u);
    }
    for (int a : h.free_atoms) {
      UnitDev u{};
      u.kind = kUnitFree;
      u.sys = s;
      u.na = 1;
      u.atom[0] = a + off;
      su.push_back(u);
    }
    S.unit_off = units_n;
    S.n_units = int(su.size());
    S.iblk_off = iblk;
    for (int u0 = 0; u0 < S.n_units; u0 += kIntegrateUnits) {
      const int nu = std::min(kIntegrateUnits, S.n_units - u0);
      iblk_sys.push_back(s);
      iblk_unit0.push_back(units_n + u0);
      iblk_nunit.push_back(nu);
      iblk_atom0.push_back(int(iatom.size()));
      int entries = 0;
      for (int k = 0; k < nu; ++k) {
        UnitDev& u = su[u0 + k];
        u.base = entries;
        for (int j = 0; j < u.na; ++j) iatom.push_back(u.atom[j]);
        entries += u.na;
      }
      iblk_natom.push_back(entries);  // <= kIntegrateTable: na <= kMaxClusterAtoms
      ++iblk;
    }
    S.n_iblk = iblk - S.iblk_off;
    units.insert(units.end(), su.begin(), su.end());
    units_n += S.n_units;

    atoms += h.n;
    slots += S.n_slots;
    blocks += S.n_blocks;
    cells += S.n_cells;
    tiles += S.tile_cap;
    e->baro[s].volume_scale = 0.01 * box_volume(h.box.data());
    e->baro[s].step = 0;
  }

  e->net.target = std::max(0, e->opt.surrogate_attempts);

  // ---- device tables ----
  Dev& d = e->d;
  d.S = n;
  d.run = e->run;
  d.n_atoms = atoms;
  d.n_slots = slots;
  d.n_blocks = blocks;
  d.tile_cap_total = tiles;
  d.cluster = e->cluster;
  d.prune = e->prune ? 1 : 0;
  d.inner = 0;
  for (int s = 0; s < n; ++s) d.inner |= e->inner_skin[s] > 0 ? 1 : 0;
  d.any_triclinic = 0;
  for (int s = 0; s < n; ++s) d.any_triclinic |= e->sd[s].triclinic ? 1 : 0;
  d.n_cells = cells;
  d.n_units = units_n;
  d.n_iblk = iblk;
  int st = MDB_OK;
  SysDev* sys_dev = nullptr;
#define TRY(x) do { st = (x); if (st) return st; } while (0)
  TRY(upload(e, "system constants", sys_dev, e->sd));
  d.sys = sys_dev;
  TRY(upload(e, "positions.x", d.px, px));
  TRY(upload(e, "positions.y", d.py, py));
  TRY(upload(e, "positions.z", d.pz, pz));
  TRY(upload(e, "velocities.x", d.vx, vx));
  TRY(upload(e, "velocities.y", d.vy, vy));
  TRY(upload(e, "velocities.z", d.vz, vz));
  TRY(alloc(e, "residual.x", d.rx, atoms));
  TRY(alloc(e, "residual.y", d.ry, atoms));
  TRY(alloc(e, "residual.z", d.rz, atoms));
  TRY(upload(e, "inverse masses", d.invm, invm));
  TRY(upload(e, "atom system", d.atom_sys, atom_sys));
  TRY(alloc(e, "rank", d.rank, atoms));
  TRY(alloc(e, "cell of atom", d.cell_of, atoms));
  TRY(alloc(e, "list reference.x", d.refx, atoms));
  TRY(alloc(e, "list reference.y", d.refy, atoms));
  TRY(alloc(e, "list reference.z", d.refz, atoms));
  TRY(alloc(e, "volume move backup.x", d.bx, atoms));
  TRY(alloc(e, "volume move backup.y", d.by, atoms));
  TRY(alloc(e, "volume move backup.z", d.bz, atoms));
  float4* prm_atom_dev = nullptr;
  TRY(upload(e, "pair parameters by atom", prm_atom_dev, prm_atom));
  d.prm_atom = prm_atom_dev;
  TRY(alloc(e, "order", d.order, slots));
  d.spread_sorted = spread_by_slot(int(slots)) ? 1 : 0;
  TRY(alloc(e, "spread order", d.spread_atom, d.spread_sorted ? slots : 1));
  TRY(alloc(e, "scatter order", d.tmp_order, slots));
  TRY(alloc(e, "pair coordinates", d.pc, slots));
  TRY(alloc(e, "pair parameters", d.prm, slots));
  TRY(alloc(e, "forces.x", d.fx, slots));
  TRY(alloc(e, "forces.y", d.fy, slots));
  TRY(alloc(e, "forces.z", d.fz, slots));
  int* tmp_i = nullptr;
  TRY(upload(e, "slot system", tmp_i, slot_sys));
  d.slot_sys = tmp_i;
  TRY(alloc(e, "block bounds lo", d.bb_lo, blocks));
  TRY(alloc(e, "block bounds hi", d.bb_hi, blocks));
  if (e->cluster < 32) {
    TRY(alloc(e, "super-cluster bounds lo", d.sb_lo, blocks / (32 / e->cluster)));
    TRY(alloc(e, "super-cluster bounds hi", d.sb_hi, blocks / (32 / e->cluster)));
  } else {
    d.sb_lo = d.bb_lo;
    d.sb_hi = d.bb_hi;
  }

  TRY(alloc(e, "tile row count", d.tile_cnt, blocks));
  TRY(alloc(e, "tile row start", d.tile_start, blocks));
  TRY(upload(e, "block system", tmp_i, block_sys));
  d.block_sys = tmp_i;
  TRY(alloc(e, "cell count", d.cell_cnt, cells));
  TRY(alloc(e, "cell start", d.cell_start, cells));
  TRY(alloc(e, "cell cursor", d.cell_cur, cells));
  TRY(upload(e, "cell system", tmp_i, cell_sys));
  d.cell_sys = tmp_i;
  TRY(upload(e, "cell order map", tmp_i, cell_map));
  d.cell_map = tmp_i;
  if (const int st_ = alloc_tile_list(e)) return st_;
  TRY(alloc(e, "surviving tiles per row", d.row_alive, blocks));
  TRY(alloc(e, "surviving tiles start", d.alive_start, blocks));
  TRY(alloc(e, "fold translations", d.fold, slots));
  TRY(alloc(e, "inner prune flag", d.prune_flag, n));
  TRY(alloc(e, "inner prune now", d.prune_now, n));
  TRY(alloc(e, "any inner prune", d.any_prune, 1));
  TRY(alloc(e, "inner prune count", d.prune_count, n));
  TRY(alloc(e, "inner prune ticket", d.inner_ticket, 1));
  if (d.inner) {
    TRY(alloc(e, "inner tile count", d.in_count, n));
    TRY(alloc(e, "inner tile prefix", d.in_prefix, n + 1));
    TRY(alloc(e, "prune reference.x", d.prx, atoms));
    TRY(alloc(e, "prune reference.y", d.pry, atoms));
    TRY(alloc(e, "prune reference.z", d.prz, atoms));
    TRY(alloc(e, "prune cluster bounds lo", d.cb_lo, blocks));
    TRY(alloc(e, "prune cluster bounds hi", d.cb_hi, blocks));
  }
  TRY(alloc(e, "tile count", d.tile_count, n));
  TRY(alloc(e, "tile need", d.tile_need, n));
  TRY(alloc(e, "list halt", d.halt, 1));
  TRY(alloc(e, "evaluated systems", e->active, n));
  d.active = nullptr;
  TRY(alloc(e, "tile prefix", d.tile_prefix, n + 1));
  TRY(alloc(e, "rebuild flag", d.rebuild_flag, n));
  TRY(alloc(e, "rebuild now", d.rebuild_now, n));
  TRY(alloc(e, "any rebuild", d.any_rebuild, 1));
  TRY(alloc(e, "status", d.err, n));

  TRY(alloc(e, "rebuild count", d.rebuild_count, n));
  TRY(alloc(e, "launch ticket", d.global_ticket, 1));
  TRY(alloc(e, "list grid barrier", d.list_barrier, 2));
  int2* ex_dev = nullptr;
  TRY(upload(e, "exclusions", ex_dev, excl));
  d.excl = ex_dev;
  TRY(upload(e, "exclusion system", tmp_i, excl_sys));
  d.excl_sys = tmp_i;
  d.n_excl = int(excl.size());
  BondDev* b_dev = nullptr;
  AngleDev* a_dev = nullptr;
  TorsionDev* t_dev = nullptr;
  ExceptionDev* x_dev = nullptr;
  RestraintDev* r_dev = nullptr;
  TRY(upload(e, "bonds", b_dev, bonds));
  TRY(upload(e, "angles", a_dev, angles));
  TRY(upload(e, "torsions", t_dev, torsions));
  TRY(upload(e, "exceptions", x_dev, exceptions));
  TRY(upload(e, "restraints", r_dev, restraints));
  d.bonds = b_dev; d.n_bonds = int(bonds.size());
  d.angles = a_dev; d.n_angles = int(angles.size());
  d.torsions = t_dev; d.n_torsions = int(torsions.size());
  d.exceptions = x_dev; d.n_exceptions = int(exceptions.size());
  d.restraints = r_dev; d.n_restraints = int(restraints.size());
  TRY(alloc(e, "pme charge grid", d.qgrid, size_t(grid_pts)));
  TRY(alloc(e, "pme spectrum", d.cgrid, size_t(cgrid_pts)));
  TRY(alloc(e, "pme potential", d.phi, size_t(grid_pts)));
  float* mod_dev = nullptr;
  float2* tw_dev = nullptr;
  TRY(upload(e, "pme moduli", mod_dev, moduli));
  TRY(upload(e, "fft twiddles", tw_dev, twiddles));
  d.moduli = mod_dev;
  d.twiddles = tw_dev;
  TRY(alloc(e, "pme energy partials", d.mesh_partial, wx.size()));
  TRY(alloc(e, "pme virial partials", d.mesh_virial, wx.size() * 6));
  FftWork* w_dev = nullptr;
  TRY(upload(e, "fft z work", w_dev, wz));
  d.fft_z = w_dev; d.n_fft_z = int(wz.size());
  TRY(upload(e, "fft y work", w_dev, wy));
  d.fft_y = w_dev; d.n_fft_y = int(wy.size());
  TRY(upload(e, "fft x work", w_dev, wx));
  d.fft_x = w_dev; d.n_fft_x = int(wx.size());
  int max_kx = 1;
  for (const SysDev& S : e->sd) max_kx = std::max(max_kx, S.grid[0]);
  d.influence_stride = kFftTile * max_kx;
  TRY(alloc(e, "pme influence function", d.influence, wx.size() * size_t(d.influence_stride)));
  TRY(upload(e, "fft plane work", w_dev, wp));
  d.fft_p = w_dev; d.n_fft_p = int(wp.size());
  // a whole x-plane in shared memory, twice, when every system's fits
  d.fft_planes = smem_p <= kPlaneSmemLimit ? 1 : 0;
  e->n_mesh_items = int(wx.size());
  TRY(alloc(e, "energies", d.energy, size_t(n) * kECount));
  {
    std::vector<int> mol_off{0}, mol_atoms;
    e->mol_first.assign(n, 0);
    e->mol_count.assign(n, 0);
    int base = 0;
    for (int s = 0; s < n; ++s) {
      e->mol_first[s] = int(mol_off.size()) - 1;
      e->mol_count[s] = int(e->hs[s].molecules.size());
      for (const auto& m : e->hs[s].molecules) {
        for (int a : m) mol_atoms.push_back(base + a);
        mol_off.push_back(int(mol_atoms.size()));
      }
      base += e->hs[s].n;
    }
    int* tmp = nullptr;
    TRY(upload(e, "molecule offsets", tmp, mol_off));
    d.mol_off = tmp;
    TRY(upload(e, "molecule atoms", tmp, mol_atoms));
    d.mol_atoms = tmp;
    int total_blocks = 0;
    e->mol_part_off.assign(n, 0);
    for (int s = 0; s < n; ++s) {
      e->mol_part_off[s] = total_blocks;
      total_blocks += molecular_offset_blocks(e->mol_count[s]);
    }
    TRY(alloc(e, "molecular virial partials", e->mol_partials, size_t(total_blocks) * 9));
  }
  UnitDev* u_dev = nullptr;
  TRY(upload(e, "integration units", u_dev, units));
  d.units = u_dev;
  TRY(upload(e, "integrate block system", tmp_i, iblk_sys));
  d.iblk_sys = tmp_i;
  TRY(upload(e, "integrate block unit", tmp_i, iblk_unit0));
  d.iblk_unit0 = tmp_i;
  TRY(upload(e, "integrate block count", tmp_i, iblk_nunit));
  d.iblk_nunit = tmp_i;
  TRY(upload(e, "integrate block table start", tmp_i, iblk_atom0));
  d.iblk_atom0 = tmp_i;
  TRY(upload(e, "integrate block table size", tmp_i, iblk_natom));
  d.iblk_natom = tmp_i;
  TRY(upload(e, "integrate block table", tmp_i, iatom));
  d.iatom = tmp_i;
  TRY(alloc(e, "momentum partials", d.mom_partial, size_t(iblk) * 3));
  TRY(alloc(e, "com velocity", d.vcom, n));
  std::vector<long long> steps(n);
  for (int s = 0; s < n; ++s) steps[s] = states[s].step;
  TRY(upload(e, "step", d.step, steps));
  TRY(alloc(e, "done count", d.done_count, n));
  TRY(alloc(e, "constraint failures", d.shake_failures, n));
#undef TRY
  e->step = states[0].step;
  set_pme_smem(smem_z, smem_y, smem_x, d.fft_planes ? smem_p : 0);

  // PME and the listed terms run beside the pair kernel at the highest
  // priority: their small, latency-bound grids take SMs as pair blocks
  // retire.  A large batch keeps every SM busy whatever runs first, and there
  // equal priorities measured 0.7% faster (64-system ensemble, 3.240 against
  // 3.262 ms per step).
  int least = 0, greatest = 0;
  CUDA_TRY(e, cudaDeviceGetStreamPriorityRange(&least, &greatest));
  const int side = d.S > 1 && d.n_slots >= (1 << 18) ? least : greatest;
  CUDA_TRY(e, cudaStreamCreateWithFlags(&e->s0, cudaStreamNonBlocking));
  CUDA_TRY(e, cudaStreamCreateWithPriority(&e->s1, cudaStreamNonBlocking, side));
  CUDA_TRY(e, cudaStreamCreateWithPriority(&e->s2, cudaStreamNonBlocking, side));
  CUDA_TRY(e, cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming));
  CUDA_TRY(e, cudaEventCreateWithFlags(&e->join1, cudaEventDisableTiming));
  CUDA_TRY(e, cudaEventCreateWithFlags(&e->join2, cudaEventDisableTiming));
  CUDA_TRY(e, cudaEventCreateWithFlags(&e->listed, cudaEventDisableTiming));
  CUDA_TRY(e, cudaEventCreate(&e->t0));
  CUDA_TRY(e, cudaEventCreate(&e->t1));
  CUDA_TRY(e, cudaDeviceSynchronize());

  launch_influence(e->d, -1, e->s0);
  // first list and the first COM velocity, by the phase kernels (a list that
  // overflows its starting capacity is grown and built again)
  if (const int st = request_rebuild(e, -1)) return st;
  for (int attempt = 0;; ++attempt) {
    launch_rebuild_sort(e->d, e->s0);
    launch_wrap(e->d, e->s0);
    launch_rebuild_tiles(e->d, e->s0);
    launch_inner_prune(e->d, e->s0);
    CUDA_TRY(e, cudaGetLastError());
    bool halted = false;
    if (const int st = list_halted(e, &halted)) return st;
    if (!halted || attempt == 4) break;
    if (const int st = grow_tile_list(e)) return st;
  }
  // the slot-ordered spread's copy of the order, until the first step writes it
  if (e->d.spread_sorted)
    CUDA_TRY(e, cudaMemcpyAsync(e->d.spread_atom, e->d.order, sizeof(int) * size_t(e->d.n_slots),
                                cudaMemcpyDeviceToDevice, e->s0));
  launch_momentum(e->d, e->s0);
  CUDA_TRY(e, cudaGetLastError());
  int status = check_device_status(e);
  if (status) return status;

  // One cooperative launch for the list kernels, if the device has
  // cooperative launch and a stream capture accepts it.
  if (prepare_list_kernel(e->device) > 0 && !(e->opt.flags & MDB_FLAG_NO_GRAPH)) {
    cudaGraph_t g = nullptr;
    bool ok = cudaStreamBeginCapture(e->s0, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    ok = launch_list(d, e->s0) && ok;
    ok = (cudaStreamEndCapture(e->s0, &g) == cudaSuccess) && ok;
    cudaGraphExec_t exec = nullptr;
    ok = ok && g && cudaGraphInstantiate(&exec, g, 0) == cudaSuccess;
    if (exec) cudaGraphExecDestroy(exec);
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();  // a refused probe leaves no sticky error behind
    e->coop_list = ok;
  } else if (prepare_list_kernel(e->device) > 0) {
    e->coop_list = true;
  }
  if (e->opt.flags & MDB_FLAG_PHASE_LAUNCHES) e->coop_list = false;
  // A large batch rebuilds some system's list nearly every step; its search
  // phases then want the full grids of separate launches more than the
  // cooperative kernel's two blocks per SM (64-system ensemble, 627k atoms:
  // 3.51 against 3.56 ms per step), and a step of milliseconds hides the
  // thirteen launches.  Single systems and small batches keep the one launch.
  if (d.S > 1 && d.n_slots >= (1 << 18)) e->coop_list = false;
  return MDB_OK;
}

// Energies by group (and the virials) of several systems from one evaluation
// of the whole engine -- the systems' terms come out of the same launches --
// and, for the first of them, the forces.  `kinetic`: also the kinetic energy
// from the velocities as they are.
int evaluate_many(mdb_engine* e, const std::vector<int>& systems, double* forces, mdb_energies* out,
                  bool kinetic) {
  const Dev& d = e->d;
  CUDA_TRY(e, cudaMemsetAsync(d.energy, 0, sizeof(unsigned long long) * d.S * kECount, e->s0));
  // the list first: one that overflows is grown and built again before any force
  for (int attempt = 0;; ++attempt) {
    list_kernels(e, e->s0);
    bool halted = false;
    if (const int st = list_halted(e, &halted)) return st;
    if (!halted || attempt == 4) break;
    if (const int st = grow_tile_list(e)) return st;
  }
  // the force kernels skip the systems not asked for
  Dev dv = d;
  if (int(systems.size()) < d.S) {
    std::vector<unsigned char> on(d.S, 0);
    for (int s : systems) on[s] = 1;
    CUDA_TRY(e, cudaMemcpyAsync(e->active, on.data(), d.S, cudaMemcpyHostToDevice, e->s0));
    CUDA_TRY(e, cudaStreamSynchronize(e->s0));  // `on` is pageable host memory
    dv.active = e->active;
  }
  launch_pme(dv, true, e->s0);
  launch_listed(dv, true, e->s0);
  launch_nonbonded(dv, true, e->s0);
  CUDA_TRY(e, cudaGetLastError());
  int st = check_device_status(e);
  if (st) return st;
  if (out) {
    for (int s : systems)
      launch_molecular_offsets(d, e->mol_first[s], e->mol_count[s], e->sd[s].slot_off,
                               e->mol_partials + size_t(e->mol_part_off[s]) * 9, e->s0);
    CUDA_TRY(e, cudaGetLastError());
    CUDA_TRY(e, cudaStreamSynchronize(e->s0));  // s0 does not order with the legacy stream
  }
  if (forces && !systems.empty()) {
    const SysDev& S = e->sd[systems[0]];
    std::vector<unsigned long long> f[3];
    std::vector<int> order(S.n_slots);
    for (auto& v : f) v.resize(S.n_slots);
    CUDA_TRY(e, cudaMemcpy(f[0].data(), d.fx + S.slot_off, sizeof(long long) * S.n_slots, cudaMemcpyDeviceToHost));
    CUDA_TRY(e, cudaMemcpy(f[1].data(), d.fy + S.slot_off, sizeof(long long) * S.n_slots, cudaMemcpyDeviceToHost));
    CUDA_TRY(e, cudaMemcpy(f[2].data(), d.fz + S.slot_off, sizeof(long long) * S.n_slots, cudaMemcpyDeviceToHost));
    CUDA_TRY(e, cudaMemcpy(order.data(), d.order + S.slot_off, sizeof(int) * S.n_slots, cudaMemcpyDeviceToHost));
    for (int k = 0; k < S.n_slots; ++k) {
      const int a = order[k];
      if (a < 0) continue;
      const int local = a - S.atom_off;
      for (int ax = 0; ax < 3; ++ax) forces[3 * local + ax] = double((long long)f[ax][k]) / 4294967296.0;
    }
  }
  if (out) {
    std::vector<double> mol_all(size_t(e->mol_part_off.back() + molecular_offset_blocks(e->mol_count.back())) * 9);
    CUDA_TRY(e, cudaMemcpy(mol_all.data(), e->mol_partials, sizeof(double) * mol_all.size(), cudaMemcpyDeviceToHost));
    std::vector<unsigned long long> en(size_t(d.S) * kECount);
    CUDA_TRY(e, cudaMemcpy(en.data(), d.energy, sizeof(long long) * en.size(), cudaMemcpyDeviceToHost));
    std::vector<double> mesh(e->n_mesh_items), mesh_vir(size_t(e->n_mesh_items) * 6);
    CUDA_TRY(e, cudaMemcpy(mesh.data(), d.mesh_partial, sizeof(double) * e->n_mesh_items, cudaMemcpyDeviceToHost));
    CUDA_TRY(e, cudaMemcpy(mesh_vir.data(), d.mesh_virial, sizeof(double) * mesh_vir.size(), cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < systems.size(); ++i) {
      const int s = systems[i];
      const HostSystem& h = e->hs[s];
      const SysDev& S = e->sd[s];
      mdb_energies& o = out[i];
      std::memset(&o, 0, sizeof(o));
      const std::vector<double> mol_part(mol_all.begin() + size_t(e->mol_part_off[s]) * 9,
                                         mol_all.begin() + size_t(e->mol_part_off[s] +
                                                                  molecular_offset_blocks(e->mol_count[s])) * 9);
      auto val = [&](int k) { return double((long long)en[size_t(S.energy_base) + k]) / 4294967296.0; };
      double em = 0, wm[6] = {0, 0, 0, 0, 0, 0};
      for (int k = 0; k < e->n_mesh_items; ++k)
        if (e->fft_x_sys[k] == s) {
          em += mesh[k];
          for (int c = 0; c < 6; ++c) wm[c] += mesh_vir[size_t(k) * 6 + c];
        }
      o.bond = val(kEBond);
      o.angle = val(kEAngle);
      o.torsion = val(kETorsion);
      o.restraint = val(kERestraint);
      o.direct_coulomb = val(kECoulomb);
      o.direct_lj = val(kELj);
      o.exclusion_correction = val(kEExclusion);
      o.exceptions = val(kEException);
      o.pairs_within_cutoff = double(static_cast<long long>(en[size_t(S.energy_base) + kEPairs]));
      o.dispersion = h.dispersion_energy;
      o.reciprocal_mesh = em;
      o.self_energy = h.self_energy;
      o.net_charge = h.net_charge_energy;
      o.direct_group = o.direct_coulomb + o.direct_lj + o.exclusion_correction + o.exceptions + o.dispersion;
      o.reciprocal_group = o.reciprocal_mesh + o.self_energy + o.net_charge;
      // virial: pairs, exceptions and bonded terms from the device accumulators,
      // the mesh sum's from the FP64 partials, and the 1/V corrections on the
      // diagonal (restraints are left out: their anchors do not scale)
      for (int k = 0; k < 9; ++k) o.virial[k] = val(kEVirial0 + k);
      const int sym[6][2] = {{0, 0}, {4, 4}, {8, 8}, {1, 3}, {2, 6}, {5, 7}};
      for (int c = 0; c < 6; ++c) {
        o.virial[sym[c][0]] += wm[c];
        if (sym[c][1] != sym[c][0]) o.virial[sym[c][1]] += wm[c];
      }
      for (int a = 0; a < 3; ++a) o.virial[4 * a] += o.dispersion + o.net_charge;
      // the molecular virial: minus the atoms' offsets from their molecule's centre
      for (int c = 0; c < 9; ++c) {
        double corr = 0;
        for (size_t b = 0; b < mol_part.size() / 9; ++b) corr += mol_part[b * 9 + c];
        o.molecular_virial[c] = o.virial[c] - corr;
      }
      o.potential = o.bond + o.angle + o.torsion + o.restraint + o.direct_group + o.reciprocal_group;
      // kinetic energy from the velocities as they are (kinetic.ts:31)
      if (kinetic) {
        std::vector<float> v[3];
        for (auto& x : v) x.resize(h.n);
        CUDA_TRY(e, cudaMemcpy(v[0].data(), d.vx + S.atom_off, sizeof(float) * h.n, cudaMemcpyDeviceToHost));
        CUDA_TRY(e, cudaMemcpy(v[1].data(), d.vy + S.atom_off, sizeof(float) * h.n, cudaMemcpyDeviceToHost));
        CUDA_TRY(e, cudaMemcpy(v[2].data(), d.vz + S.atom_off, sizeof(float) * h.n, cudaMemcpyDeviceToHost));
        double ke = 0;
        for (int a = 0; a < h.n; ++a)
          if (h.mass[a] > 0)
            ke += h.mass[a] * (double(v[0][a]) * v[0][a] + double(v[1][a]) * v[1][a] + double(v[2][a]) * v[2][a]);
        o.kinetic = 0.5 * ke;
        o.degrees_of_freedom = h.dof;
        o.temperature = h.dof > 0 ? 2 * o.kinetic / (h.dof * kBoltzmann) : 0;
      }
    }
  }
  // the step loop expects cleared accumulators
  CUDA_TRY(e, cudaMemsetAsync(d.fx, 0, sizeof(long long) * d.n_slots, e->s0));
  CUDA_TRY(e, cudaMemsetAsync(d.fy, 0, sizeof(long long) * d.n_slots, e->s0));
  CUDA_TRY(e, cudaMemsetAsync(d.fz, 0, sizeof(long long) * d.n_slots, e->s0));
  CUDA_TRY(e, cudaStreamSynchronize(e->s0));
  return MDB_OK;
}

int evaluate(mdb_engine* e, int s, double* forces, mdb_energies* out, bool kinetic = true) {
  return evaluate_many(e, std::vector<int>{s}, forces, out, kinetic);
}

int get_positions(mdb_engine* e, int s, double* out) {
  const SysDev& S = e->sd[s];
  const int n = S.n_atoms;
  std::vector<long long> p[3];
  for (auto& v : p) v.resize(n);
  CUDA_TRY(e, cudaStreamSynchronize(e->s0));
  CUDA_TRY(e, cudaMemcpy(p[0].data(), e->d.px + S.atom_off, sizeof(long long) * n, cudaMemcpyDeviceToHost));
  CUDA_TRY(e, cudaMemcpy(p[1].data(), e->d.py + S.atom_off, sizeof(long long) * n, cudaMemcpyDeviceToHost));
  CUDA_TRY(e, cudaMemcpy(p[2].data(), e->d.pz + S.atom_off, sizeof(long long) * n, cudaMemcpyDeviceToHost));
  for (int a = 0; a < n; ++a)
    for (int k = 0; k < 3; ++k) out[3 * a + k] = double(p[k][a]) / 4294967296.0;
  return MDB_OK;
}

int set_positions(mdb_engine* e, int s, const double* in, bool clear_residual) {
  const SysDev& S = e->sd[s];
  const int n = S.n_atoms;
  std::vector<long long> p[3];
  for (auto& v : p) v.resize(n);
  for (int a = 0; a < n; ++a)
    for (int k = 0; k < 3; ++k) {
      if (!std::isfinite(in[3 * a + k]) || std::fabs(in[3 * a + k]) > 1.0e6)
        return fail(e, MDB_ERR_RANGE, "positions must be finite and inside the fixed-point range");
      p[k][a] = to_fixed_host(in[3 * a + k]);
    }
  CUDA_TRY(e, cudaStreamSynchronize(e->s0));
  CUDA_TRY(e, cudaMemcpy(e->d.px + S.atom_off, p[0].data(), sizeof(long long) * n, cudaMemcpyHostToDevice));
  CUDA_TRY(e, cudaMemcpy(e->d.py + S.atom_off, p[1].data(), sizeof(long long) * n, cudaMemcpyHostToDevice));
  CUDA_TRY(e, cudaMemcpy(e->d.pz + S.atom_off, p[2].data(), sizeof(long long) * n, cudaMemcpyHostToDevice));
  if (clear_residual) {
    CUDA_TRY(e, cudaMemset(e->d.rx + S.atom_off, 0, sizeof(float) * n));
    CUDA_TRY(e, cudaMemset(e->d.ry + S.atom_off, 0, sizeof(float) * n));
    CUDA_TRY(e, cudaMemset(e->d.rz + S.atom_off, 0, sizeof(float) * n));
  }
  return request_rebuild(e, s);
}

int set_box(mdb_engine* e, int s, const double* box) {
  HostSystem& h = e->hs[s];
  double reduced[9];
  if (!reduce_box(box, reduced)) return fail(e, MDB_ERR_INVALID_ARGUMENT, "degenerate box");
  double widths[3];
  perpendicular_widths(reduced, widths);
  if (h.cutoff > 0.5 * std::min({widths[0], widths[1], widths[2]}))
    return fail(e, MDB_ERR_CUTOFF_TOO_LARGE_FOR_BOX, "the cutoff does not fit the new box");
  std::copy(reduced, reduced + 9, h.box.begin());
  std::copy(reduced, reduced + 9, e->box_at_rebuild[s].begin());
  update_box_constants(h);
  fill_box(h, e->sd[s], true);
  CUDA_TRY(e, cudaStreamSynchronize(e->s0));
  CUDA_TRY(e, cudaMemcpy(const_cast<SysDev*>(e->d.sys) + s, &e->sd[s], sizeof(SysDev), cudaMemcpyHostToDevice));
  launch_influence(e->d, s, e->s0);
  CUDA_TRY(e, cudaGetLastError());
  return request_rebuild(e, s);
}

// Volume moves' box changes (or their undo) that keep the tile list: the
// tiles' shifts follow the new box from their lattice counts, the pair
// coordinates follow the scaled positions, and a device displacement test asks
// for a rebuild only if some atom has gone half the skin from the list's
// reference (k_after_box_change).  A rebuild is still asked for when the
// pair-coordinate scale changes or the box has drifted by more than 1% per
// axis since the engine last asked for one on a box change: the tiles'
// per-pair flags were set for the box the list was built in.
int move_boxes(mdb_engine* e, const std::vector<int>& sys, const std::vector<std::array<double, 9>>& boxes) {
  if (sys.empty()) return MDB_OK;
  std::vector<int> rebuild;
  for (size_t i = 0; i < sys.size(); ++i) {
    const int s = sys[i];
    HostSystem& h = e->hs[s];
    double reduced[9];
    if (!reduce_box(boxes[i].data(), reduced)) return fail(e, MDB_ERR_INVALID_ARGUMENT, "degenerate box");
    double widths[3];
    perpendicular_widths(reduced, widths);
    if (h.cutoff > 0.5 * std::min({widths[0], widths[1], widths[2]}))
      return fail(e, MDB_ERR_CUTOFF_TOO_LARGE_FOR_BOX, "the cutoff does not fit the new box");
    std::copy(reduced, reduced + 9, h.box.begin());
    update_box_constants(h);
    const int shift = e->sd[s].pc_shift;
    fill_box(h, e->sd[s], true);
    bool again = e->sd[s].pc_shift != shift;
    for (int k = 0; k < 3; ++k) again |= std::fabs(reduced[4 * k] / e->box_at_rebuild[s][4 * k] - 1.0) > 0.01;
    if (again) {
      std::copy(reduced, reduced + 9, e->box_at_rebuild[s].begin());
      rebuild.push_back(s);
    }
  }
  // every system's constants in one copy, after the work already queued
  CUDA_TRY(e, cudaStreamSynchronize(e->s0));
  CUDA_TRY(e, cudaMemcpy(const_cast<SysDev*>(e->d.sys), e->sd.data(), sizeof(SysDev) * e->d.S,
                         cudaMemcpyHostToDevice));
  launch_influence(e->d, sys.size() == 1 ? sys[0] : -1, e->s0);
  for (int s : sys)
    if (std::find(rebuild.begin(), rebuild.end(), s) == rebuild.end())
      launch_after_box_change(e->d, s, e->sd[s].n_slots, e->sd[s].tile_cap, e->s0);
  CUDA_TRY(e, cudaGetLastError());
  if (!rebuild.empty()) {
    std::vector<int> now(e->d.S, 0);
    CUDA_TRY(e, cudaStreamSynchronize(e->s0));
    CUDA_TRY(e, cudaMemcpy(now.data(), e->d.rebuild_now, sizeof(int) * e->d.S, cudaMemcpyDeviceToHost));
    for (int s : rebuild) now[s] = 1;
    const int one = 1;
    CUDA_TRY(e, cudaMemcpy(e->d.rebuild_now, now.data(), sizeof(int) * e->d.S, cudaMemcpyHostToDevice));
    CUDA_TRY(e, cudaMemcpy(e->d.any_rebuild, &one, sizeof(int), cudaMemcpyHostToDevice));
  }
  return MDB_OK;
}

// ---- the barostat's screening network (no reference counterpart) ----------
// Inputs: dlnV, the energy components and the molecular virial's diagonal per
// atom, the box diagonal, and the first-order change -tr(W_mol) dlnV / 3 per
// atom.  The network learns what the first-order term misses, which is second
// order in the move: its target is (dU - first order) / (atoms x dlnV^2), a
// smooth function of the state (the compressibility term) whose error stays on
// the kT scale however large the system, and which carries over to moves of
// another size -- the barostat rescales its moves as it runs, and a target
// learnt in plain (dU - first order) would have to be extrapolated in dlnV.
double first_order_change(const mdb_energies& en, double dlnv) {
  return -(en.molecular_virial[0] + en.molecular_virial[4] + en.molecular_virial[8]) * dlnv / 3.0;
}

void surrogate_features(const mdb_energies& en, const HostSystem& h, const double* box, double dlnv,
                        double* f) {
  const double n = std::max(1, h.n);
  const double raw[kMlpIn] = {dlnv,
                              en.bond / n,
                              en.angle / n,
                              en.torsion / n,
                              en.direct_coulomb / n,
                              en.direct_lj / n,
                              (en.exclusion_correction + en.exceptions) / n,
                              en.reciprocal_mesh / n,
                              en.dispersion / n,
                              en.molecular_virial[0] / n,
                              en.molecular_virial[4] / n,
                              en.molecular_virial[8] / n,
                              box[0],
                              box[4],
                              box[8],
                              // the first-order change under molecular scaling, -tr(W_mol) dlnV / 3
                              -(en.molecular_virial[0] + en.molecular_virial[4] + en.molecular_virial[8]) * dlnv /
                                  (3 * n)};
  for (int k = 0; k < kMlpIn; ++k) f[k] = raw[k];
}

int surrogate_alloc(mdb_engine* e, Surrogate& net, int samples) {
#define TRY(x)              \
  do {                      \
    const int st_ = (x);    \
    if (st_) return st_;    \
  } while (0)
  TRY(alloc(e, "surrogate weights", net.dev.w, kMlpParams));
  TRY(alloc(e, "surrogate adam m", net.dev.m, kMlpParams));
  TRY(alloc(e, "surrogate adam v", net.dev.v, kMlpParams));
  TRY(alloc(e, "surrogate weights bf16", net.dev.w_bf16, kMlpParams));
  TRY(alloc(e, "surrogate adam step", net.dev.step_count, 1));
  TRY(alloc(e, "surrogate inputs", net.x, size_t(std::max(samples, 2)) * kMlpIn));
  TRY(alloc(e, "surrogate targets", net.t, std::max(samples, 2)));
  TRY(alloc(e, "surrogate outputs", net.y, 2));
  TRY(alloc(e, "surrogate losses", net.loss, samples / kMlpBatch + 2));
  TRY(alloc(e, "surrogate inference inputs", net.xi, size_t(e->d.S) * 2 * kMlpIn));
  TRY(alloc(e, "surrogate inference outputs", net.yi, size_t(e->d.S) * 2));
#undef TRY
  return MDB_OK;
}

// Standardise the collected attempts, then train on the device from a seeded
// start (mlp_train).  Attempts whose move is under a tenth of the largest are
// left out: dividing by dlnV^2 would turn their energy noise into large targets.
int surrogate_train(mdb_engine* e, Surrogate& net, uint32_t seed, int epochs) {
  double largest = 0;
  for (double v : net.dlnv) largest = std::max(largest, std::fabs(v));
  std::vector<int> use;
  for (int i = 0; i < int(net.dlnv.size()); ++i)
    if (std::fabs(net.dlnv[i]) >= 0.1 * largest && net.dlnv[i] != 0) use.push_back(i);
  const int n = int(use.size());
  if (n < kMlpBatch) return MDB_OK;
  std::vector<double> feats(size_t(n) * kMlpIn), target(n);
  for (int i = 0; i < n; ++i) {
    const int j = use[i];
    for (int k = 0; k < kMlpIn; ++k) feats[size_t(i) * kMlpIn + k] = net.feats[size_t(j) * kMlpIn + k];
    target[i] = net.delta_u[j] / (net.dlnv[j] * net.dlnv[j]);
  }
  for (int k = 0; k < kMlpIn; ++k) {
    double m = 0, v = 0;
    for (int i = 0; i < n; ++i) m += feats[size_t(i) * kMlpIn + k];
    m /= n;
    for (int i = 0; i < n; ++i) v += (feats[size_t(i) * kMlpIn + k] - m) * (feats[size_t(i) * kMlpIn + k] - m);
    net.mu[k] = m;
    net.sd[k] = std::sqrt(v / n) > 1e-12 ? std::sqrt(v / n) : 1.0;
  }
  {
    double m = 0, v = 0;
    for (double t : target) m += t;
    m /= n;
    for (double t : target) v += (t - m) * (t - m);
    net.mu_t = m;
    net.sd_t = std::sqrt(v / n) > 1e-12 ? std::sqrt(v / n) : 1.0;
  }
  int st = surrogate_alloc(e, net, n);
  if (st) return st;
  std::vector<float> x(size_t(n) * kMlpIn), t(n);
  for (int i = 0; i < n; ++i) {
    for (int k = 0; k < kMlpIn; ++k)
      x[size_t(i) * kMlpIn + k] = float((feats[size_t(i) * kMlpIn + k] - net.mu[k]) / net.sd[k]);
    t[i] = float((target[i] - net.mu_t) / net.sd_t);
  }
  CUDA_TRY(e, cudaMemcpy(net.x, x.data(), sizeof(float) * x.size(), cudaMemcpyHostToDevice));
  CUDA_TRY(e, cudaMemcpy(net.t, t.data(), sizeof(float) * t.size(), cudaMemcpyHostToDevice));
  net.dev.lr = 2e-3f;
  net.dev.beta1 = 0.9f;
  net.dev.beta2 = 0.999f;
  net.dev.eps = 1e-8f;
  std::vector<double> losses;
  // its own events: a timed run (mdb_run_timed) may be holding the engine's
  cudaEvent_t fit0 = nullptr, fit1 = nullptr;
  CUDA_TRY(e, cudaEventCreate(&fit0));
  CUDA_TRY(e, cudaEventCreate(&fit1));
  cudaEventRecord(fit0, e->s0);
  const cudaError_t fit = mlp_train(net.dev, net.x, net.t, n, epochs, seed, net.loss, &losses, e->s0);
  cudaEventRecord(fit1, e->s0);
  float fit_ms = 0;
  if (fit == cudaSuccess && cudaEventSynchronize(fit1) == cudaSuccess) cudaEventElapsedTime(&fit_ms, fit0, fit1);
  cudaEventDestroy(fit0);
  cudaEventDestroy(fit1);
  CUDA_TRY(e, fit);
  net.fit_ms += fit_ms;
  net.final_loss = losses.empty() ? 0.0 : losses.back();
  net.active = true;
  return MDB_OK;
}

// Predicted potential changes (kJ/mol) of moves dlnv[i] from states with
// energies en[i] and boxes box[i] of systems sys[i], by one device forward
// pass over all of them.
int surrogate_predict(mdb_engine* e, Surrogate& net, const std::vector<int>& sys, const mdb_energies* en,
                      const std::vector<std::array<double, 9>>& box, const std::vector<double>& dlnv,
                      std::vector<double>& out) {
  const int n = int(sys.size());
  out.assign(n, 0.0);
  if (n == 0) return MDB_OK;
  std::vector<float> x(size_t(n) * kMlpIn);
  for (int i = 0; i < n; ++i) {
    double f[kMlpIn];
    surrogate_features(en[i], e->hs[sys[i]], box[i].data(), dlnv[i], f);
    for (int k = 0; k < kMlpIn; ++k) x[size_t(i) * kMlpIn + k] = float((f[k] - net.mu[k]) / net.sd[k]);
  }
  std::vector<float> y(n);
  CUDA_TRY(e, cudaMemcpyAsync(net.xi, x.data(), sizeof(float) * x.size(), cudaMemcpyHostToDevice, e->s0));
  launch_mlp_forward(net.dev.w_bf16, net.xi, n, net.yi, e->s0);
  CUDA_TRY(e, cudaMemcpyAsync(y.data(), net.yi, sizeof(float) * n, cudaMemcpyDeviceToHost, e->s0));
  CUDA_TRY(e, cudaStreamSynchronize(e->s0));
  for (int i = 0; i < n; ++i)
    out[i] = first_order_change(en[i], dlnv[i]) +
             (double(y[i]) * net.sd_t + net.mu_t) * std::max(1, e->hs[sys[i]].n) * dlnv[i] * dlnv[i];
  return MDB_OK;
}

// threefry2x32([draw, seed], [BAROSTAT_DOMAIN, 0]) (loop.ts:614-622): the
// barostat's next uniform number, one counter per system.
double barostat_uniform(BarostatState& b, uint32_t seed) {
  uint32_t c0 = uint32_t(b.draw++), c1 = seed, k0 = 0x6a09e667u, k1 = 0;
  static const int rot[8] = {13, 15, 26, 6, 17, 29, 16, 24};
  const uint32_t ks[3] = {k0, k1, 0x1bd11bdau ^ k0 ^ k1};
  uint32_t x0 = c0 + ks[0], x1 = c1 + ks[1];
  for (int r = 0; r < 20; ++r) {
    x0 += x1;
    x1 = ((x1 << rot[r % 8]) | (x1 >> (32 - rot[r % 8]))) ^ x0;
    if ((r + 1) % 4 == 0) {
      const uint32_t inj = uint32_t((r + 1) / 4);
      x0 += ks[inj % 3];
      x1 += ks[(inj + 1) % 3] + inj;
    }
  }
  return (double(x0 >> 9) + 0.5) * std::ldexp(1.0, -23);
}

// Boxes and positions of volume moves, on the device: back up, scale every
// molecule's centre, move the boxes (the list is kept unless an atom went too far).
int apply_volume_moves(mdb_engine* e, const std::vector<int>& sys, const std::vector<double>& scale) {
  std::vector<std::array<double, 9>> boxes(sys.size());
  for (size_t i = 0; i < sys.size(); ++i) {
    const int s = sys[i];
    launch_scale_molecules(e->d, e->mol_first[s], e->mol_count[s], scale[i], e->s0);
    for (int k = 0; k < 9; ++k) boxes[i][k] = e->hs[s].box[k] * scale[i];
  }
  CUDA_TRY(e, cudaGetLastError());
  return move_boxes(e, sys, boxes);
}

int undo_volume_moves(mdb_engine* e, const std::vector<int>& sys, const std::vector<std::array<double, 9>>& old_box) {
  for (int s : sys) launch_restore_positions(e->d, e->sd[s].atom_off, e->sd[s].n_atoms, e->s0);
  CUDA_TRY(e, cudaGetLastError());
  return move_boxes(e, sys, old_box);
}

// One Monte Carlo volume move for each system in `due` (src/gpu/loop.ts:602-641,
// src/reference/barostat.ts:210-274), all of them together: one evaluation of
// the engine gives every system's current energy, the moves are proposed and
// applied, and one more evaluation gives the proposals' energies.  Each
// system draws from its own counter, so a system's moves are the ones it
// would make alone.  With a trained screening network the moves go through
// delayed acceptance (Christen & Fox 2005): stage 1 accepts with
// a1 = min(1, exp(-w~/kT)) from the network's predicted change, and only the
// systems that pass go on to the exact energy; stage 2 accepts with
// min(1, exp(-w/kT) a1(y->x)/a1(x->y)), the reverse move's stage-1
// probability evaluated with the network at the proposal, so every chain
// keeps the exact NPT distribution.
int barostat_round(mdb_engine* e, const std::vector<int>& due) {
  Surrogate& net = e->net;
  const int n = int(due.size());
  std::vector<mdb_energies> e0(n);
  int st = evaluate_many(e, due, nullptr, e0.data(), false);
  if (st) return st;
  struct Move {
    std::array<double, 9> old_box;
    double volume, dv, scale, dlnv, volume_term, kT, a1 = 1.0;
    bool exact = true;
  };
  std::vector<Move> mv(n);
  for (int i = 0; i < n; ++i) {
    const int s = due[i];
    HostSystem& h = e->hs[s];
    BarostatState& b = e->baro[s];
    Move& m = mv[i];
    m.old_box = h.box;
    m.volume = box_volume(h.box.data());
    m.dv = b.volume_scale * 2 * (barostat_uniform(b, e->opt.seed) - 0.5);
    const double nv = m.volume + m.dv;
    m.scale = std::cbrt(nv / m.volume);
    m.dlnv = std::log(nv / m.volume);
    m.kT = kBoltzmann * h.barostat_temperature;
    m.volume_term = h.barostat_pressure * 0.06022140762081242 * m.dv - double(h.molecules.size()) * m.kT * m.dlnv;
  }
  const bool screen = net.active && !net.disabled;
  std::vector<double> du_pred;
  if (screen) {
    std::vector<std::array<double, 9>> boxes(n);
    std::vector<double> dl(n);
    for (int i = 0; i < n; ++i) {
      boxes[i] = mv[i].old_box;
      dl[i] = mv[i].dlnv;
    }
    if ((st = surrogate_predict(e, net, due, e0.data(), boxes, dl, du_pred))) return st;
  }
  std::vector<int> exact_sys;
  std::vector<int> exact_idx;
  for (int i = 0; i < n; ++i) {
    BarostatState& b = e->baro[due[i]];
    Move& m = mv[i];
    b.attempts++;
    b.window_attempts++;
    if (screen) {
      m.a1 = screen_probability(du_pred[i], m.volume_term, m.kT);
      m.exact = barostat_uniform(b, e->opt.seed) < m.a1;
      if (!m.exact) b.screened++;  // rejected by the network alone: no exact evaluation
    }
    if (m.exact) {
      exact_sys.push_back(due[i]);
      exact_idx.push_back(i);
    }
  }
  {
    std::vector<double> scales;
    for (int i : exact_idx) scales.push_back(mv[i].scale);
    if ((st = apply_volume_moves(e, exact_sys, scales))) return st;
  }
  std::vector<mdb_energies> e1(exact_sys.size());
  if (!exact_sys.empty() && (st = evaluate_many(e, exact_sys, nullptr, e1.data(), false))) return st;
  std::vector<double> du_rev;
  if (screen && !exact_sys.empty()) {
    std::vector<std::array<double, 9>> boxes(exact_sys.size());
    std::vector<double> dl(exact_sys.size());
    for (size_t k = 0; k < exact_sys.size(); ++k) {
      boxes[k] = e->hs[exact_sys[k]].box;
      dl[k] = -mv[exact_idx[k]].dlnv;
    }
    if ((st = surrogate_predict(e, net, exact_sys, e1.data(), boxes, dl, du_rev))) return st;
  }
  bool train = false;
  std::vector<int> undo_sys;
  std::vector<std::array<double, 9>> undo_box;
  for (size_t k = 0; k < exact_sys.size(); ++k) {
    const int s = exact_sys[k], i = exact_idx[k];
    HostSystem& h = e->hs[s];
    BarostatState& b = e->baro[s];
    Move& m = mv[i];
    b.exact++;
    const double du = e1[k].potential - e0[i].potential;
    const double w = du + m.volume_term;
    bool accepted = false;
    if (screen) {
      const double a2 = exact_stage_probability(w, du_rev[k], m.volume_term, m.kT, m.a1);
      accepted = barostat_uniform(b, e->opt.seed) < a2;
      // the exact stage checks the network's prediction
      const double err = du_pred[i] - du;
      net.err2 = net.checked == 0 ? err * err : 0.98 * net.err2 + 0.02 * err * err;
      if (++net.checked >= 50 && std::sqrt(net.err2) > kSurrogateMaxRmsKT * m.kT) net.disabled = true;
    } else {
      accepted = plain_accept(w, m.kT, [&] { return barostat_uniform(b, e->opt.seed); });
      if (net.target > 0 && !net.active) {
        double f[kMlpIn];
        surrogate_features(e0[i], h, m.old_box.data(), m.dlnv, f);
        for (double v : f) net.feats.push_back(float(v));
        // what the first-order term misses, per atom like the energy features
        net.delta_u.push_back((du - first_order_change(e0[i], m.dlnv)) / std::max(1, h.n));
        net.dlnv.push_back(m.dlnv);
        train |= int(net.delta_u.size()) >= net.target;
      }
    }
    if (accepted) {
      b.accepted++;
      b.window_accepted++;
    } else {
      undo_sys.push_back(s);
      undo_box.push_back(m.old_box);
    }
  }
  if ((st = undo_volume_moves(e, undo_sys, undo_box))) return st;
  if (train && (st = surrogate_train(e, net, e->opt.seed, 300))) return st;
  for (int i = 0; i < n; ++i) {
    BarostatState& b = e->baro[due[i]];
    if (b.window_attempts < 10) continue;
    if (b.window_accepted < 0.25 * b.window_attempts) {
      b.volume_scale /= 1.1;
      b.window_attempts = b.window_accepted = 0;
    } else if (b.window_accepted > 0.75 * b.window_attempts) {
      b.volume_scale = std::min(b.volume_scale * 1.1, mv[i].volume * 0.3);
      b.window_attempts = b.window_accepted = 0;
    }
  }
  return MDB_OK;
}

int run(mdb_engine* e, int64_t steps) {
  int freq = 0;
  for (const auto& h : e->hs)
    if (h.barostat_frequency > 0) freq = freq == 0 ? h.barostat_frequency : std::min(freq, h.barostat_frequency);
  int64_t remaining = steps;
  int stalled = 0;
  while (remaining > 0) {
    int64_t chunk = std::min<int64_t>(remaining, e->opt.max_batch);
    if (freq > 0) {
      int64_t until = chunk;
      for (size_t s = 0; s < e->hs.size(); ++s)
        if (e->hs[s].barostat_frequency > 0)
          until = std::min<int64_t>(until, std::max<int64_t>(1, e->hs[s].barostat_frequency - e->baro[s].step));
      chunk = until;
    }
    const int64_t before = e->step;
    int st = run_steps(e, chunk);
    if (st) return st;
    // a list that overflowed stopped the integrator at the step whose rebuild
    // overflowed: grow it, rebuild, and run the steps that did not happen
    bool halted = false;
    if ((st = list_halted(e, &halted))) return st;
    if (halted) {
      long long now = 0;
      CUDA_TRY(e, cudaMemcpy(&now, e->d.step, sizeof(long long), cudaMemcpyDeviceToHost));
      e->step = now;
      chunk = now - before;
      if (chunk == 0 && ++stalled > 4) return fail(e, MDB_ERR_CAPACITY, "the tile list kept overflowing");
      if ((st = grow_tile_list(e))) return st;
    } else {
      stalled = 0;
    }
    remaining -= chunk;
    if (freq > 0) {
      std::vector<int> due;
      for (size_t s = 0; s < e->hs.size(); ++s) {
        auto& h = e->hs[s];
        auto& b = e->baro[s];
        if (h.barostat_frequency <= 0) continue;
        b.step += chunk;  // barostat.ts:129 barostatActsAfterSteps
        if (b.step < h.barostat_frequency) continue;
        b.step -= h.barostat_frequency;
        due.push_back(int(s));
      }
      if (!due.empty() && (st = barostat_round(e, due))) return st;
    }
  }
  return check_device_status(e);
}

bool bad_system(const mdb_engine* e, int32_t s) { return !e || s < 0 || s >= int32_t(e->hs.size()); }

// Kernels one graph-replayed step launches: the list kernels (one cooperative
// launch, or 5 sort + 1 wrap + 6 tile-list kernels, 3 more when rebuilds
// prune), the inner-list kernel, PME (spread, 3 transform passes or 5 without
// the plane kernels, gather), listed, nonbonded, integrator.
int launches_per_step(const mdb_engine* e) {
  const Dev& d = e->d;
  return (e->coop_list ? 1 : 5 + 1 + 6 + (d.prune ? 3 : 0)) + (d.inner ? 1 : 0) +
         (d.n_fft_z ? (d.fft_planes ? 5 : 7) : 0) +
         (d.n_bonds + d.n_angles + d.n_torsions + d.n_exceptions + d.n_restraints > 0 ? 1 : 0) + 1 + 1;
}

}  // namespace

// ====================================================================== ABI
extern "C" {

int mdb_abi_version(void) { return MDB_ABI_VERSION; }

const char* mdb_status_string(int status) {
  switch (status) {
    case MDB_OK: return "ok";
    case MDB_ERR_INVALID_ARGUMENT: return "invalid argument";
    case MDB_ERR_UNSUPPORTED_FORCE: return "unsupported force";
    case MDB_ERR_CUTOFF_TOO_LARGE_FOR_BOX: return "cutoff too large for box";
    case MDB_ERR_CLUSTER_TOO_LARGE: return "constraint cluster too large";
    case MDB_ERR_NOT_CONVERGED: return "constraints did not converge";
    case MDB_ERR_CAPACITY: return "device table capacity exceeded";
    case MDB_ERR_RANGE: return "fixed-point range exceeded";
    case MDB_ERR_DEVICE: return "device error";
    case MDB_ERR_TIMEOUT: return "device wait timed out";
    case MDB_ERR_NO_DEVICE: return "no CUDA device";
    case MDB_ERR_NOT_SMOOTH: return "mesh size not 2/3/5/7-smooth";
    case MDB_ERR_DEVICE_LOST: return "device lost";
    default: return "unknown status";
  }
}

int mdb_device_count(int32_t* out) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) n = 0;
  if (out) *out = n;
  return n > 0 ? MDB_OK : MDB_ERR_NO_DEVICE;
}

int mdb_batch_create(int32_t n, const mdb_system_desc* systems, const mdb_state_desc* states,
                     const mdb_run_options* options, mdb_engine** out) {
  if (!out || n <= 0 || !systems || !states || !options) return MDB_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  auto* e = new mdb_engine();
  const int st = build_engine(e, n, systems, states, options);
  *out = e;  // returned even on failure so mdb_last_error can explain; caller destroys
  return st;
}

int mdb_create(const mdb_system_desc* system, const mdb_state_desc* state, const mdb_run_options* options,
               mdb_engine** out) {
  return mdb_batch_create(1, system, state, options, out);
}

int mdb_destroy(mdb_engine* e, int64_t* leaked_bytes) {
  if (!e) return MDB_ERR_INVALID_ARGUMENT;
  if (e->s0) cudaStreamSynchronize(e->s0);
  for (auto& g : e->graphs) cudaGraphExecDestroy(g.second);
  int64_t leaked = 0;
  for (auto& a : e->allocs)
    if (cudaFree(a.ptr) != cudaSuccess) leaked += int64_t(a.bytes);
  for (cudaEvent_t ev : {e->fork, e->listed, e->join1, e->join2, e->t0, e->t1})
    if (ev) cudaEventDestroy(ev);
  for (cudaStream_t s : {e->s0, e->s1, e->s2})
    if (s) cudaStreamDestroy(s);
  if (leaked_bytes) *leaked_bytes = leaked;
  delete e;
  return MDB_OK;
}

const char* mdb_last_error(const mdb_engine* e) { return e ? e->error.c_str() : "no engine"; }

int mdb_system_count(const mdb_engine* e, int32_t* out) {
  if (!e || !out) return MDB_ERR_INVALID_ARGUMENT;
  *out = int32_t(e->hs.size());
  return MDB_OK;
}

// The candidate grid: tile shape (8x8 or 32x32 clusters), tile pruning at
// rebuilds (a cheaper pair kernel against a longer rebuild), list skin
// (rebuild frequency against tile count), spatial-sort cell width (how compact
// a cluster is) and, for 8x8 tiles, an inner list re-pruned between rebuilds
// (which lets a long skin keep a short pair list).
int mdb_autotune(const mdb_system_desc* system, const mdb_state_desc* state, const mdb_run_options* options,
                 int32_t steps, mdb_tuning* best, double* best_ms_per_step, int32_t* tried) {
  return mdb_autotune_batch(1, system, state, options, steps, best, best_ms_per_step, tried);
}

int mdb_autotune_batch(int32_t n, const mdb_system_desc* systems, const mdb_state_desc* states,
                       const mdb_run_options* options, int32_t steps, mdb_tuning* best, double* best_ms_per_step,
                       int32_t* tried) {
  if (n <= 0 || !systems || !states || !options || !best || steps <= 0) return MDB_ERR_INVALID_ARGUMENT;
  struct Lists { double skin, inner; };
  static const Lists kLists8[] = {{0.15, -1.0}, {0.20, -1.0}, {0.30, 0.08}, {0.40, 0.08}, {0.50, 0.10}};
  static const Lists kLists32[] = {{0.15, -1.0}, {0.20, -1.0}};
  static const double kCells8[] = {0.20, 0.25};
  static const double kCells32[] = {0.20, 0.25, 0.35};
  static const int kPrune[] = {1, 2};
  // A batch keeps the device busy, so only the slots read and the list work
  // count: 8x8 tiles (32x32 ones never won a batch) over a finer ladder of
  // skins and inner skins, and no pruning at rebuild (the inner list prunes).
  static const Lists kListsBatch[] = {{0.15, -1.0}, {0.20, -1.0}, {0.25, -1.0}, {0.25, 0.06}, {0.30, 0.06},
                                      {0.30, 0.08}, {0.35, 0.08}, {0.40, 0.08}, {0.40, 0.10}, {0.50, 0.10}};
  std::vector<mdb_tuning> grid;
  if (n > 1) {
    for (const Lists& l : kListsBatch)
      for (double cell : kCells8) grid.push_back(mdb_tuning{l.skin, cell, 8, 2, l.inner});
  } else {
    for (int prune : kPrune) {
      for (const Lists& l : kLists8)
        for (double cell : kCells8) grid.push_back(mdb_tuning{l.skin, cell, 8, prune, l.inner});
      for (const Lists& l : kLists32)
        for (double cell : kCells32) grid.push_back(mdb_tuning{l.skin, cell, 32, prune, l.inner});
    }
  }
  double best_ms = std::numeric_limits<double>::infinity();
  int count = 0, last = MDB_OK;
  for (const mdb_tuning& t : grid) {
    mdb_run_options o = *options;
    const std::vector<mdb_tuning> every(size_t(n), t);
    o.tuning = every.data();
    mdb_engine* e = nullptr;
    int st = mdb_batch_create(n, systems, states, &o, &e);
    double ms = 0;
    if (st == MDB_OK) st = mdb_run(e, steps);  // warm-up: lists, graph capture
    if (st == MDB_OK) st = mdb_run_timed(e, steps, &ms);
    if (e) mdb_destroy(e, nullptr);
    ++count;
    if (st != MDB_OK) {  // a candidate may overflow a table; the others still count
      last = st;
      continue;
    }
    if (ms / steps < best_ms) {
      best_ms = ms / steps;
      *best = t;
    }
  }
  if (tried) *tried = count;
  if (best_ms_per_step) *best_ms_per_step = best_ms;
  return std::isfinite(best_ms) ? MDB_OK : last;
}

int mdb_run(mdb_engine* e, int64_t steps) {
  if (!e || steps < 0) return MDB_ERR_INVALID_ARGUMENT;
  return run(e, steps);
}

int mdb_run_timed(mdb_engine* e, int64_t steps, double* device_ms) {
  if (!e || steps < 0 || !device_ms) return MDB_ERR_INVALID_ARGUMENT;
  CUDA_TRY(e, cudaStreamSynchronize(e->s0));
  CUDA_TRY(e, cudaEventRecord(e->t0, e->s0));
  int st = run(e, steps);
  if (st) return st;
  CUDA_TRY(e, cudaEventRecord(e->t1, e->s0));
  CUDA_TRY(e, cudaEventSynchronize(e->t1));
  float ms = 0;
  CUDA_TRY(e, cudaEventElapsedTime(&ms, e->t0, e->t1));
  *device_ms = ms;
  return MDB_OK;
}

int mdb_set_step(mdb_engine* e, int64_t step) {
  if (!e || step < 0) return MDB_ERR_INVALID_ARGUMENT;
  CUDA_TRY(e, cudaStreamSynchronize(e->s0));
  std::vector<long long> v(e->d.S, step);
  CUDA_TRY(e, cudaMemcpy(e->d.step, v.data(), sizeof(long long) * e->d.S, cudaMemcpyHostToDevice));
  e->step = step;
  return MDB_OK;
}

int mdb_get_step(const mdb_engine* e, int64_t* step) {
  if (!e || !step) return MDB_ERR_INVALID_ARGUMENT;
  *step = e->step;
  return MDB_OK;
}

int mdb_get_positions(mdb_engine* e, int32_t s, double* out) {
  if (bad_system(e, s) || !out) return MDB_ERR_INVALID_ARGUMENT;
  return get_positions(e, s, out);
}

int mdb_get_velocities(mdb_engine* e, int32_t s, double* out) {
  if (bad_system(e, s) || !out) return MDB_ERR_INVALID_ARGUMENT;
  const SysDev& S = e->sd[s];
  const int n = S.n_atoms;
  std::vector<float> v[3];
  for (auto& x : v) x.resize(n);
  CUDA_TRY(e, cudaStreamSynchronize(e->s0));
  CUDA_TRY(e, cudaMemcpy(v[0].data(), e->d.vx + S.atom_off, sizeof(float) * n, cudaMemcpyDeviceToHost));
  CUDA_TRY(e, cudaMemcpy(v[1].data(), e->d.vy + S.atom_off, sizeof(float) * n, cudaMemcpyDeviceToHost));
  CUDA_TRY(e, cudaMemcpy(v[2].data(), e->d.vz + S.atom_off, sizeof(float) * n, cudaMemcpyDeviceToHost));
  for (int a = 0; a < n; ++a)
    for (int k = 0; k < 3; ++k) out[3 * a + k] = v[k][a];
  return MDB_OK;
}

int mdb_set_positions(mdb_engine* e, int32_t s, const double* positions) {
  if (bad_system(e, s) || !positions) return MDB_ERR_INVALID_ARGUMENT;
  return set_positions(e, s, positions, true);
}

int mdb_set_velocities(mdb_engine* e, int32_t s, const double* velocities) {
  if (bad_system(e, s) || !velocities) return MDB_ERR_INVALID_ARGUMENT;
  const SysDev& S = e->sd[s];
  const int n = S.n_atoms;
  std::vector<float> v[3];
  for (auto& x : v) x.resize(n);
  for (int a = 0; a < n; ++a)
    for (int k = 0; k < 3; ++k) v[k][a] = float(velocities[3 * a + k]);
  CUDA_TRY(e, cudaStreamSynchronize(e->s0));
  CUDA_TRY(e, cudaMemcpy(e->d.vx + S.atom_off, v[0].data(), sizeof(float) * n, cudaMemcpyHostToDevice));
  CUDA_TRY(e, cudaMemcpy(e->d.vy + S.atom_off, v[1].data(), sizeof(float) * n, cudaMemcpyHostToDevice));
  CUDA_TRY(e, cudaMemcpy(e->d.vz + S.atom_off, v[2].data(), sizeof(float) * n, cudaMemcpyHostToDevice));
  launch_momentum(e->d, e->s0);
  CUDA_TRY(e, cudaStreamSynchronize(e->s0));
  return MDB_OK;
}

int mdb_set_box(mdb_engine* e, int32_t s, const double box[9]) {
  if (bad_system(e, s) || !box) return MDB_ERR_INVALID_ARGUMENT;
  return set_box(e, s, box);
}

int mdb_get_box(const mdb_engine* e, int32_t s, double box[9]) {
  if (bad_system(e, s) || !box) return MDB_ERR_INVALID_ARGUMENT;
  std::copy(e->hs[s].box.begin(), e->hs[s].box.end(), box);
  return MDB_OK;
}

int mdb_get_mesh(const mdb_engine* e, int32_t s, int32_t mesh[3]) {
  if (bad_system(e, s) || !mesh) return MDB_ERR_INVALID_ARGUMENT;
  for (int k = 0; k < 3; ++k) mesh[k] = e->hs[s].grid[k];
  return MDB_OK;
}

int mdb_evaluate(mdb_engine* e, int32_t s, double* forces, mdb_energies* energies) {
  if (bad_system(e, s)) return MDB_ERR_INVALID_ARGUMENT;
  return evaluate(e, s, forces, energies);
}

int mdb_potential(mdb_engine* e, int32_t s, const double* positions, double* forces, mdb_energies* energies) {
  if (bad_system(e, s) || !positions) return MDB_ERR_INVALID_ARGUMENT;
  const int n = e->hs[s].n;
  std::vector<double> saved(3 * n);
  int st = get_positions(e, s, saved.data());
  if (st) return st;
  if ((st = set_positions(e, s, positions, false))) return st;
  st = evaluate(e, s, forces, energies);
  const int restore = set_positions(e, s, saved.data(), false);
  return st ? st : restore;
}

int mdb_get_barostat_stats(const mdb_engine* e, int32_t s, mdb_barostat_stats* out) {
  if (bad_system(e, s) || !out) return MDB_ERR_INVALID_ARGUMENT;
  std::memset(out, 0, sizeof(*out));
  out->attempts = e->baro[s].attempts;
  out->accepted = e->baro[s].accepted;
  out->volume_scale = e->baro[s].volume_scale;
  // the current state's energy every attempt, the proposal's when not screened
  out->exact_evaluations = e->baro[s].attempts + e->baro[s].exact;
  out->screened = e->baro[s].screened;
  const Surrogate& net = e->net;
  out->surrogate_active = net.active && !net.disabled ? 1 : 0;
  out->surrogate_disabled = net.disabled ? 1 : 0;
  out->training_samples = int64_t(net.delta_u.size());
  out->surrogate_rms = std::sqrt(net.err2);
  out->training_loss = net.final_loss;
  out->training_ms = net.fit_ms;
  return MDB_OK;
}

int mdb_get_cell_geometry(const mdb_engine* e, int32_t s, int32_t divisions[3], double extent[3]) {
  if (bad_system(e, s) || !divisions || !extent) return MDB_ERR_INVALID_ARGUMENT;
  for (int k = 0; k < 3; ++k) {
    divisions[k] = e->sd[s].cdim[k];
    extent[k] = e->hs[s].box[k * 4] / e->sd[s].cdim[k];
  }
  return MDB_OK;
}

int mdb_get_passes_per_step(const mdb_engine* e, int32_t* out) {
  if (!e || !out) return MDB_ERR_INVALID_ARGUMENT;
  *out = launches_per_step(e);
  return MDB_OK;
}

int mdb_get_neighbour_stats(mdb_engine* e, int32_t s, mdb_neighbour_stats* out) {
  if (bad_system(e, s) || !out) return MDB_ERR_INVALID_ARGUMENT;
  CUDA_TRY(e, cudaStreamSynchronize(e->s0));
  long long rebuilds = 0;
  int tiles = 0, err = 0;
  CUDA_TRY(e, cudaMemcpy(&rebuilds, e->d.rebuild_count + s, sizeof(long long), cudaMemcpyDeviceToHost));
  CUDA_TRY(e, cudaMemcpy(&tiles, e->d.tile_count + s, sizeof(int), cudaMemcpyDeviceToHost));
  CUDA_TRY(e, cudaMemcpy(&err, e->d.err + s, sizeof(int), cudaMemcpyDeviceToHost));
  out->rebuilds = rebuilds;
  out->tiles = tiles;
  out->tile_capacity = e->sd[s].tile_cap;
  out->blocks = e->sd[s].n_blocks;
  out->overflowed = (err & kErrTileCapacity) || e->list_grown > 0 ? 1 : 0;
  out->list_grown = e->list_grown;
  out->skin = e->skin[s];
  out->inner_tiles = tiles;
  out->prunes = 0;
  out->inner_skin = 0;
  out->tile_atoms = e->cluster;
  if (e->d.inner) {
    int inner = 0;
    long long prunes = 0;
    CUDA_TRY(e, cudaMemcpy(&inner, e->d.in_count + s, sizeof(int), cudaMemcpyDeviceToHost));
    CUDA_TRY(e, cudaMemcpy(&prunes, e->d.prune_count + s, sizeof(long long), cudaMemcpyDeviceToHost));
    out->inner_tiles = inner;
    out->prunes = prunes;
    out->inner_skin = e->inner_skin[s] > 0 ? std::min(e->inner_skin[s], e->skin[s]) : 0.0;
  }
  return MDB_OK;
}

int mdb_profile_step(mdb_engine* e, int32_t repeats, mdb_profile* out) {
  if (!e || !out || repeats <= 0) return MDB_ERR_INVALID_ARGUMENT;
  std::memset(out, 0, sizeof(*out));
  const Dev& d = e->d;
  cudaStream_t st = e->s0;
  auto time = [&](auto&& body) -> double {
    cudaEventRecord(e->t0, st);
    for (int r = 0; r < repeats; ++r) body();
    cudaEventRecord(e->t1, st);
    cudaEventSynchronize(e->t1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e->t0, e->t1);
    return double(ms) / repeats;
  };
  // pairs and tiles at this configuration
  // every system (the pair counts below are the whole launch's)
  std::vector<int> all(d.S);
  std::iota(all.begin(), all.end(), 0);
  std::vector<mdb_energies> en(d.S);
  int status = evaluate_many(e, all, nullptr, en.data(), false);
  if (status) return status;
  // pairs of every system of the engine: the pair kernel's launch covers them all
  {
    std::vector<unsigned long long> all(size_t(d.S) * kECount);
    CUDA_TRY(e, cudaMemcpy(all.data(), d.energy, sizeof(unsigned long long) * all.size(), cudaMemcpyDeviceToHost));
    int64_t pairs = 0;
    for (int s = 0; s < d.S; ++s) pairs += static_cast<long long>(all[size_t(s) * kECount + kEPairs]);
    out->pairs_within_cutoff = pairs;
  }
  int tiles = 0;
  CUDA_TRY(e, cudaMemcpy(&tiles, d.tile_prefix + d.S, sizeof(int), cudaMemcpyDeviceToHost));
  out->tiles = tiles;
  out->tile_atoms = d.cluster;
  out->inner_tiles = tiles;
  if (d.inner) {
    int inner = 0;
    CUDA_TRY(e, cudaMemcpy(&inner, d.in_prefix + d.S, sizeof(int), cudaMemcpyDeviceToHost));
    out->inner_tiles = inner;
  }
  out->atoms = d.n_atoms;
  for (const auto& h : e->hs) out->mesh_points += int64_t(h.grid[0]) * h.grid[1] * h.grid[2];
  out->repeats = repeats;
  // whole step from a graph (warmed once)
  status = run_steps(e, 1);
  if (status) return status;
  out->ms_step = time([&] { run_steps(e, 1); });
  // the list kernels with no rebuild due, then with one forced
  list_kernels(e, st);
  CUDA_TRY(e, cudaMemsetAsync(d.any_rebuild, 0, sizeof(int), st));
  out->ms_list_check = time([&] { list_kernels(e, st); });
  std::vector<int> ones(d.S, 1);
  const int one = 1;
  out->ms_list_rebuild = time([&] {
    cudaMemcpyAsync(d.rebuild_now, ones.data(), sizeof(int) * d.S, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d.any_rebuild, &one, sizeof(int), cudaMemcpyHostToDevice, st);
    list_kernels(e, st);
  });
  CUDA_TRY(e, cudaGetLastError());
  if (d.inner)
    out->ms_inner_prune = time([&] {
      cudaMemcpyAsync(d.prune_now, ones.data(), sizeof(int) * d.S, cudaMemcpyHostToDevice, st);
      cudaMemcpyAsync(d.any_prune, &one, sizeof(int), cudaMemcpyHostToDevice, st);
      list_kernels(e, st);
    });
  out->ms_nonbonded = time([&] { launch_nonbonded(d, false, st); });
  out->ms_listed = time([&] { launch_listed(d, false, st); });
  out->ms_pme_spread = time([&] { launch_pme_spread(d, st); });
  out->ms_pme_fft = time([&] { launch_pme_fft(d, false, st); });
  out->ms_pme_gather = time([&] { launch_pme_gather(d, st); });
  out->ms_pme = time([&] { launch_pme(d, false, st); });
  // the timings above piled up forces; the integrator is timed on cleared ones,
  // so its constraint solves see an ordinary step
  CUDA_TRY(e, cudaMemsetAsync(d.fx, 0, sizeof(long long) * d.n_slots, st));
  CUDA_TRY(e, cudaMemsetAsync(d.fy, 0, sizeof(long long) * d.n_slots, st));
  CUDA_TRY(e, cudaMemsetAsync(d.fz, 0, sizeof(long long) * d.n_slots, st));
  out->ms_integrate = time([&] { launch_integrate(d, st); });
  // per step: the list kernels (one cooperative launch, or 5 sort + 1 wrap +
  // 6 tile-list kernels, 3 more when rebuilds prune), the inner-list kernel,
  // PME (spread, 3 transform passes or 5 without the plane kernels, gather),
  // listed, nonbonded, integrator
  out->launches_per_step = launches_per_step(e);
  CUDA_TRY(e, cudaMemsetAsync(d.fx, 0, sizeof(long long) * d.n_slots, st));
  CUDA_TRY(e, cudaMemsetAsync(d.fy, 0, sizeof(long long) * d.n_slots, st));
  CUDA_TRY(e, cudaMemsetAsync(d.fz, 0, sizeof(long long) * d.n_slots, st));
  CUDA_TRY(e, cudaGetLastError());
  return check_device_status(e);
}

int mdb_memory_report(const mdb_engine* e, char* buffer, int64_t capacity, int64_t* total_bytes) {
  if (!e) return MDB_ERR_INVALID_ARGUMENT;
  std::ostringstream os;
  int64_t total = 0;
  for (const auto& a : e->allocs) {
    os << a.label << "=" << a.bytes << ";";
    total += int64_t(a.bytes);
  }
  if (total_bytes) *total_bytes = total;
  if (buffer && capacity > 0) {
    const std::string s = os.str();
    const size_t n = std::min<size_t>(s.size(), size_t(capacity - 1));
    std::memcpy(buffer, s.data(), n);
    buffer[n] = '\0';
  }
  return MDB_OK;
}

}  // extern "C"
