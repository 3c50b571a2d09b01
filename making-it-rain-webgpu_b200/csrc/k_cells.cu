// k_cells.cu -- folding positions into the cell, the deterministic spatial
// sort, and the cluster-pair tile list with its interaction masks.
//
// Replaces the reference's wrap + counting-sort cell list + sort_cells
// (src/gpu/kernels/cell-list.wgsl:140-331) and its three-pass Verlet list
// (nonbonded-pairs.wgsl:412-497) with a B200-shaped design:
//   * atoms are sorted along a Morton curve of ~0.3 nm fractional cells, so 32
//     consecutive slots form a compact cluster (a "block");
//   * the list holds block pairs (tiles) whose bounding boxes come within
//     cutoff + skin, plus one 32-bit interaction mask per tile row that removes
//     exclusions, padding and the lower triangle of diagonal tiles;
//   * the order inside a cell is ascending atom index, written by rank rather
//     than by atomics, so two runs build bit-identical lists.
// A rebuild happens only when the integrator saw an atom move more than skin/2
// (verlet.wgsl:57), decided on the device; every phase kernel returns at once
// when no system asked for one.
#include <algorithm>

#include "device_state.h"

namespace mdb {
namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ int grid_stride_start() { return blockIdx.x * blockDim.x + threadIdx.x; }
__device__ __forceinline__ int grid_stride() { return gridDim.x * blockDim.x; }

// Fractional coordinates of a 2^32 fixed-point position, exactly, and the
// position folded into the cell (fixed64.wgsl:335 does the same with f32
// estimates and a bounded loop; here the lattice count is exact).
struct Folded {
  long long x, y, z;           // folded position, 2^32 fixed
  unsigned int fa, fb, fc;     // fractional parts, 2^-32 units
};

__device__ __forceinline__ Folded fold(const SysDev& S, long long x, long long y, long long z) {
  const long long fa = fixed_mul(x, S.inv_fx[0]) + fixed_mul(y, S.inv_fx[3]) + fixed_mul(z, S.inv_fx[6]);
  const long long fb = fixed_mul(y, S.inv_fx[4]) + fixed_mul(z, S.inv_fx[7]);
  const long long fc = fixed_mul(z, S.inv_fx[8]);
  const long long na = fa >> 32, nb = fb >> 32, nc = fc >> 32;
  Folded f;
  f.x = x - na * S.box_fx[0] - nb * S.box_fx[3] - nc * S.box_fx[6];
  f.y = y - nb * S.box_fx[4] - nc * S.box_fx[7];
  f.z = z - nc * S.box_fx[8];
  f.fa = static_cast<unsigned int>(fa & 0xffffffffll);
  f.fb = static_cast<unsigned int>(fb & 0xffffffffll);
  f.fc = static_cast<unsigned int>(fc & 0xffffffffll);
  return f;
}

__device__ __forceinline__ int to_pair_coordinate(long long v, int shift) {
  const int down = 32 - shift;
  return static_cast<int>((v + (1ll << (down - 1))) >> down);
}

__device__ __forceinline__ int cell_index(unsigned int frac, int dim) {
  const int c = static_cast<int>((static_cast<unsigned long long>(frac) * static_cast<unsigned>(dim)) >> 32);
  return c < dim ? c : dim - 1;
}

// ---------------------------------------------------------------- phases --

__device__ void phase_cells_clear(const Dev& d) {
  for (int c = grid_stride_start(); c < d.n_cells; c += grid_stride()) {
    if (!d.rebuild_now[d.cell_sys[c]]) continue;
    d.cell_cnt[c] = 0;
    d.cell_cur[c] = 0;
  }
}

__device__ void phase_cells_assign(const Dev& d) {
  for (int a = grid_stride_start(); a < d.n_atoms; a += grid_stride()) {
    const int s = d.atom_sys[a];
    if (!d.rebuild_now[s]) continue;
    const SysDev& S = d.sys[s];
    const Folded f = fold(S, d.px[a], d.py[a], d.pz[a]);
    const int cx = cell_index(f.fa, S.cdim[0]), cy = cell_index(f.fb, S.cdim[1]),
              cz = cell_index(f.fc, S.cdim[2]);
    const int local = d.cell_map[S.cell_off + (cx * S.cdim[1] + cy) * S.cdim[2] + cz];
    const int gc = S.cell_off + local;
    d.cell_of[a] = gc;
    atomicAdd(&d.cell_cnt[gc], 1);
  }
}

// Exclusive scan of `in[0..n)` into `out`, one block, in order.  Returns total.
__device__ int block_exclusive_scan(const int* in, int* out, int n) {
  __shared__ int warp_sums[kThreads / 32];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int base = 0; base < n; base += blockDim.x) {
    const int i = base + threadIdx.x;
    const int v = i < n ? in[i] : 0;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
      int w = lane < (kThreads / 32) ? warp_sums[lane] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += y;
      }
      if (lane < (kThreads / 32)) warp_sums[lane] = w;
    }
    __syncthreads();
    const int before = (warp > 0 ? warp_sums[warp - 1] : 0) + carry;
    if (i < n) out[i] = before + x - v;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = before + x;
    __syncthreads();
  }
  return carry;
}

__device__ void phase_cells_scan(const Dev& d) {
  for (int s = blockIdx.x; s < d.S; s += gridDim.x) {
    if (!d.rebuild_now[s]) continue;
    const SysDev& S = d.sys[s];
    block_exclusive_scan(d.cell_cnt + S.cell_off, d.cell_start + S.cell_off, S.n_cells);
  }
}

__device__ void phase_cells_scatter(const Dev& d) {
  for (int a = grid_stride_start(); a < d.n_atoms; a += grid_stride()) {
    const int s = d.atom_sys[a];
    if (!d.rebuild_now[s]) continue;
    const int gc = d.cell_of[a];
    const int slot = d.cell_start[gc] + atomicAdd(&d.cell_cur[gc], 1);
    d.tmp_order[d.sys[s].slot_off + slot] = a;
  }
}

// Ascending atom index inside each cell, by rank: the order is a function of
// the positions alone, whatever order the scatter's atomics landed in
// (cell-list.wgsl:319 sort_cells).
__device__ void phase_cells_order(const Dev& d) {
  for (int gs = grid_stride_start(); gs < d.n_slots; gs += grid_stride()) {
    const int s = d.slot_sys[gs];
    if (!d.rebuild_now[s]) continue;
    const SysDev& S = d.sys[s];
    const int local = gs - S.slot_off;
    if (local >= S.n_atoms) {
      d.order[gs] = -1;
      continue;
    }
    const int a = d.tmp_order[gs];
    const int gc = d.cell_of[a];
    const int st = d.cell_start[gc], cnt = d.cell_cnt[gc];
    int r = 0;
    for (int k = 0; k < cnt; ++k) r += d.tmp_order[S.slot_off + st + k] < a;
    d.order[S.slot_off + st + r] = a;
    d.rank[a] = st + r;
  }
}

// Every step, every system: pair coordinates of each slot, folded into the
// cell, as int32 at 2^pc_shift per nm (cell-list.wgsl:140 `wrap`).
__device__ void phase_wrap(const Dev& d) {
  for (int gs = grid_stride_start(); gs < d.n_slots; gs += grid_stride()) {
    const int a = d.order[gs];
    if (a < 0) {
      d.pc[gs] = make_int4(0, 0, 0, 0);
      continue;
    }
    const SysDev& S = d.sys[d.slot_sys[gs]];
    const Folded f = fold(S, d.px[a], d.py[a], d.pz[a]);
    d.pc[gs] = make_int4(to_pair_coordinate(f.x, S.pc_shift), to_pair_coordinate(f.y, S.pc_shift),
                         to_pair_coordinate(f.z, S.pc_shift), 0);
  }
}

// Warp per block: parameters in slot order, bounding box, and the reference
// positions the displacement test measures against.
__device__ void phase_tiles_blocks(const Dev& d) {
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; b < d.n_blocks; b += warps) {
    const int s = d.block_sys[b];
    if (!d.rebuild_now[s]) continue;
    const SysDev& S = d.sys[s];
    const int gs = b * 32 + lane;
    const int a = d.order[gs];
    float lo[3] = {3.0e38f, 3.0e38f, 3.0e38f}, hi[3] = {-3.0e38f, -3.0e38f, -3.0e38f};
    if (a >= 0) {
      d.prm[gs] = d.prm_atom[a];
      d.refx[a] = d.px[a];
      d.refy[a] = d.py[a];
      d.refz[a] = d.pz[a];
      const int4 p = d.pc[gs];
      lo[0] = hi[0] = p.x * S.pc_inv;
      lo[1] = hi[1] = p.y * S.pc_inv;
      lo[2] = hi[2] = p.z * S.pc_inv;
    } else {
      d.prm[gs] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        lo[k] = fminf(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], o));
        hi[k] = fmaxf(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], o));
      }
    if (lane == 0) {
      d.bb_lo[b] = make_float4(lo[0], lo[1], lo[2], 0.f);
      d.bb_hi[b] = make_float4(hi[0], hi[1], hi[2], 0.f);
    }
  }
}

// Do blocks I and J of one system come within cutoff + skin under some
// periodic image?  Box-to-box gap distance, minimised over images.
__device__ __forceinline__ bool blocks_near(const SysDev& S, const Dev& d, int I, int J) {
  const float4 li = d.bb_lo[I], hi_ = d.bb_hi[I], lj = d.bb_lo[J], hj = d.bb_hi[J];
  const float hx = 0.5f * (hi_.x - li.x) + 0.5f * (hj.x - lj.x);
  const float hy = 0.5f * (hi_.y - li.y) + 0.5f * (hj.y - lj.y);
  const float hz = 0.5f * (hi_.z - li.z) + 0.5f * (hj.z - lj.z);
  float dx = 0.5f * (lj.x + hj.x) - 0.5f * (li.x + hi_.x);
  float dy = 0.5f * (lj.y + hj.y) - 0.5f * (li.y + hi_.y);
  float dz = 0.5f * (lj.z + hj.z) - 0.5f * (li.z + hi_.z);
  const float* B = S.box_f;
  // sequential reduction c, b, a (src/reference/forces/nonbonded.ts:241)
  const float kc = rintf(dz / B[8]);
  dx -= kc * B[6]; dy -= kc * B[7]; dz -= kc * B[8];
  const float kb = rintf(dy / B[4]);
  dx -= kb * B[3]; dy -= kb * B[4];
  dx -= rintf(dx / B[0]) * B[0];
  if (!S.triclinic) {
    const float gx = fmaxf(fabsf(dx) - hx, 0.f), gy = fmaxf(fabsf(dy) - hy, 0.f), gz = fmaxf(fabsf(dz) - hz, 0.f);
    return gx * gx + gy * gy + gz * gz < S.list2;
  }
  float best = 3.0e38f;
  for (int k = -1; k <= 1; ++k)
    for (int j = -1; j <= 1; ++j)
      for (int i = -1; i <= 1; ++i) {
        const float x = dx + i * B[0] + j * B[3] + k * B[6];
        const float y = dy + j * B[4] + k * B[7];
        const float z = dz + k * B[8];
        const float gx = fmaxf(fabsf(x) - hx, 0.f), gy = fmaxf(fabsf(y) - hy, 0.f), gz = fmaxf(fabsf(z) - hz, 0.f);
        best = fminf(best, gx * gx + gy * gy + gz * gz);
      }
  return best < S.list2;
}

__device__ void phase_tiles_count(const Dev& d) {
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int I = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; I < d.n_blocks; I += warps) {
    const int s = d.block_sys[I];
    if (!d.rebuild_now[s]) continue;
    const SysDev& S = d.sys[s];
    const int end = S.block_off + S.n_blocks;
    int count = 0;
    for (int J0 = I; J0 < end; J0 += 32) {
      const int J = J0 + lane;
      const bool near = J < end && blocks_near(S, d, I, J);
      count += __popc(__ballot_sync(0xffffffffu, near));
    }
    if (lane == 0) d.tile_cnt[I] = count;
  }
}

__device__ void phase_tiles_scan(const Dev& d) {
  for (int s = blockIdx.x; s < d.S; s += gridDim.x) {
    if (!d.rebuild_now[s]) continue;
    const SysDev& S = d.sys[s];
    const int total = block_exclusive_scan(d.tile_cnt + S.block_off, d.tile_start + S.block_off, S.n_blocks);
    if (threadIdx.x == 0) {
      if (total > S.tile_cap) atomicOr(&d.err[s], kErrTileCapacity);
      d.tile_count[s] = total < S.tile_cap ? total : S.tile_cap;
    }
  }
}

__device__ void phase_tiles_fill(const Dev& d) {
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int I = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; I < d.n_blocks; I += warps) {
    const int s = d.block_sys[I];
    if (!d.rebuild_now[s]) continue;
    const SysDev& S = d.sys[s];
    const int end = S.block_off + S.n_blocks;
    const int Il = I - S.block_off;
    const bool row_valid = Il * 32 + lane < S.n_atoms;
    int at = d.tile_start[I];
    for (int J0 = I; J0 < end; J0 += 32) {
      const int J = J0 + lane;
      const bool near = J < end && blocks_near(S, d, I, J);
      unsigned int bits = __ballot_sync(0xffffffffu, near);
      while (bits) {
        const int k = __ffs(bits) - 1;
        bits &= bits - 1;
        const int Jk = J0 + k;
        if (at < S.tile_cap) {
          const int t = S.tile_off + at;
          if (lane == 0) d.tiles[t] = make_int2(I, Jk);
          const int Jl = Jk - S.block_off;
          const int nj = min(32, S.n_atoms - Jl * 32);
          unsigned int valid = nj >= 32 ? 0xffffffffu : ((1u << nj) - 1u);
          if (Jk == I) valid &= lane == 31 ? 0u : (0xffffffffu << (lane + 1));
          d.masks[static_cast<long long>(t) * 32 + lane] = row_valid ? valid : 0u;
        }
        ++at;
      }
    }
  }
}

// Clear the mask bit of every excluded pair in the tile that holds it.
__device__ void phase_tiles_exclusions(const Dev& d) {
  for (int e = grid_stride_start(); e < d.n_excl; e += grid_stride()) {
    const int s = d.excl_sys[e];
    if (!d.rebuild_now[s]) continue;
    const SysDev& S = d.sys[s];
    const int2 pr = d.excl[e];
    int sa = d.rank[pr.x], sb = d.rank[pr.y];
    if (sa > sb) { const int t = sa; sa = sb; sb = t; }
    const int I = S.block_off + (sa >> 5), J = S.block_off + (sb >> 5);
    const int lane = sa & 31, bit = sb & 31;
    int lo = d.tile_start[I];
    int hi = lo + d.tile_cnt[I];
    if (hi > S.tile_cap) hi = S.tile_cap;
    // tiles of row I are in ascending J
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      const int Jm = d.tiles[S.tile_off + mid].y;
      if (Jm < J) lo = mid + 1;
      else hi = mid;
    }
    if (lo < d.tile_start[I] + d.tile_cnt[I] && lo < S.tile_cap && d.tiles[S.tile_off + lo].y == J)
      atomicAnd(&d.masks[static_cast<long long>(S.tile_off + lo) * 32 + lane], ~(1u << bit));
  }
}

__device__ void phase_tiles_finish(const Dev& d) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    int total = 0;
    for (int s = 0; s < d.S; ++s) {
      d.tile_prefix[s] = total;
      total += d.tile_count[s];
      if (d.rebuild_now[s]) d.rebuild_count[s] += 1;
      d.rebuild_now[s] = 0;
    }
    d.tile_prefix[d.S] = total;
    *d.any_rebuild = 0;
  }
}

// Grid-wide barrier for the cooperative list kernel: arrive on a counter,
// the last arrival bumps the generation, the others wait on it with a bounded
// spin.  A wait that gives up records kErrTimeout and returns, so a scheduling
// fault becomes an error status and never a hung GPU.
__device__ bool grid_barrier(unsigned int* bar, int* err) {
  __syncthreads();
  __shared__ int ok;
  if (threadIdx.x == 0) {
    ok = 1;
    volatile unsigned int* gen = bar + 1;
    const unsigned int mine = *gen;
    __threadfence();
    if (atomicAdd(bar, 1u) + 1u == gridDim.x) {
      bar[0] = 0u;
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      long long spins = 0;
      while (*gen == mine) {
        if (++spins > (1ll << 22)) {
          atomicOr(err, kErrTimeout);
          ok = 0;
          break;
        }
        __nanosleep(32);
      }
    }
    __threadfence();
  }
  __syncthreads();
  return ok != 0;
}

// One launch per step.  With no rebuild requested it only folds the pair
// coordinates; otherwise it runs the sort and tile-list phases with a grid
// barrier between them.
__global__ void __launch_bounds__(kThreads) k_list(Dev d) {
  const bool rebuild = *d.any_rebuild != 0;
  if (!rebuild) {
    phase_wrap(d);
    return;
  }
  int* err = d.err;  // system 0's word carries a barrier timeout
  phase_cells_clear(d);
  if (!grid_barrier(d.list_barrier, err)) return;
  phase_cells_assign(d);
  if (!grid_barrier(d.list_barrier, err)) return;
  phase_cells_scan(d);
  if (!grid_barrier(d.list_barrier, err)) return;
  phase_cells_scatter(d);
  if (!grid_barrier(d.list_barrier, err)) return;
  phase_cells_order(d);
  if (!grid_barrier(d.list_barrier, err)) return;
  phase_wrap(d);
  if (!grid_barrier(d.list_barrier, err)) return;
  phase_tiles_blocks(d);
  if (!grid_barrier(d.list_barrier, err)) return;
  phase_tiles_count(d);
  if (!grid_barrier(d.list_barrier, err)) return;
  phase_tiles_scan(d);
  if (!grid_barrier(d.list_barrier, err)) return;
  phase_tiles_fill(d);
  if (!grid_barrier(d.list_barrier, err)) return;
  phase_tiles_exclusions(d);
  if (!grid_barrier(d.list_barrier, err)) return;
  phase_tiles_finish(d);
}

// The same phases as separate launches (the path the graph-free debug mode
// and devices without cooperative launch take).
#define MDB_PHASE_KERNEL(name, guarded)                            \
  __global__ void __launch_bounds__(kThreads) k_##name(Dev d) {   \
    if (guarded && !*d.any_rebuild) return;                        \
    phase_##name(d);                                               \
  }
MDB_PHASE_KERNEL(cells_clear, true)
MDB_PHASE_KERNEL(cells_assign, true)
MDB_PHASE_KERNEL(cells_scan, true)
MDB_PHASE_KERNEL(cells_scatter, true)
MDB_PHASE_KERNEL(cells_order, true)
MDB_PHASE_KERNEL(wrap, false)
MDB_PHASE_KERNEL(tiles_blocks, true)
MDB_PHASE_KERNEL(tiles_count, true)
MDB_PHASE_KERNEL(tiles_scan, true)
MDB_PHASE_KERNEL(tiles_fill, true)
MDB_PHASE_KERNEL(tiles_exclusions, true)
MDB_PHASE_KERNEL(tiles_finish, true)
#undef MDB_PHASE_KERNEL

int blocks_for(int n, int threads, int cap = 148 * 8) {
  const int b = (n + threads - 1) / threads;
  return b < 1 ? 1 : (b > cap ? cap : b);
}

int g_list_grid = 0;

}  // namespace

// Size the cooperative grid once: every block resident at the same time.
int prepare_list_kernel(int device) {
  int per_sm = 0, sms = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_list, kThreads, 0) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return 0;
  int coop = 0;
  cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device);
  g_list_grid = coop ? std::max(1, std::min(per_sm, 2)) * sms : 0;
  return g_list_grid;
}

bool launch_list(const Dev& d, cudaStream_t st) {
  if (g_list_grid <= 0) return false;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(g_list_grid);
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_list, d) == cudaSuccess;
}

void launch_rebuild_sort(const Dev& d, cudaStream_t st) {
  k_cells_clear<<<blocks_for(d.n_cells, kThreads), kThreads, 0, st>>>(d);
  k_cells_assign<<<blocks_for(d.n_atoms, kThreads), kThreads, 0, st>>>(d);
  k_cells_scan<<<d.S < 148 ? d.S : 148, kThreads, 0, st>>>(d);
  k_cells_scatter<<<blocks_for(d.n_atoms, kThreads), kThreads, 0, st>>>(d);
  k_cells_order<<<blocks_for(d.n_slots, kThreads), kThreads, 0, st>>>(d);
}

void launch_wrap(const Dev& d, cudaStream_t st) {
  k_wrap<<<blocks_for(d.n_slots, kThreads), kThreads, 0, st>>>(d);
}

void launch_rebuild_tiles(const Dev& d, cudaStream_t st) {
  const int warp_blocks = blocks_for(d.n_blocks * 32, kThreads);
  k_tiles_blocks<<<warp_blocks, kThreads, 0, st>>>(d);
  k_tiles_count<<<warp_blocks, kThreads, 0, st>>>(d);
  k_tiles_scan<<<d.S < 148 ? d.S : 148, kThreads, 0, st>>>(d);
  k_tiles_fill<<<warp_blocks, kThreads, 0, st>>>(d);
  k_tiles_exclusions<<<blocks_for(d.n_excl, kThreads), kThreads, 0, st>>>(d);
  k_tiles_finish<<<1, 32, 0, st>>>(d);
}

}  // namespace mdb
