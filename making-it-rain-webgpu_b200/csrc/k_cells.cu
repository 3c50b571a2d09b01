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
  long long na, nb, nc;        // lattice translation taken off
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
  f.na = na;
  f.nb = nb;
  f.nc = nc;
  return f;
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

// Exclusive scan of `in[0..n)` into `out`, one block, in order.  Returns the
// total.  Each warp owns a contiguous segment: pass one sums the segments
// (coalesced), the block adds up the warps before each, pass two scans every
// segment 32 elements at a time from its carry.
__device__ int block_exclusive_scan(const int* in, int* out, int n) {
  __shared__ int warp_total[kThreads / 32];
  __shared__ int total;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int per = ((n + nw - 1) / nw + 31) / 32 * 32;
  const int lo = min(n, warp * per), hi = min(n, lo + per);
  int sum = 0;
  for (int i = lo + lane; i < hi; i += 32) sum += in[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
  if (lane == 0) warp_total[warp] = sum;
  __syncthreads();
  int carry = 0;
  for (int w = 0; w < warp; ++w) carry += warp_total[w];
  if (threadIdx.x == 0) {
    int t = 0;
    for (int w = 0; w < nw; ++w) t += warp_total[w];
    total = t;
  }
  for (int base = lo; base < hi; base += 32) {
    const int i = base + lane;
    const int v = i < hi ? in[i] : 0;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (i < hi) out[i] = carry + x - v;
    carry += __shfl_sync(0xffffffffu, x, 31);
  }
  __syncthreads();
  const int t = total;
  __syncthreads();  // the shared words are free for the next call
  return t;
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

// Every step, every system: pair coordinates of each slot as int32 at
// 2^pc_shift per nm (cell-list.wgsl:140 `wrap`).  A rebuild folds each atom
// into the cell and records the lattice translation it took (three signed
// 10-bit counts); between rebuilds the same translation is applied, so the
// coordinates move continuously (an atom leaves the cell by at most half the
// skin before the next rebuild) and the tiles' lattice shifts stay valid.
//
// With an inner list, a system about to be pruned (or rebuilt) also takes its
// atoms' positions as the new prune reference and empties its inner list.
__device__ void phase_wrap(const Dev& d) {
  if (d.inner && blockIdx.x == 0)
    for (int s = threadIdx.x; s < d.S; s += blockDim.x)
      if (d.rebuild_now[s] || d.prune_now[s]) d.in_count[s] = 0;
  // Lanes of a warp hold 32 consecutive slots (n_slots is a multiple of 32),
  // one system's, so the inner-list branch below is warp-uniform.
  for (int gs = grid_stride_start(); gs < d.n_slots; gs += grid_stride()) {
    const int a = d.order[gs];
    const int s = d.slot_sys[gs];
    const SysDev& S = d.sys[s];
    int4 p = make_int4(0, 0, 0, 0);
    if (a >= 0) {
      if (d.inner && (d.rebuild_now[s] || d.prune_now[s])) {
        d.prx[a] = d.px[a];
        d.pry[a] = d.py[a];
        d.prz[a] = d.pz[a];
      }
      long long na, nb, nc;
      if (d.rebuild_now[s]) {
        const Folded f = fold(S, d.px[a], d.py[a], d.pz[a]);
        na = f.na;
        nb = f.nb;
        nc = f.nc;
        d.fold[gs] = int((na & 1023) | ((nb & 1023) << 10) | ((nc & 1023) << 20));
      } else {
        unpack_fold(d.fold[gs], na, nb, nc);
      }
      p = pair_coordinate(S, d.px[a], d.py[a], d.pz[a], na, nb, nc);
    }
    d.pc[gs] = p;
    if (d.inner && (d.rebuild_now[s] || d.prune_now[s])) {
      // the cluster's bounding box at these coordinates, for the inner prune
      const int C = d.cluster;
      float lo[3] = {3.0e38f, 3.0e38f, 3.0e38f}, hi[3] = {-3.0e38f, -3.0e38f, -3.0e38f};
      if (a >= 0) {
        lo[0] = hi[0] = p.x * S.pc_inv;
        lo[1] = hi[1] = p.y * S.pc_inv;
        lo[2] = hi[2] = p.z * S.pc_inv;
      }
      for (int o = C / 2; o > 0; o >>= 1)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          lo[k] = fminf(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], o, C));
          hi[k] = fmaxf(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], o, C));
        }
      if ((gs & (C - 1)) == 0) {
        d.cb_lo[gs / C] = make_float4(lo[0], lo[1], lo[2], 0.f);
        d.cb_hi[gs / C] = make_float4(hi[0], hi[1], hi[2], 0.f);
      }
    }
  }
}

// A group of C lanes per cluster (32/C clusters per warp): parameters in slot
// order, the cluster's bounding box, and the reference positions the
// displacement test measures against.  Every lane takes part in every
// shuffle; only the writes depend on whether the cluster's system rebuilds.
template <int C>
__device__ void phase_tiles_blocks(const Dev& d) {
  constexpr int G = 32 / C;
  const int lane = threadIdx.x & 31, g = lane / C, l = lane & (C - 1);
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int wb = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; wb * G < d.n_blocks; wb += warps) {
    const int b = wb * G + g;
    const bool valid = b < d.n_blocks;
    const int s = valid ? d.block_sys[b] : 0;
    const bool work = valid && d.rebuild_now[s];
    const SysDev& S = d.sys[s];
    const int gs = b * C + l;
    const int a = work ? d.order[gs] : -1;
    float lo[3] = {3.0e38f, 3.0e38f, 3.0e38f}, hi[3] = {-3.0e38f, -3.0e38f, -3.0e38f};
    if (work) {
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
    }
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int o = C / 2; o > 0; o >>= 1) {
        lo[k] = fminf(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], o, C));
        hi[k] = fmaxf(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], o, C));
      }
    if (work && l == 0) {
      d.bb_lo[b] = make_float4(lo[0], lo[1], lo[2], 0.f);
      d.bb_hi[b] = make_float4(hi[0], hi[1], hi[2], 0.f);
    }
    if (C < 32) {
      // the warp's 32/C clusters form one super-cluster (a system's clusters
      // start at a multiple of 32 slots, so it never straddles two systems)
#pragma unroll
      for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int o = C; o < 32; o <<= 1) {
          lo[k] = fminf(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], o));
          hi[k] = fmaxf(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], o));
        }
      if (work && lane == 0) {
        d.sb_lo[wb] = make_float4(lo[0], lo[1], lo[2], 0.f);
        d.sb_hi[wb] = make_float4(hi[0], hi[1], hi[2], 0.f);
      }
    }
  }
}

// Do two boxes of one system come within cutoff + skin under some periodic
// image?  Box-to-box gap distance, minimised over images.  An empty
// cluster's box is inverted (lo = +3e38, hi = -3e38): its gap is infinite.
__device__ __forceinline__ bool boxes_near(const SysDev& S, float4 li, float4 hi_, float4 lj, float4 hj) {
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
  // When every centre distance that could pass (list + both half-diagonals)
  // is below half the cell's narrowest width, the sequential reduction above
  // already gives the minimum image, as it does for the reference's cutoff.
  const bool one_image = !S.triclinic || sqrtf(S.list2) + sqrtf(hx * hx + hy * hy + hz * hz) < 0.5f * S.min_width;
  if (one_image) {
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

// The lattice shift (in pair-coordinate units, applied to J) of the image
// that brings box J nearest box I, as boxes_near finds it; w carries that
// image's lattice counts (so a box change can recompute the shift without a
// rebuild) and the per-pair flag, set when that
// one image might not hold every pair of the tile within the cutoff: when
// 2 (|h_I| + |h_J|) + list + cutoff reaches the cell's narrowest width (h the
// half-diagonals), another image of some pair could come inside the cutoff,
// and the pair kernel takes the minimum image per pair instead.
__device__ __forceinline__ int4 tile_image(const SysDev& S, float4 li, float4 hi_, float4 lj, float4 hj) {
  float dx = 0.5f * (lj.x + hj.x) - 0.5f * (li.x + hi_.x);
  float dy = 0.5f * (lj.y + hj.y) - 0.5f * (li.y + hi_.y);
  float dz = 0.5f * (lj.z + hj.z) - 0.5f * (li.z + hi_.z);
  const float* B = S.box_f;
  const float kc = rintf(dz / B[8]);
  dx -= kc * B[6]; dy -= kc * B[7]; dz -= kc * B[8];
  const float kb = rintf(dy / B[4]);
  dx -= kb * B[3]; dy -= kb * B[4];
  const float ka = rintf(dx / B[0]);
  dx -= ka * B[0];
  int na = -int(ka), nb = -int(kb), nc = -int(kc);
  const float hx = 0.5f * (hi_.x - li.x) + 0.5f * (hj.x - lj.x);
  const float hy = 0.5f * (hi_.y - li.y) + 0.5f * (hj.y - lj.y);
  const float hz = 0.5f * (hi_.z - li.z) + 0.5f * (hj.z - lj.z);
  if (S.triclinic && sqrtf(S.list2) + sqrtf(hx * hx + hy * hy + hz * hz) >= 0.5f * S.min_width) {
    float best = 3.0e38f;
    int bi = 0, bj = 0, bk = 0;
    for (int k = -1; k <= 1; ++k)
      for (int j = -1; j <= 1; ++j)
        for (int i = -1; i <= 1; ++i) {
          const float x = dx + i * B[0] + j * B[3] + k * B[6];
          const float y = dy + j * B[4] + k * B[7];
          const float z = dz + k * B[8];
          const float gx = fmaxf(fabsf(x) - hx, 0.f), gy = fmaxf(fabsf(y) - hy, 0.f), gz = fmaxf(fabsf(z) - hz, 0.f);
          const float g = gx * gx + gy * gy + gz * gz;
          if (g < best) {
            best = g;
            bi = i;
            bj = j;
            bk = k;
          }
        }
    na += bi;
    nb += bj;
    nc += bk;
  }
  // wrapping 32-bit arithmetic: the pair kernel adds this to a coordinate and
  // subtracts another; the result, a separation inside the cutoff, fits
  const unsigned int sx = unsigned(na) * unsigned(S.pc_box[0]) + unsigned(nb) * unsigned(S.pc_box[3]) +
                          unsigned(nc) * unsigned(S.pc_box[6]);
  const unsigned int sy = unsigned(nb) * unsigned(S.pc_box[4]) + unsigned(nc) * unsigned(S.pc_box[7]);
  const unsigned int sz = unsigned(nc) * unsigned(S.pc_box[8]);
  const float ei = 0.5f * sqrtf((hi_.x - li.x) * (hi_.x - li.x) + (hi_.y - li.y) * (hi_.y - li.y) +
                                (hi_.z - li.z) * (hi_.z - li.z));
  const float ej = 0.5f * sqrtf((hj.x - lj.x) * (hj.x - lj.x) + (hj.y - lj.y) * (hj.y - lj.y) +
                                (hj.z - lj.z) * (hj.z - lj.z));
  const bool per_pair = 2.f * (ei + ej) + sqrtf(S.list2) + sqrtf(S.cut2) >= S.min_width;
  return make_int4(int(sx), int(sy), int(sz), tile_flags(per_pair, na, nb, nc));
}

// Position of the k-th (from 0) set bit of m, or -1.
__device__ __forceinline__ int nth_set_bit(unsigned int m, int k) {
  for (int i = 0; i < k && m; ++i) m &= m - 1;
  return m ? __ffs(m) - 1 : -1;
}

// Tiles of row I, in ascending J.  The search is two-level: the 32-slot
// super-cluster of J (kSub = 32 / C clusters) must come near I's cluster
// before the clusters inside it are tested, 32 / kSub super-clusters to a
// pass of the warp, and every near tile is written by its own lane.  The
// count pass (WRITE false) sizes the rows; after the scan the fill pass
// (WRITE true) writes them at their place in the dense list.  Rows vary a lot:
// a cluster that straddles a jump of the space-filling curve (where it leaves
// the sort grid and comes back) has a large box and a long row.
template <int C, bool WRITE>
__device__ void phase_tiles_find(const Dev& d) {
  constexpr int kSub = 32 / C;         // clusters per super-cluster
  constexpr int kBatch = 32 / kSub;    // super-clusters per pass
  constexpr int kWords = C * C / 32;   // mask words per tile
  constexpr unsigned kRowAll = C == 32 ? 0xffffffffu : ((1u << C) - 1u);
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  const unsigned below = (1u << lane) - 1u;
  for (int I = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; I < d.n_blocks; I += warps) {
    const int s = d.block_sys[I];
    if (!d.rebuild_now[s]) continue;
    const SysDev& S = d.sys[s];
    // the row's tiles go to [base, base + cap) of the dense list
    const long long base = static_cast<long long>(S.tile_off) + (WRITE ? d.tile_start[I] : 0);
    const int cap = WRITE ? min(d.tile_cnt[I], S.tile_cap - d.tile_start[I]) : 0;
    const int sI = I / kSub, sEnd = (S.block_off + S.n_blocks) / kSub;
    const float4 li = d.bb_lo[I], hi_ = d.bb_hi[I];
    const int Il = I - S.block_off;
    int count = 0;
    for (int J0 = sI; J0 < sEnd; J0 += 32) {
      const int SJ = J0 + lane;
      const bool near = SJ < sEnd && boxes_near(S, li, hi_, d.sb_lo[SJ], d.sb_hi[SJ]);
      const unsigned int supers = __ballot_sync(0xffffffffu, near);
      if (C == 32) {
        // no super level: the boxes tested are the clusters themselves, and a
        // 32x32 tile's mask is one word per row, so every lane writes its row
        const unsigned int found = __ballot_sync(0xffffffffu, near && SJ >= I);
        unsigned int f = found;
        while (f) {
          const int src = __ffs(f) - 1;
          f &= f - 1;
          const int Jt = J0 + src;
          const int pos = count + __popc(found & ((1u << src) - 1u));
          if (WRITE && pos < cap) {
            if (lane == 0) {
              (d.prune ? d.raw_tiles : d.tiles)[base + pos] = make_int2(I, Jt);
              (d.prune ? d.raw_shift : d.tile_shift)[base + pos] = tile_image(S, li, hi_, d.bb_lo[Jt], d.bb_hi[Jt]);
            }
            const int Jl = Jt - S.block_off;
            const int nj = max(0, min(C, S.n_atoms - Jl * C));
            unsigned int valid = nj >= C ? kRowAll : ((1u << nj) - 1u);
            if (Jt == I) valid &= lane == C - 1 ? 0u : (kRowAll << (lane + 1));
            if (Il * C + lane >= S.n_atoms) valid = 0u;
            (d.prune ? d.raw_masks : d.masks)[(base + pos) * kWords + lane] = valid;
          }
        }
        count += __popc(found);
        continue;
      }
      unsigned int rest = supers;
      while (rest) {
        // lanes k * kSub .. k * kSub + kSub - 1 take the k-th remaining near super-cluster
        const int k = lane / kSub, sub = lane % kSub;
        const int nth = nth_set_bit(rest, k);
        const int J = nth >= 0 ? (J0 + nth) * kSub + sub : -1;
        const bool tile = J >= I && boxes_near(S, li, hi_, d.bb_lo[J], d.bb_hi[J]);
        const unsigned int found = __ballot_sync(0xffffffffu, tile);
        const int at = count + __popc(found & below);
        if (WRITE && tile && at < cap) {
          (d.prune ? d.raw_tiles : d.tiles)[base + at] = make_int2(I, J);
          (d.prune ? d.raw_shift : d.tile_shift)[base + at] = tile_image(S, li, hi_, d.bb_lo[J], d.bb_hi[J]);
          const int Jl = J - S.block_off;
          const int nj = max(0, min(C, S.n_atoms - Jl * C));
          const unsigned int cols = nj >= C ? kRowAll : ((1u << nj) - 1u);
          unsigned int words[kWords];
#pragma unroll
          for (int w = 0; w < kWords; ++w) words[w] = 0u;
#pragma unroll
          for (int r = 0; r < C; ++r) {
            unsigned int row = Il * C + r < S.n_atoms ? cols : 0u;
            if (J == I) row &= r == C - 1 ? 0u : ((kRowAll << (r + 1)) & kRowAll);
            words[(r * C) >> 5] |= row << ((r * C) & 31);
          }
#pragma unroll
          unsigned int* masks = d.prune ? d.raw_masks : d.masks;
#pragma unroll
          for (int w = 0; w < kWords; ++w) masks[(base + at) * kWords + w] = words[w];
        }
        count += __popc(found);
        for (int b = 0; b < kBatch && rest; ++b) rest &= rest - 1;  // the super-clusters this pass took
      }
    }
    if (!WRITE && lane == 0) {
      d.tile_cnt[I] = count;
      d.row_alive[I] = 0;
    }
  }
}

__device__ void phase_tiles_scan(const Dev& d) {
  for (int s = blockIdx.x; s < d.S; s += gridDim.x) {
    if (!d.rebuild_now[s]) continue;
    const SysDev& S = d.sys[s];
    const int total = block_exclusive_scan(d.tile_cnt + S.block_off, d.tile_start + S.block_off, S.n_blocks);
    if (threadIdx.x == 0) {
      // a list that needs more tiles than the system's capacity is cut there,
      // and the engine's halt word stops the integrator, so no step runs on
      // the cut list: the host grows the capacity to `tile_need` and rebuilds
      // before it runs the remaining steps
      d.tile_need[s] = total;
      if (total > S.tile_cap) {
        atomicOr(&d.err[s], kErrTileCapacity);
        atomicExch(d.halt, 1);
      }
      d.tile_count[s] = total < S.tile_cap ? total : S.tile_cap;
    }
  }
}

// Drop the tiles whose atoms are all farther apart than cutoff + skin (the
// box test is conservative: about a fifth of 8x8 tiles have no pair inside).
// Tiles are spread over every warp, 32/C at a time, one group of C lanes per
// tile running the pair kernel's rotation on distances only; the verdict goes
// to tile_alive and the row's survivor count.
template <int C>
__device__ void phase_tiles_prune(const Dev& d) {
  constexpr int G = 32 / C;
  const int lane = threadIdx.x & 31, g = lane / C, l = lane & (C - 1);
  const int warps = (gridDim.x * blockDim.x) >> 5;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int src = (l + 1) & (C - 1);
  constexpr unsigned kGroup = C == 32 ? 0xffffffffu : ((1u << C) - 1u);
  for (int s = 0; s < d.S; ++s) {
    if (!d.rebuild_now[s]) continue;
    const SysDev& S = d.sys[s];
    const int n = d.tile_count[s];
    const float inv = S.pc_inv, list2 = S.list2 * (1.0f + 1e-5f);
    for (int b = warp * G; b < n; b += warps * G) {
      const int t = b + g;
      const bool active = t < n;
      const long long ti = S.tile_off + (active ? t : 0);
      const int2 tile = d.raw_tiles[ti];
      const int4 sh = d.raw_shift[ti];
      unsigned int mask = active ? row_bits<C>(d.raw_masks, ti, l) : 0u;
      mask = (mask >> l) | (mask << ((C - l) & (C - 1)));  // bit k <-> j = l + k (mod C)
      const int4 pi = d.pc[tile.x * C + l];
      int4 pj = d.pc[tile.y * C + l];
      if (!tile_per_pair(sh.w)) {
        pj.x = int(unsigned(pj.x) + unsigned(sh.x));
        pj.y = int(unsigned(pj.y) + unsigned(sh.y));
        pj.z = int(unsigned(pj.z) + unsigned(sh.z));
      }
      bool hit = false;
#pragma unroll
      for (int k = 0; k < C; ++k) {
        int dx = int(unsigned(pj.x) - unsigned(pi.x)), dy = int(unsigned(pj.y) - unsigned(pi.y)),
            dz = int(unsigned(pj.z) - unsigned(pi.z));
        if (tile_per_pair(sh.w)) {
          if (S.triclinic) min_image<true>(S, dx, dy, dz);
          else min_image<false>(S, dx, dy, dz);
        }
        const float rx = dx * inv, ry = dy * inv, rz = dz * inv;
        hit |= ((mask >> k) & 1u) && rx * rx + ry * ry + rz * rz < list2;
        pj.x = __shfl_sync(0xffffffffu, pj.x, src, C);
        pj.y = __shfl_sync(0xffffffffu, pj.y, src, C);
        pj.z = __shfl_sync(0xffffffffu, pj.z, src, C);
      }
      const unsigned int hits = __ballot_sync(0xffffffffu, hit);
      const bool alive = ((hits >> (g * C)) & kGroup) != 0u;
      if (active && l == 0) {
        d.tile_alive[ti] = alive ? 1 : 0;
        if (alive) atomicAdd(&d.row_alive[tile.x], 1);
      }
    }
  }
}

__device__ void phase_tiles_rescan(const Dev& d) {
  for (int s = blockIdx.x; s < d.S; s += gridDim.x) {
    if (!d.rebuild_now[s]) continue;
    const SysDev& S = d.sys[s];
    const int total = block_exclusive_scan(d.row_alive + S.block_off, d.alive_start + S.block_off, S.n_blocks);
    if (threadIdx.x == 0) d.tile_count[s] = total;
  }
}

// Warp per row: the row's surviving tiles, in order, into the list the pair
// kernel reads; the row's start and count follow them.
template <int C>
__device__ void phase_tiles_compact(const Dev& d) {
  constexpr int kWords = C * C / 32;
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int I = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; I < d.n_blocks; I += warps) {
    const int s = d.block_sys[I];
    if (!d.rebuild_now[s]) continue;
    const SysDev& S = d.sys[s];
    const int old_start = d.tile_start[I], old_n = min(d.tile_cnt[I], S.tile_cap - old_start);
    const int new_start = d.alive_start[I];
    int written = 0;
    for (int k0 = 0; k0 < old_n; k0 += 32) {
      const int k = k0 + lane;
      const long long src = static_cast<long long>(S.tile_off) + old_start + k;
      const bool keep = k < old_n && d.tile_alive[src];
      const unsigned int keepers = __ballot_sync(0xffffffffu, keep);
      const long long dst = static_cast<long long>(S.tile_off) + new_start + written +
                            __popc(keepers & ((1u << lane) - 1u));
      if (keep) {
        d.tiles[dst] = d.raw_tiles[src];
        d.tile_shift[dst] = d.raw_shift[src];
        if (C < 32)
          for (int w = 0; w < kWords; ++w) d.masks[dst * kWords + w] = d.raw_masks[src * kWords + w];
      }
      if (C == 32) {
        // a 32x32 tile's mask is 32 words: the warp copies each kept tile's
        unsigned int f = keepers;
        while (f) {
          const int from = __ffs(f) - 1;
          f &= f - 1;
          const long long sidx = static_cast<long long>(S.tile_off) + old_start + k0 + from;
          const long long didx = static_cast<long long>(S.tile_off) + new_start + written +
                                 __popc(keepers & ((1u << from) - 1u));
          d.masks[didx * kWords + lane] = d.raw_masks[sidx * kWords + lane];
        }
      }
      written += __popc(keepers);
    }
    if (lane == 0) {
      d.tile_start[I] = new_start;
      d.tile_cnt[I] = written;
    }
  }
}

// Clear the mask bit of every excluded pair in the tile that holds it.
template <int C>
__device__ void phase_tiles_exclusions(const Dev& d) {
  for (int e = grid_stride_start(); e < d.n_excl; e += grid_stride()) {
    const int s = d.excl_sys[e];
    if (!d.rebuild_now[s]) continue;
    const SysDev& S = d.sys[s];
    const int2 pr = d.excl[e];
    int sa = d.rank[pr.x], sb = d.rank[pr.y];
    if (sa > sb) { const int t = sa; sa = sb; sb = t; }
    const int I = S.block_off + sa / C, J = S.block_off + sb / C;
    const int row = sa % C, bit = sb % C;
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
    if (lo < d.tile_start[I] + d.tile_cnt[I] && lo < S.tile_cap && d.tiles[S.tile_off + lo].y == J) {
      const long long t = static_cast<long long>(S.tile_off) + lo;
      if (C == 32) atomicAnd(&d.masks[t * 32 + row], ~(1u << bit));
      else atomicAnd(&d.masks[t * (C * C / 32) + (row >> 2)], ~(1u << ((row & 3) * 8 + bit)));
    }
  }
}

// The inner list of every system that rebuilt or is due a prune: the outer
// tiles with an unexcluded pair closer than cutoff + inner skin (GROMACS's
// dynamic pruning, Pall et al., J. Chem. Phys. 153, 134110 (2020), made
// exact: a prune is due as soon as any atom has moved half the inner skin, so
// a dropped tile has no pair inside the cutoff until the next one and the
// pair kernel's results are bit-identical to running the whole outer list).
// A warp takes 32 consecutive outer tiles and one atomicAdd reserves room for
// the survivors, which keep their order.  Chunks land in any order; the pair
// kernel's sums do not depend on it (per-tile f32 partials become int64 fixed
// point), and a chunk spans at most two rows.
//
// 8x8 tiles: one lane per tile; a tile whose clusters' current boxes are out
// of reach is dropped at once, the others test their pairs until the first one
// within reach, on f32 offsets from the tile's first atom (exact integer
// differences, then one rounding), with the J cluster in registers --
// independent loads and no shuffles.  Tiles flagged for per-pair images (the
// cell is too small for one shift per tile) take each pair's minimum image, as
// the pair kernel does, in cells narrower than cutoff + list radius + 1 nm,
// where nearly every tile is flagged; in wider cells the few flagged tiles
// are kept without a test.  32x32 tiles (too many registers for that) keep a tile if some
// atom of I is within reach of J's current bounding box and some atom of J of
// I's, which any pair within reach implies: conservative, one lane per atom.
template <int C>
__device__ bool tile_within_reach(const Dev& d, const SysDev& S, long long ti, float reach2, int lane);

template <>
__device__ bool tile_within_reach<8>(const Dev& d, const SysDev& S, long long ti, float reach2, int) {
  const int2 tile = __ldcg(&d.tiles[ti]);
  const int4 sh = __ldcg(&d.tile_shift[ti]);
  const float inv = S.pc_inv;
  if (tile_per_pair(sh.w)) {
    if (!S.prune_per_pair) return true;
    // per-pair images (small cells): the pair kernel's own minimum image of each pair
    const unsigned int w0 = __ldcg(&d.masks[ti * 2]), w1 = __ldcg(&d.masks[ti * 2 + 1]);
    int4 qj[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) qj[j] = d.pc[tile.y * 8 + j];
    for (int i = 0; i < 8; ++i) {
      const unsigned int row = ((i < 4 ? w0 : w1) >> ((i & 3) * 8)) & 0xFFu;
      if (!row) continue;
      const int4 qi = d.pc[tile.x * 8 + i];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        if (!((row >> j) & 1u)) continue;
        int dx = int(unsigned(qj[j].x) - unsigned(qi.x)), dy = int(unsigned(qj[j].y) - unsigned(qi.y)),
            dz = int(unsigned(qj[j].z) - unsigned(qi.z));
        if (S.triclinic) min_image<true>(S, dx, dy, dz);
        else min_image<false>(S, dx, dy, dz);
        const float rx = dx * inv, ry = dy * inv, rz = dz * inv;
        if (rx * rx + ry * ry + rz * rz < reach2) return true;
      }
    }
    return false;
  }
  {
    // the clusters' current boxes first: most outer tiles of a long skin are
    // out of reach box to box and need no pair loop (the margin covers the
    // boxes' f32 rounding)
    const float4 ilo = d.cb_lo[tile.x], ihi = d.cb_hi[tile.x], jlo = d.cb_lo[tile.y], jhi = d.cb_hi[tile.y];
    const float sx = sh.x * inv, sy = sh.y * inv, sz = sh.z * inv;
    const float gx = fmaxf(fmaxf(jlo.x + sx - ihi.x, ilo.x - (jhi.x + sx)), 0.f);
    const float gy = fmaxf(fmaxf(jlo.y + sy - ihi.y, ilo.y - (jhi.y + sy)), 0.f);
    const float gz = fmaxf(fmaxf(jlo.z + sz - ihi.z, ilo.z - (jhi.z + sz)), 0.f);
    if (gx * gx + gy * gy + gz * gz >= reach2 * (1.0f + 4e-5f)) return false;
  }
  const unsigned int w0 = __ldcg(&d.masks[ti * 2]), w1 = __ldcg(&d.masks[ti * 2 + 1]);
  // both clusters' sixteen atoms in one round of loads, then the 64 tests
  // (loading each i atom inside the loop made a chain of eight round trips)
  int4 qi[8], qj[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    qi[k] = d.pc[tile.x * 8 + k];
    qj[k] = d.pc[tile.y * 8 + k];
  }
  const int4 r0 = qi[0];
  const unsigned ox = unsigned(r0.x) - unsigned(sh.x), oy = unsigned(r0.y) - unsigned(sh.y),
                 oz = unsigned(r0.z) - unsigned(sh.z);
  float jx[8], jy[8], jz[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    jx[j] = int(unsigned(qj[j].x) - ox) * inv;
    jy[j] = int(unsigned(qj[j].y) - oy) * inv;
    jz[j] = int(unsigned(qj[j].z) - oz) * inv;
  }
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const unsigned int row = ((i < 4 ? w0 : w1) >> ((i & 3) * 8)) & 0xFFu;
    const float ix = int(unsigned(qi[i].x) - unsigned(r0.x)) * inv,
                iy = int(unsigned(qi[i].y) - unsigned(r0.y)) * inv,
                iz = int(unsigned(qi[i].z) - unsigned(r0.z)) * inv;
    bool hit = false;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const float dx = jx[j] - ix, dy = jy[j] - iy, dz = jz[j] - iz;
      hit |= ((row >> j) & 1u) && dx * dx + dy * dy + dz * dz < reach2;
    }
    if (hit) return true;  // most kept tiles stop at their first rows
  }
  return false;
}

template <>
__device__ bool tile_within_reach<32>(const Dev& d, const SysDev& S, long long ti, float reach2, int l) {
  const int2 tile = __ldcg(&d.tiles[ti]);
  const int4 sh = __ldcg(&d.tile_shift[ti]);
  const unsigned int row = __ldcg(&d.masks[ti * 32 + l]);
  const unsigned int cols = __reduce_or_sync(0xffffffffu, row);
  if (tile_per_pair(sh.w)) return true;  // warp-uniform: one tile per warp
  const float inv = S.pc_inv;
  const float4 ilo = d.cb_lo[tile.x], ihi = d.cb_hi[tile.x];
  const float4 jlo = d.cb_lo[tile.y], jhi = d.cb_hi[tile.y];
  const float sx = sh.x * inv, sy = sh.y * inv, sz = sh.z * inv;
  const int4 qi = d.pc[tile.x * 32 + l], qj = d.pc[tile.y * 32 + l];
  const float ix = qi.x * inv, iy = qi.y * inv, iz = qi.z * inv;
  const float jx = qj.x * inv + sx, jy = qj.y * inv + sy, jz = qj.z * inv + sz;
  const float ax = fmaxf(fmaxf(jlo.x + sx - ix, ix - (jhi.x + sx)), 0.f);
  const float ay = fmaxf(fmaxf(jlo.y + sy - iy, iy - (jhi.y + sy)), 0.f);
  const float az = fmaxf(fmaxf(jlo.z + sz - iz, iz - (jhi.z + sz)), 0.f);
  const float bx = fmaxf(fmaxf(ilo.x - jx, jx - ihi.x), 0.f);
  const float by = fmaxf(fmaxf(ilo.y - jy, jy - ihi.y), 0.f);
  const float bz = fmaxf(fmaxf(ilo.z - jz, jz - ihi.z), 0.f);
  const bool hit_i = row != 0u && ax * ax + ay * ay + az * az < reach2;
  const bool hit_j = ((cols >> l) & 1u) && bx * bx + by * by + bz * bz < reach2;
  return __any_sync(0xffffffffu, hit_i) && __any_sync(0xffffffffu, hit_j);
}

template <int C>
__device__ void phase_inner(const Dev& d) {
  constexpr int kWords = C * C / 32;
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  for (int s = 0; s < d.S; ++s) {
    if (!d.rebuild_now[s] && !d.prune_now[s]) continue;
    const SysDev& S = d.sys[s];
    const int n = min(d.tile_count[s], S.tile_cap);
    const float reach2 = S.inner2 * (1.0f + 1e-5f);
    // each system's first chunk goes to the warp after the previous system's
    // last (the outer list's offsets, which this kernel only reads), so a
    // batch of small systems spreads over every warp instead of the first few
    const int first = (d.tile_prefix[s] >> 5) % warps;
    for (int c0 = ((warp - first + warps) % warps) * 32; c0 < n; c0 += warps * 32) {
      unsigned int keep = 0u;  // bit k: outer tile c0 + k survives (the same in every lane)
      if (C == 8) {
        const bool alive = c0 + lane < n && tile_within_reach<C>(d, S, S.tile_off + c0 + lane, reach2, lane);
        keep = __ballot_sync(0xffffffffu, alive);
      } else {
        for (int k = 0; k < 32 && c0 + k < n; ++k)
          if (tile_within_reach<C>(d, S, S.tile_off + c0 + k, reach2, lane)) keep |= 1u << k;
      }
      const int count = __popc(keep);
      int base = 0;
      if (lane == 0 && count) base = atomicAdd(&d.in_count[s], count);
      base = __shfl_sync(0xffffffffu, base, 0);
      if ((keep >> lane) & 1u) {
        const long long from = static_cast<long long>(S.tile_off) + c0 + lane;
        const long long to = static_cast<long long>(S.tile_off) + base + __popc(keep & ((1u << lane) - 1u));
        d.in_tiles[to] = __ldcg(&d.tiles[from]);
        d.in_shift[to] = __ldcg(&d.tile_shift[from]);
        if (C < 32) {
#pragma unroll
          for (int w = 0; w < kWords; ++w) d.in_masks[to * kWords + w] = __ldcg(&d.masks[from * kWords + w]);
        }
      }
      if (C == 32) {
        // a 32x32 tile's mask is 32 words: the warp copies each kept tile's
        unsigned int f = keep;
        while (f) {
          const int k = __ffs(f) - 1;
          f &= f - 1;
          const long long from = static_cast<long long>(S.tile_off) + c0 + k;
          const long long to = static_cast<long long>(S.tile_off) + base + __popc(keep & ((1u << k) - 1u));
          d.in_masks[to * kWords + lane] = __ldcg(&d.masks[from * kWords + lane]);
        }
      }
    }
  }
}

// After the outer list: per-system offsets and rebuild counts.  Without an
// inner list the rebuild requests are cleared here; with one, the inner-list
// kernel that follows still needs them and clears them itself.
__device__ void phase_tiles_finish(const Dev& d) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    int total = 0;
    for (int s = 0; s < d.S; ++s) {
      d.tile_prefix[s] = total;
      total += d.tile_count[s];
      if (d.rebuild_now[s]) d.rebuild_count[s] += 1;
      if (!d.inner) d.rebuild_now[s] = 0;
    }
    d.tile_prefix[d.S] = total;
    if (!d.inner) *d.any_rebuild = 0;
  }
}

// After the inner list (one thread): its offsets, the prune count, and every
// list request cleared for the next step.
__device__ void inner_finish(const Dev& d) {
  int total = 0;
  for (int s = 0; s < d.S; ++s) {
    d.in_prefix[s] = total;
    total += d.in_count[s];
    if (d.prune_now[s] && !d.rebuild_now[s]) d.prune_count[s] += 1;
    d.prune_now[s] = 0;
    d.rebuild_now[s] = 0;
  }
  d.in_prefix[d.S] = total;
  *d.any_rebuild = 0;
  *d.any_prune = 0;
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

// One launch per step.  With no rebuild requested it returns at once, or folds
// the pair coordinates when a prune is due; otherwise it runs the sort and
// tile-list phases with a grid barrier between them.
template <int C>
__global__ void __launch_bounds__(kThreads) k_list(Dev d) {
  const bool rebuild = *d.any_rebuild != 0;
  int* err = d.err;  // system 0's word carries a barrier timeout
  if (!rebuild) {
    // the integrator wrote this step's pair coordinates; the wrap runs again
    // only for a prune, which needs reference positions and cluster boxes
    if (*d.any_prune) phase_wrap(d);
    return;
  }
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
  phase_tiles_blocks<C>(d);
  if (!grid_barrier(d.list_barrier, err)) return;
  phase_tiles_find<C, false>(d);
  if (!grid_barrier(d.list_barrier, err)) return;
  phase_tiles_scan(d);
  if (!grid_barrier(d.list_barrier, err)) return;
  phase_tiles_find<C, true>(d);
  if (!grid_barrier(d.list_barrier, err)) return;
  if (d.prune) {
    phase_tiles_prune<C>(d);
    if (!grid_barrier(d.list_barrier, err)) return;
    phase_tiles_rescan(d);
    if (!grid_barrier(d.list_barrier, err)) return;
    phase_tiles_compact<C>(d);
    if (!grid_barrier(d.list_barrier, err)) return;
  }
  phase_tiles_exclusions<C>(d);
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
MDB_PHASE_KERNEL(tiles_scan, true)
MDB_PHASE_KERNEL(tiles_rescan, true)
MDB_PHASE_KERNEL(tiles_finish, true)
#undef MDB_PHASE_KERNEL
// the wrap, when a rebuild or a prune is due (otherwise the integrator wrote
// the pair coordinates at the end of the previous step)
__global__ void __launch_bounds__(kThreads) k_wrap(Dev d) {
  if (!*d.any_rebuild && !*d.any_prune) return;
  phase_wrap(d);
}
// The inner list, its own launch after the list kernels (a full grid, where
// the cooperative list kernel has two blocks per SM): nothing to do unless a
// system rebuilt or is due a prune.  The last block to finish writes the
// offsets and clears the requests; every block has read them by then, since
// each reads them before taking its ticket.
template <int C>
__global__ void __launch_bounds__(kThreads) k_inner_prune(Dev d) {
  wait_for_predecessor();
  release_successor();
  if (!*d.any_rebuild && !*d.any_prune) return;
  phase_inner<C>(d);
  __shared__ int last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(d.inner_ticket, 1) == int(gridDim.x) - 1;
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    inner_finish(d);
    *d.inner_ticket = 0;
  }
}
#define MDB_PHASE_KERNEL_C(name)                                   \
  template <int C>                                                 \
  __global__ void __launch_bounds__(kThreads) k_##name(Dev d) {   \
    if (!*d.any_rebuild) return;                                   \
    phase_##name<C>(d);                                            \
  }
MDB_PHASE_KERNEL_C(tiles_blocks)
MDB_PHASE_KERNEL_C(tiles_prune)
MDB_PHASE_KERNEL_C(tiles_compact)
template <int C>
__global__ void __launch_bounds__(kThreads) k_tiles_count(Dev d) {
  if (!*d.any_rebuild) return;
  phase_tiles_find<C, false>(d);
}
template <int C>
__global__ void __launch_bounds__(kThreads) k_tiles_fill(Dev d) {
  if (!*d.any_rebuild) return;
  phase_tiles_find<C, true>(d);
}
MDB_PHASE_KERNEL_C(tiles_exclusions)
#undef MDB_PHASE_KERNEL_C

int blocks_for(int n, int threads, int cap = 148 * 8) {
  const int b = (n + threads - 1) / threads;
  return b < 1 ? 1 : (b > cap ? cap : b);
}

int g_list_grid = 0;

}  // namespace

// Size the cooperative grid once: every block resident at the same time.
int prepare_list_kernel(int device) {
  int per_sm = 0, sms = 0;
  int per_sm8 = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_list<32>, kThreads, 0) != cudaSuccess) return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm8, k_list<8>, kThreads, 0) != cudaSuccess) return 0;
  per_sm = std::min(per_sm, per_sm8);
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
  if (d.cluster == 8) return cudaLaunchKernelEx(&cfg, k_list<8>, d) == cudaSuccess;
  return cudaLaunchKernelEx(&cfg, k_list<32>, d) == cudaSuccess;
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

template <int C>
void rebuild_tiles(const Dev& d, cudaStream_t st) {
  const int warp_blocks = blocks_for(d.n_blocks * 32, kThreads);
  k_tiles_blocks<C><<<warp_blocks, kThreads, 0, st>>>(d);
  k_tiles_count<C><<<warp_blocks, kThreads, 0, st>>>(d);
  k_tiles_scan<<<d.S < 148 ? d.S : 148, kThreads, 0, st>>>(d);
  k_tiles_fill<C><<<warp_blocks, kThreads, 0, st>>>(d);
  if (d.prune) {
    k_tiles_prune<C><<<148 * 4, kThreads, 0, st>>>(d);
    k_tiles_rescan<<<d.S < 148 ? d.S : 148, kThreads, 0, st>>>(d);
    k_tiles_compact<C><<<warp_blocks, kThreads, 0, st>>>(d);
  }
  k_tiles_exclusions<C><<<blocks_for(d.n_excl, kThreads), kThreads, 0, st>>>(d);
  k_tiles_finish<<<1, 32, 0, st>>>(d);
}

void launch_inner_prune(const Dev& d, cudaStream_t st) {
  if (!d.inner) return;
  if (d.cluster == 8) launch_chained(k_inner_prune<8>, 148 * 4, kThreads, 0, st, d);
  else launch_chained(k_inner_prune<32>, 148 * 4, kThreads, 0, st, d);
}

void launch_rebuild_tiles(const Dev& d, cudaStream_t st) {
  if (d.cluster == 8) rebuild_tiles<8>(d, st);
  else rebuild_tiles<32>(d, st);
}

}  // namespace mdb
