// k_pme.cu -- reciprocal-space PME: B-spline spread, 3D real-to-complex FFT
// with the Ewald convolution fused into the x pass, complex-to-real FFT, and
// the force gather.
//
// Physics follows src/gpu/kernels/pme.wgsl:124 (spread), fft.wgsl:60,
// pme-convolve.wgsl:34, pme-interpolate.wgsl:105 and the f64 oracle
// src/reference/forces/pme.ts:93-263: order-5 cardinal B-splines on a mesh
// laid out in fractional coordinates, E = sum_k f(k) |Q(k)|^2 with
// f = (2 pi / V) ONE_4PI_EPS0 exp(-k^2/4a^2) / (k^2 |b(m)|^2), and the grid
// multiplied by 2 f before the inverse transform.
//
// B200 shape:
//   * the spline argument u = r . (K o B^-1) is formed exactly in 2^32 fixed
//     point from the int64 positions (a 64x64->128-bit product), so the grid
//     index and the weight fraction carry no f32 coordinate rounding;
//   * the charge grid is int64 fixed point filled with atomics, so the spread
//     is order independent and runs are bit-identical;
//   * the transform is three passes, each CTA running a Stockham mixed-radix
//     (2, 3, 4, 5, 7) FFT over whole lines in shared memory: one CTA per
//     x-plane does z (int64 -> complex, real-to-complex, clearing the grid it
//     read) and y; the x pass does x forward + convolution + x inverse; one
//     CTA per x-plane does y inverse and z complex-to-real.  Meshes whose
//     planes do not fit shared memory take separate z and y passes (five in
//     all).  The reference's 7-13 global passes per direction and its
//     separate load/convolve passes disappear.
#include <array>
#include <cmath>
#include <cstring>
#include <mutex>

#include "device_state.h"
#include "prep.h"

namespace mdb {
namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// exp(-2 pi i t / R) for the small DFTs.
__constant__ float2 kRoot3[3] = {{1.f, 0.f}, {-0.500000000f, -0.866025404f}, {-0.500000000f, 0.866025404f}};
__constant__ float2 kRoot5[5] = {{1.f, 0.f},
                                 {0.309016994f, -0.951056516f},
                                 {-0.809016994f, -0.587785252f},
                                 {-0.809016994f, 0.587785252f},
                                 {0.309016994f, 0.951056516f}};
__constant__ float2 kRoot7[7] = {{1.f, 0.f},
                                 {0.623489802f, -0.781831482f},
                                 {-0.222520934f, -0.974927912f},
                                 {-0.900968868f, -0.433883739f},
                                 {-0.900968868f, 0.433883739f},
                                 {-0.222520934f, 0.974927912f},
                                 {0.623489802f, 0.781831482f}};

template <int R>
__device__ __forceinline__ float2 root(int t, int sign) {
  float2 w;
  if (R == 3) w = kRoot3[t];
  else if (R == 5) w = kRoot5[t];
  else w = kRoot7[t];
  if (sign > 0) w.y = -w.y;
  return w;
}

template <int R>
__device__ __forceinline__ void small_dft(float2* v, int sign) {
  if (R == 2) {
    const float2 a = v[0], b = v[1];
    v[0] = make_float2(a.x + b.x, a.y + b.y);
    v[1] = make_float2(a.x - b.x, a.y - b.y);
  } else if (R == 4) {
    const float2 a0 = make_float2(v[0].x + v[2].x, v[0].y + v[2].y);
    const float2 a1 = make_float2(v[0].x - v[2].x, v[0].y - v[2].y);
    const float2 b0 = make_float2(v[1].x + v[3].x, v[1].y + v[3].y);
    float2 b1 = make_float2(v[1].x - v[3].x, v[1].y - v[3].y);
    // multiply by -i (forward) or +i (inverse)
    b1 = sign < 0 ? make_float2(b1.y, -b1.x) : make_float2(-b1.y, b1.x);
    v[0] = make_float2(a0.x + b0.x, a0.y + b0.y);
    v[2] = make_float2(a0.x - b0.x, a0.y - b0.y);
    v[1] = make_float2(a1.x + b1.x, a1.y + b1.y);
    v[3] = make_float2(a1.x - b1.x, a1.y - b1.y);
  } else {
    float2 out[R];
#pragma unroll
    for (int m = 0; m < R; ++m) {
      float2 s = v[0];
#pragma unroll
      for (int q = 1; q < R; ++q) {
        const float2 w = root<R>((m * q) % R, sign);
        s.x += v[q].x * w.x - v[q].y * w.y;
        s.y += v[q].x * w.y + v[q].y * w.x;
      }
      out[m] = s;
    }
#pragma unroll
    for (int m = 0; m < R; ++m) v[m] = out[m];
  }
}

// Quotient by a per-stage divisor d > 1 without a division: magic = 2^32 / d
// rounded up is exact for numerator x divisor < 2^32 (all FFT indices here
// are below 2^16).  d = 1 (magic 0) means the numerator itself.
__device__ __forceinline__ unsigned quotient(unsigned x, unsigned magic) { return magic ? __umulhi(x, magic) : x; }
__host__ __device__ __forceinline__ unsigned magic_for(unsigned d) { return d > 1 ? 0xFFFFFFFFu / d + 1u : 0u; }

template <int R>
__device__ __forceinline__ void stage_butterfly(const float2* src, float2* dst, int n, int j, int ns,
                                                unsigned ns_magic, int step, const float2* tw, int sign) {
  const int bf = n / R;
  const int jq = int(quotient(unsigned(j), ns_magic));
  const int k = j - jq * ns;
  float2 v[R];
#pragma unroll
  for (int q = 0; q < R; ++q) {
    float2 x = src[j + q * bf];
    if (q > 0 && k > 0) {
      float2 w = tw[k * q * step];  // k q step < ns R step = n
      if (sign > 0) w.y = -w.y;
      x = cmul(x, w);
    }
    v[q] = x;
  }
  small_dft<R>(v, sign);
  const int dest = jq * ns * R + k;
#pragma unroll
  for (int q = 0; q < R; ++q) dst[dest + q * ns] = v[q];
}

// A transform's twiddle table (n entries) into shared memory, where the
// butterflies read it: a global read in every butterfly stage otherwise.
__device__ __forceinline__ void stage_twiddles(float2* dst, const float2* src, int n) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = __ldg(&src[i]);
}

// Stockham autosort over `nl` lines of length n in shared memory
// (src/reference/fft.ts:128 is the f64 restatement of the same recursion).
// Returns the buffer holding the result.
__device__ float2* fft_lines(float2* a, float2* b, int n, int nl, const int* radices, int nrad,
                             const float2* tw, int sign) {
  int ns = 1;
  for (int st = 0; st < nrad; ++st) {
    const int r = radices[st];
    const int bf = n / r;
    const int step = n / (ns * r);
    const unsigned bf_magic = magic_for(unsigned(bf)), ns_magic = magic_for(unsigned(ns));
    for (int idx = threadIdx.x; idx < nl * bf; idx += blockDim.x) {
      const int line = int(quotient(unsigned(idx), bf_magic)), j = idx - line * bf;
      const float2* src = a + line * n;
      float2* dst = b + line * n;
      switch (r) {
        case 2: stage_butterfly<2>(src, dst, n, j, ns, ns_magic, step, tw, sign); break;
        case 3: stage_butterfly<3>(src, dst, n, j, ns, ns_magic, step, tw, sign); break;
        case 4: stage_butterfly<4>(src, dst, n, j, ns, ns_magic, step, tw, sign); break;
        case 5: stage_butterfly<5>(src, dst, n, j, ns, ns_magic, step, tw, sign); break;
        default: stage_butterfly<7>(src, dst, n, j, ns, ns_magic, step, tw, sign); break;
      }
    }
    __syncthreads();
    float2* t = a;
    a = b;
    b = t;
    ns *= r;
  }
  return a;
}

// ------------------------------------------------------------- splines ----
// Order-5 cardinal B-spline weights and derivatives at fraction w
// (src/reference/forces/bspline.ts:55, the same recursion in f32).
__device__ __forceinline__ void bspline5(float w, float* th, float* dth) {
  float lo[5];
  lo[0] = 1.f - w;
  lo[1] = w;
  lo[2] = 0.f;
  lo[3] = 0.f;
  lo[4] = 0.f;
#pragma unroll
  for (int k = 3; k <= 4; ++k) {
    const float dv = 1.f / (k - 1);
    lo[k - 1] = dv * w * lo[k - 2];
#pragma unroll
    for (int j = 1; j < k - 1; ++j) lo[k - j - 1] = dv * ((w + j) * lo[k - j - 2] + (k - j - w) * lo[k - j - 1]);
    lo[0] = dv * (1.f - w) * lo[0];
  }
  if (dth) {
    dth[0] = -lo[0];
#pragma unroll
    for (int j = 1; j < 5; ++j) dth[j] = lo[j - 1] - lo[j];
  }
#pragma unroll
  for (int j = 0; j < 5; ++j) th[j] = lo[j];
  const float dv = 0.25f;
  th[4] = dv * w * th[3];
#pragma unroll
  for (int j = 1; j < 4; ++j) th[4 - j] = dv * ((w + j) * th[3 - j] + (5 - j - w) * th[4 - j]);
  th[0] = dv * (1.f - w) * th[0];
}

struct Spline {
  int base[3];
  float th[3][5], dth[3][5];
};

__device__ __forceinline__ void spline_for(const SysDev& S, long long x, long long y, long long z,
                                           Spline& sp, bool derivatives) {
  const long long u[3] = {fixed_mul(x, S.umat[0]) + fixed_mul(y, S.umat[1]) + fixed_mul(z, S.umat[2]),
                          fixed_mul(y, S.umat[3]) + fixed_mul(z, S.umat[4]), fixed_mul(z, S.umat[5])};
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const long long cell = u[k] >> 32;
    const float w = static_cast<float>(static_cast<unsigned int>(u[k] & 0xffffffffll)) * 2.3283064365386963e-10f;
    long long b = (cell - (kPmeOrder - 1)) % S.grid[k];
    if (b < 0) b += S.grid[k];
    sp.base[k] = static_cast<int>(b);
    bspline5(w, sp.th[k], derivatives ? sp.dth[k] : nullptr);
  }
}

// ---------------------------------------------------------------- spread --
// Both spreads read nothing the list kernels write, so they run on their own
// stream while the list kernels sort and rebuild.
//
// By atom (engines under one block of slots per SM): a block takes up to
// kSplineAtoms atoms: their splines are computed once each into shared memory,
// then all its threads share the 25 (ix, iy) rows of 5 z points per atom, so
// no thread makes more than a few atomics in a row (one thread per atom making
// all 125 left the kernel latency-bound at any size).  Consecutive atoms are
// neighbours in space (molecules, solvent laid down in order), so block b
// takes atoms b, b + B, b + 2B, ... (B blocks): atoms spread at once sit far
// apart on the mesh.  The grid is int64 fixed point: the order of the atomics
// does not change the sums.
constexpr int kSplineAtoms = 128;  // at most; 32, 64 and 256 measured slower
static_assert(kSplineAtoms <= kThreads, "one thread per atom computes the splines");

struct SplineTable {
  int base[kSplineAtoms][3];
  float th[kSplineAtoms][3][5];
  float q[kSplineAtoms];
  int sys[kSplineAtoms];
};

__global__ void __launch_bounds__(kThreads) k_spread(Dev d, int per) {
  wait_for_predecessor();
  __shared__ SplineTable t;
  const int nblocks = gridDim.x;
  for (int first = blockIdx.x; first < d.n_atoms; first += nblocks * per) {
    // atom k (< per <= kSplineAtoms) of this round is first + k * nblocks
    if (threadIdx.x < per) {
      const int k = threadIdx.x, a = first + k * nblocks;
      float q = 0.f;
      if (a < d.n_atoms && sys_active(d, d.atom_sys[a])) q = d.prm_atom[a].w;
      t.q[k] = q;
      if (q != 0.f) {
        const int s = d.atom_sys[a];
        Spline sp;
        spline_for(d.sys[s], d.px[a], d.py[a], d.pz[a], sp, false);
        t.sys[k] = s;
        for (int ax = 0; ax < 3; ++ax) {
          t.base[k][ax] = sp.base[ax];
          for (int i = 0; i < kPmeOrder; ++i) t.th[k][ax][i] = sp.th[ax][i];
        }
      }
    }
    __syncthreads();
    for (int w = threadIdx.x; w < per * kPmeOrder * kPmeOrder; w += blockDim.x) {
      const int k = w / (kPmeOrder * kPmeOrder), r = w - k * kPmeOrder * kPmeOrder;
      const float q = t.q[k];
      if (q == 0.f) continue;
      const SysDev& S = d.sys[t.sys[k]];
      const int Kx = S.grid[0], Ky = S.grid[1], Kz = S.grid[2];
      const int ix = r / kPmeOrder, iy = r - ix * kPmeOrder;
      int gx = t.base[k][0] + ix;
      if (gx >= Kx) gx -= Kx;
      int gy = t.base[k][1] + iy;
      if (gy >= Ky) gy -= Ky;
      const float wxy = q * t.th[k][0][ix] * t.th[k][1][iy];
      unsigned long long* row = d.qgrid + S.grid_off + (static_cast<long long>(gx) * Ky + gy) * Kz;
#pragma unroll
      for (int iz = 0; iz < kPmeOrder; ++iz) {
        int gz = t.base[k][2] + iz;
        if (gz >= Kz) gz -= Kz;
        add_fixed(&row[gz], wxy * t.th[k][2][iz]);
      }
    }
    __syncthreads();
  }
}

// By slot (larger engines): the slots of a snapshot of the list's sorted
// order that the integrator writes at the end of every step (`spread_atom`),
// so the order the list kernels are rewriting is never read.  A block takes
// 128 consecutive slots -- four super-clusters along the space-filling curve,
// a compact piece of space -- adds their charges into a patch of the mesh in
// shared memory, and adds the patch's nonzero points to the grid: about a
// fifth of the global atomics of spreading each atom's 125 points directly.
// The patch holds the block's spline bases (unwrapped around its first atom)
// plus the 5-point stencil; a block whose patch would not fit (a cluster torn
// across a jump of the curve) or whose slots reach into the next system
// spreads directly.  Every contribution is the same fixed-point value as in
// the by-atom spread, so the grid is the same to the bit.  The shared-memory
// phases make a block's chain longer: below one block per SM (the 12k-atom
// peptide) the by-atom kernel finishes first; above it this one takes less
// time (the 27k-atom octahedron 7% less, a 64-system ensemble of 627k atoms
// 45% less).
constexpr int kPatchSlots = 128;
constexpr int kPatchPoints = 4096;  // 32 KB of int64

__global__ void __launch_bounds__(kThreads) k_spread_sorted(Dev d) {
  wait_for_predecessor();
  // the patch's fixed-point sums in two 32-bit halves (hi = v >> 20 signed,
  // lo = the low 20 bits), so the adds are 32-bit shared atomics: at most 128
  // atoms add to a point, which keeps both halves far from overflow
  __shared__ int patch_hi[kPatchPoints];
  __shared__ unsigned int patch_lo[kPatchPoints];
  __shared__ int base[kPatchSlots][3];
  __shared__ float th[kPatchSlots][3][5];
  __shared__ float qs[kPatchSlots];
  __shared__ int sysk[kPatchSlots];
  __shared__ int lo_part[kPatchSlots / 32][3], hi_part[kPatchSlots / 32][3];
  __shared__ int lo[3], ext[3], use_patch;
  const int first = blockIdx.x * kPatchSlots;
  if (first >= d.n_slots) return;
  const int last = min(d.n_slots, first + kPatchSlots) - 1;
  // a block may hold the end of one system and the start of the next: then
  // every atom spreads directly into its own system's grid
  const int s = d.slot_sys[first];
  const bool one_system = d.slot_sys[last] == s;
  const int a0 = d.spread_atom[first];
  if (one_system && (a0 < 0 || !sys_active(d, s))) return;  // padding only, or a skipped system
  const SysDev& S = d.sys[s];
  const int K[3] = {S.grid[0], S.grid[1], S.grid[2]};
  // splines; in a one-system block the bases unwrapped around the first slot's atom
  const int t = threadIdx.x;
  int ub[3] = {0, 0, 0};
  bool live = false;
  if (t < kPatchSlots) {
    const int gs = first + t;
    float q = 0.f;
    int st = s;
    if (gs <= last) {
      st = d.slot_sys[gs];
      const int a = d.spread_atom[gs];
      if (a >= 0 && sys_active(d, st)) q = d.prm_atom[a].w;
      if (q != 0.f) {
        const SysDev& Sa = d.sys[st];
        Spline sp;
        spline_for(Sa, d.px[a], d.py[a], d.pz[a], sp, false);
        Spline sp0;
        if (one_system) spline_for(S, d.px[a0], d.py[a0], d.pz[a0], sp0, false);
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) {
          int b = sp.base[ax];
          if (one_system) {
            const int r = sp0.base[ax];
            if (b - r > K[ax] / 2) b -= K[ax];
            if (r - b > K[ax] / 2) b += K[ax];
          }
          ub[ax] = b;
          base[t][ax] = b;
          for (int i = 0; i < kPmeOrder; ++i) th[t][ax][i] = sp.th[ax][i];
        }
        live = true;
      }
    }
    qs[t] = q;
    sysk[t] = st;
  }
  // the bases' range: warp reductions, then the block's
  if (t < kPatchSlots) {
    const int big = 1 << 30;
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
      const int mn = __reduce_min_sync(0xffffffffu, live ? ub[ax] : big);
      const int mx = __reduce_max_sync(0xffffffffu, live ? ub[ax] : -big);
      if ((t & 31) == 0) {
        lo_part[t >> 5][ax] = mn;
        hi_part[t >> 5][ax] = mx;
      }
    }
  }
  __syncthreads();
  if (t == 0) {
    int points = 1;
    bool fits = one_system;
    for (int ax = 0; ax < 3; ++ax) {
      int mn = lo_part[0][ax], mx = hi_part[0][ax];
      for (int w = 1; w < kPatchSlots / 32; ++w) {
        mn = min(mn, lo_part[w][ax]);
        mx = max(mx, hi_part[w][ax]);
      }
      lo[ax] = mn;
      ext[ax] = mx - mn + kPmeOrder;
      fits = fits && mx >= mn && ext[ax] <= K[ax];
      points *= max(ext[ax], 1);
    }
    use_patch = fits && points <= kPatchPoints;
  }
  __syncthreads();
  if (use_patch) {
    const int ex = ext[0], ey = ext[1], ez = ext[2], np = ex * ey * ez;
    for (int i = t; i < np; i += blockDim.x) {
      patch_hi[i] = 0;
      patch_lo[i] = 0u;
    }
    __syncthreads();
    for (int w = t; w < kPatchSlots * kPmeOrder * kPmeOrder; w += blockDim.x) {
      const int k = w / (kPmeOrder * kPmeOrder), r = w - k * kPmeOrder * kPmeOrder;
      const float q = qs[k];
      if (q == 0.f) continue;
      const int ix = r / kPmeOrder, iy = r - ix * kPmeOrder;
      const float wxy = q * th[k][0][ix] * th[k][1][iy];
      const int row = ((base[k][0] - lo[0] + ix) * ey + (base[k][1] - lo[1] + iy)) * ez + (base[k][2] - lo[2]);
#pragma unroll
      for (int iz = 0; iz < kPmeOrder; ++iz) {
        const long long v = to_fixed(wxy * th[k][2][iz]);
        atomicAdd(&patch_hi[row + iz], static_cast<int>(v >> 20));
        atomicAdd(&patch_lo[row + iz], static_cast<unsigned int>(v & 0xFFFFF));
      }
    }
    __syncthreads();
    for (int i = t; i < np; i += blockDim.x) {
      const unsigned long long v = static_cast<unsigned long long>(
          (static_cast<long long>(patch_hi[i]) << 20) + static_cast<long long>(patch_lo[i]));
      if (!v) continue;
      const int px = i / (ey * ez), rem = i - px * ey * ez, py = rem / ez, pz = rem - py * ez;
      int gx = (lo[0] + px) % K[0], gy = (lo[1] + py) % K[1], gz = (lo[2] + pz) % K[2];
      if (gx < 0) gx += K[0];
      if (gy < 0) gy += K[1];
      if (gz < 0) gz += K[2];
      atomicAdd(d.qgrid + S.grid_off + (static_cast<long long>(gx) * K[1] + gy) * K[2] + gz, v);
    }
  } else {
    // the direct spread of each atom's 125 points, into its own system's grid
    for (int w = t; w < kPatchSlots * kPmeOrder * kPmeOrder; w += blockDim.x) {
      const int k = w / (kPmeOrder * kPmeOrder), r = w - k * kPmeOrder * kPmeOrder;
      const float q = qs[k];
      if (q == 0.f) continue;
      const SysDev& Sk = d.sys[sysk[k]];
      const int Kx = Sk.grid[0], Ky = Sk.grid[1], Kz = Sk.grid[2];
      const int ix = r / kPmeOrder, iy = r - ix * kPmeOrder;
      int gx = (base[k][0] + ix) % Kx, gy = (base[k][1] + iy) % Ky;
      if (gx < 0) gx += Kx;
      if (gy < 0) gy += Ky;
      const float wxy = q * th[k][0][ix] * th[k][1][iy];
      unsigned long long* row = d.qgrid + Sk.grid_off + (static_cast<long long>(gx) * Ky + gy) * Kz;
#pragma unroll
      for (int iz = 0; iz < kPmeOrder; ++iz) {
        int gz = (base[k][2] + iz) % Kz;
        if (gz < 0) gz += Kz;
        add_fixed(&row[gz], wxy * th[k][2][iz]);
      }
    }
  }
}

// --------------------------------------------------------------- z pass ---
// int64 charge grid -> complex half spectrum along z, clearing the grid.
__global__ void __launch_bounds__(kThreads) k_fft_z_forward(Dev d) {
  wait_for_predecessor();
  extern __shared__ float2 smem[];
  const FftWork w = d.fft_z[blockIdx.x];
  if (!sys_active(d, w.sys)) return;  // the whole block: before any barrier
  const SysDev& S = d.sys[w.sys];
  const int Kz = S.grid[2], kzh = S.kzh;
  float2* A = smem;
  float2* B = smem + w.n * Kz;
  unsigned long long* grid = d.qgrid + S.grid_off + static_cast<long long>(w.a) * Kz;
  for (int i = threadIdx.x; i < w.n * Kz; i += blockDim.x) {
    const long long v = static_cast<long long>(grid[i]);
    A[i] = make_float2(from_fixed(v), 0.f);
    grid[i] = 0ull;
  }
  __syncthreads();
  const float2* R = fft_lines(A, B, Kz, w.n, S.radices[2], S.nradix[2], d.twiddles + S.tw_off[2], -1);
  float2* out = d.cgrid + S.cgrid_off + static_cast<long long>(w.a) * kzh;
  for (int i = threadIdx.x; i < w.n * kzh; i += blockDim.x) {
    const int line = i / kzh, k = i - line * kzh;
    out[i] = R[line * Kz + k];
  }
}

// --------------------------------------------------------------- y pass ---
__global__ void __launch_bounds__(kThreads) k_fft_y(Dev d, int sign) {
  wait_for_predecessor();
  extern __shared__ float2 smem[];
  const FftWork w = d.fft_y[blockIdx.x];
  if (!sys_active(d, w.sys)) return;  // the whole block: before any barrier
  const SysDev& S = d.sys[w.sys];
  const int Ky = S.grid[1], kzh = S.kzh;
  float2* A = smem;
  float2* B = smem + w.n * Ky;
  float2* base = d.cgrid + S.cgrid_off + static_cast<long long>(w.a) * Ky * kzh + w.b;
  for (int i = threadIdx.x; i < w.n * Ky; i += blockDim.x) {
    const int y = i / w.n, l = i - y * w.n;
    A[l * Ky + y] = base[static_cast<long long>(y) * kzh + l];
  }
  __syncthreads();
  const float2* R = fft_lines(A, B, Ky, w.n, S.radices[1], S.nradix[1], d.twiddles + S.tw_off[1], sign);
  for (int i = threadIdx.x; i < w.n * Ky; i += blockDim.x) {
    const int y = i / w.n, l = i - y * w.n;
    base[static_cast<long long>(y) * kzh + l] = R[l * Ky + y];
  }
}

// ------------------------------------------- x pass with the convolution ---
// The Ewald influence function (pme-convolve.wgsl:34; pme.ts:160-209) at
// mesh index (mx, my, kz) of the half spectrum, mb the signed y index; the
// wave vector and its square come back for the virial.  0 at the origin.
// Written with explicit roundings so the table and the energy variant agree
// to the bit.
__device__ __forceinline__ float influence(const SysDev& S, const float* modx, const float* mody, const float* modz,
                                           int Kx, int mx, int mb, int my, int kz, float& kx, float& ky, float& kzv,
                                           float& k2) {
  if (mx == 0 && my == 0 && kz == 0) return 0.f;
  const float two_pi = 6.283185307179586f;
  const float* M = S.inv_f;
  const float ma = static_cast<float>(mx <= Kx / 2 ? mx : mx - Kx), fb = static_cast<float>(mb),
              mc = static_cast<float>(kz);  // kz <= Kz/2 on the half spectrum
  kx = __fmul_rn(two_pi, __fmul_rn(ma, M[0]));
  ky = __fmul_rn(two_pi, fmaf(fb, M[4], __fmul_rn(ma, M[3])));
  kzv = __fmul_rn(two_pi, fmaf(mc, M[8], fmaf(fb, M[7], __fmul_rn(ma, M[6]))));
  k2 = fmaf(kzv, kzv, fmaf(ky, ky, __fmul_rn(kx, kx)));
  const float den = __fmul_rn(__fmul_rn(__fmul_rn(k2, modx[mx]), mody[my]), modz[kz]);
  return __fdiv_rn(__fmul_rn(S.pme_pref, expf(__fmul_rn(k2, S.exp_scale))), den);
}

// The influence function of every x-pass work item of system `s` (all
// systems: s < 0), in the order the x pass visits its elements.  Run after
// every change of a box.
__global__ void __launch_bounds__(kThreads) k_influence(Dev d, int s) {
  const FftWork w = d.fft_x[blockIdx.x];
  if (s >= 0 && w.sys != s) return;
  const SysDev& S = d.sys[w.sys];
  const int Kx = S.grid[0], Ky = S.grid[1];
  const float* modx = d.moduli + S.mod_off;
  const float* mody = modx + Kx;
  const float* modz = mody + Ky;
  const int my = w.a, mb = my <= Ky / 2 ? my : my - Ky;
  float* table = d.influence + static_cast<long long>(blockIdx.x) * d.influence_stride;
  for (int i = threadIdx.x; i < w.n * Kx; i += blockDim.x) {
    const int l = i / Kx, mx = i - l * Kx;
    float kx, ky, kzv, k2;
    table[i] = influence(S, modx, mody, modz, Kx, mx, mb, my, w.b + l, kx, ky, kzv, k2);
  }
}

template <bool ENERGY>
__global__ void __launch_bounds__(kThreads) k_fft_x_convolve(Dev d) {
  wait_for_predecessor();
  extern __shared__ float2 smem[];
  __shared__ double partial[7][kThreads / 32];
  const FftWork w = d.fft_x[blockIdx.x];
  if (!sys_active(d, w.sys)) return;  // the whole block: before any barrier
  const SysDev& S = d.sys[w.sys];
  const int Kx = S.grid[0], Ky = S.grid[1], Kz = S.grid[2], kzh = S.kzh;
  float2* A = smem;
  float2* B = smem + w.n * Kx;
  float2* twx = smem + 2 * kFftTile * Kx;  // the twiddles, after the two tiles of lines
  stage_twiddles(twx, d.twiddles + S.tw_off[0], Kx);
  const long long stride = static_cast<long long>(Ky) * kzh;
  float2* base = d.cgrid + S.cgrid_off + static_cast<long long>(w.a) * kzh + w.b;
  const unsigned n_magic = magic_for(unsigned(w.n)), kx_magic = magic_for(unsigned(Kx));
  for (int i0 = threadIdx.x; i0 < w.n * Kx; i0 += 2 * blockDim.x) {
    float2 v[2];
    int x[2], l[2];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const int i = i0 + u * blockDim.x;
      x[u] = int(quotient(unsigned(i), n_magic));
      l[u] = i - x[u] * w.n;
      v[u] = i < w.n * Kx ? __ldcg(&base[x[u] * stride + l[u]]) : make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int u = 0; u < 2; ++u)
      if (i0 + u * int(blockDim.x) < w.n * Kx) A[l[u] * Kx + x[u]] = v[u];
  }
  __syncthreads();
  float2* R = fft_lines(A, B, Kx, w.n, S.radices[0], S.nradix[0], twx, -1);
  float2* other = R == A ? B : A;
  // Convolution (pme-convolve.wgsl:34; pme.ts:160-209) on the half spectrum.
  double energy = 0.0;
  double vir[6] = {0, 0, 0, 0, 0, 0};  // xx yy zz xy xz yz
  const int my = w.a;
  const int mb = my <= Ky / 2 ? my : my - Ky;
  const float* modx = d.moduli + S.mod_off;
  const float* mody = modx + Kx;
  const float* modz = mody + Ky;
  // the force variant (every MD step) reads the influence function from the
  // table k_influence fills at every box change; the energy variant needs the
  // wave vectors for the virial and evaluates it here, the same function
  const float* table = d.influence + static_cast<long long>(blockIdx.x) * d.influence_stride;
  for (int i = threadIdx.x; i < w.n * Kx; i += blockDim.x) {
    const int l = int(quotient(unsigned(i), kx_magic)), mx = i - l * Kx;
    const int kz = w.b + l;
    float2 v = R[i];
    float factor, kx = 0.f, ky = 0.f, kzv = 0.f, k2 = 1.f;
    if (ENERGY) factor = influence(S, modx, mody, modz, Kx, mx, mb, my, kz, kx, ky, kzv, k2);
    else factor = __ldg(&table[i]);
    if (ENERGY) {
      const double weight = (kz == 0 || (2 * kz == Kz)) ? 1.0 : 2.0;
      const double ek =
          weight * static_cast<double>(factor) * (static_cast<double>(v.x) * v.x + static_cast<double>(v.y) * v.y);
      energy += ek;
      // -dE_k/d eps_ab = E_k (delta_ab - 2 k_a k_b (1/k^2 + 1/(4 alpha^2)))
      const double c = 2.0 * (1.0 / static_cast<double>(k2) - static_cast<double>(S.exp_scale));
      const double ka = kx, kb = ky, kc = kzv;
      vir[0] += ek * (1.0 - c * ka * ka);
      vir[1] += ek * (1.0 - c * kb * kb);
      vir[2] += ek * (1.0 - c * kc * kc);
      vir[3] -= ek * c * ka * kb;
      vir[4] -= ek * c * ka * kc;
      vir[5] -= ek * c * kb * kc;
    }
    v.x *= 2.f * factor;
    v.y *= 2.f * factor;
    R[i] = v;
  }
  __syncthreads();
  const float2* Q = fft_lines(R, other, Kx, w.n, S.radices[0], S.nradix[0], twx, +1);
  for (int i = threadIdx.x; i < w.n * Kx; i += blockDim.x) {
    const int x = int(quotient(unsigned(i), n_magic)), l = i - x * w.n;
    base[x * stride + l] = Q[l * Kx + x];
  }
  if (ENERGY) {
    // fixed-order block reduction in FP64: deterministic
    double val[7] = {energy, vir[0], vir[1], vir[2], vir[3], vir[4], vir[5]};
#pragma unroll
    for (int c = 0; c < 7; ++c) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) val[c] += __shfl_xor_sync(0xffffffffu, val[c], o);
      if ((threadIdx.x & 31) == 0) partial[c][threadIdx.x >> 5] = val[c];
    }
    __syncthreads();
    if (threadIdx.x < 7) {
      double total = 0.0;
      for (int k = 0; k < (blockDim.x >> 5); ++k) total += partial[threadIdx.x][k];
      if (threadIdx.x == 0) d.mesh_partial[blockIdx.x] = total;
      else d.mesh_virial[blockIdx.x * 6 + threadIdx.x - 1] = total;
    }
  }
}

// ------------------------------------------------- whole x-plane passes ---
// With the plane in shared memory one CTA does both the z and the y
// transforms of an x-plane (Ky x Kz grid points; 2 x 16 Ky Kz bytes), so a
// forward or inverse transform is three launches instead of five and the
// launches that remain have a plane of work each.
constexpr int kPlaneThreads = 512;

__global__ void __launch_bounds__(kPlaneThreads) k_fft_zy_forward(Dev d) {
  wait_for_predecessor();
  extern __shared__ float2 smem[];
  const FftWork w = d.fft_p[blockIdx.x];
  if (!sys_active(d, w.sys)) return;  // the whole block: before any barrier
  const SysDev& S = d.sys[w.sys];
  const int Ky = S.grid[1], Kz = S.grid[2], kzh = S.kzh;
  const unsigned ky_magic = magic_for(unsigned(Ky)), kzh_magic = magic_for(unsigned(kzh)),
                 rest_magic = magic_for(unsigned(Kz - kzh));
  float2* A = smem;
  float2* B = smem + Ky * Kz;
  float2* twz = smem + 2 * Ky * Kz;  // the twiddles, after the two planes
  float2* twy = twz + Kz;
  stage_twiddles(twz, d.twiddles + S.tw_off[2], Kz);
  stage_twiddles(twy, d.twiddles + S.tw_off[1], Ky);
  unsigned long long* grid = d.qgrid + S.grid_off + static_cast<long long>(w.a) * Ky * Kz;
  // four loads in flight per thread before any is used
  for (int i0 = threadIdx.x; i0 < Ky * Kz; i0 += 4 * blockDim.x) {
    long long v[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int i = i0 + u * blockDim.x;
      v[u] = i < Ky * Kz ? static_cast<long long>(__ldcg(&grid[i])) : 0;
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int i = i0 + u * blockDim.x;
      if (i < Ky * Kz) {
        A[i] = make_float2(from_fixed(v[u]), 0.f);
        grid[i] = 0ull;  // consumer clears: the next spread starts from zero
      }
    }
  }
  __syncthreads();
  float2* R = fft_lines(A, B, Kz, Ky, S.radices[2], S.nradix[2], twz, -1);
  float2* T = R == A ? B : A;
  // the half spectrum's kz columns become y-lines
  for (int i = threadIdx.x; i < kzh * Ky; i += blockDim.x) {
    const int k = int(quotient(unsigned(i), ky_magic)), y = i - k * Ky;
    T[k * Ky + y] = R[y * Kz + k];
  }
  __syncthreads();
  const float2* Y = fft_lines(T, R, Ky, kzh, S.radices[1], S.nradix[1], twy, -1);
  float2* out = d.cgrid + S.cgrid_off + static_cast<long long>(w.a) * Ky * kzh;
  for (int i = threadIdx.x; i < Ky * kzh; i += blockDim.x) {
    const int y = int(quotient(unsigned(i), kzh_magic)), k = i - y * kzh;
    out[i] = Y[k * Ky + y];
  }
}

__global__ void __launch_bounds__(kPlaneThreads) k_fft_yz_inverse(Dev d) {
  wait_for_predecessor();
  extern __shared__ float2 smem[];
  const FftWork w = d.fft_p[blockIdx.x];
  if (!sys_active(d, w.sys)) return;  // the whole block: before any barrier
  const SysDev& S = d.sys[w.sys];
  const int Ky = S.grid[1], Kz = S.grid[2], kzh = S.kzh;
  const unsigned ky_magic = magic_for(unsigned(Ky)), kzh_magic = magic_for(unsigned(kzh)),
                 rest_magic = magic_for(unsigned(Kz - kzh));
  float2* A = smem;
  float2* B = smem + Ky * Kz;
  float2* twz = smem + 2 * Ky * Kz;  // the twiddles, after the two planes
  float2* twy = twz + Kz;
  stage_twiddles(twz, d.twiddles + S.tw_off[2], Kz);
  stage_twiddles(twy, d.twiddles + S.tw_off[1], Ky);
  const float2* in = d.cgrid + S.cgrid_off + static_cast<long long>(w.a) * Ky * kzh;
  for (int i0 = threadIdx.x; i0 < Ky * kzh; i0 += 4 * blockDim.x) {
    float2 v[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int i = i0 + u * blockDim.x;
      v[u] = i < Ky * kzh ? __ldcg(&in[i]) : make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int i = i0 + u * blockDim.x;
      if (i < Ky * kzh) {
        const int y = int(quotient(unsigned(i), kzh_magic)), k = i - y * kzh;
        A[k * Ky + y] = v[u];
      }
    }
  }
  __syncthreads();
  float2* Y = fft_lines(A, B, Ky, kzh, S.radices[1], S.nradix[1], twy, +1);
  float2* Z = Y == A ? B : A;
  for (int i = threadIdx.x; i < Ky * kzh; i += blockDim.x) {
    const int y = int(quotient(unsigned(i), kzh_magic)), k = i - y * kzh;
    Z[y * Kz + k] = Y[k * Ky + y];
  }
  __syncthreads();
  // the rest of each z-line from Hermitian symmetry (the result is real)
  for (int i = threadIdx.x; i < Ky * (Kz - kzh); i += blockDim.x) {
    const int y = int(quotient(unsigned(i), rest_magic)), k = kzh + (i - y * (Kz - kzh));
    const float2 c = Z[y * Kz + (Kz - k)];
    Z[y * Kz + k] = make_float2(c.x, -c.y);
  }
  __syncthreads();
  const float2* R = fft_lines(Z, Y, Kz, Ky, S.radices[2], S.nradix[2], twz, +1);
  float* out = d.phi + S.grid_off + static_cast<long long>(w.a) * Ky * Kz;
  for (int i = threadIdx.x; i < Ky * Kz; i += blockDim.x) out[i] = R[i].x;
}

// ---------------------------------------------------------- z inverse ----
// complex half spectrum -> real potential grid along z.
__global__ void __launch_bounds__(kThreads) k_fft_z_inverse(Dev d) {
  wait_for_predecessor();
  extern __shared__ float2 smem[];
  const FftWork w = d.fft_z[blockIdx.x];
  if (!sys_active(d, w.sys)) return;  // the whole block: before any barrier
  const SysDev& S = d.sys[w.sys];
  const int Kz = S.grid[2], kzh = S.kzh;
  float2* A = smem;
  float2* B = smem + w.n * Kz;
  const float2* in = d.cgrid + S.cgrid_off + static_cast<long long>(w.a) * kzh;
  for (int i = threadIdx.x; i < w.n * kzh; i += blockDim.x) {
    const int line = i / kzh, k = i - line * kzh;
    A[line * Kz + k] = in[i];
  }
  __syncthreads();
  for (int i = threadIdx.x; i < w.n * (Kz - kzh); i += blockDim.x) {
    const int line = i / (Kz - kzh), k = kzh + (i - line * (Kz - kzh));
    const float2 c = A[line * Kz + (Kz - k)];
    A[line * Kz + k] = make_float2(c.x, -c.y);
  }
  __syncthreads();
  const float2* R = fft_lines(A, B, Kz, w.n, S.radices[2], S.nradix[2], d.twiddles + S.tw_off[2], +1);
  float* out = d.phi + S.grid_off + static_cast<long long>(w.a) * Kz;
  for (int i = threadIdx.x; i < w.n * Kz; i += blockDim.x) out[i] = R[i].x;
}

// ---------------------------------------------------------------- gather --
__global__ void __launch_bounds__(kThreads) k_gather(Dev d) {
  wait_for_predecessor();
  for (int gs = blockIdx.x * blockDim.x + threadIdx.x; gs < d.n_slots; gs += gridDim.x * blockDim.x) {
    const int a = d.order[gs];
    if (a < 0) continue;
    const float q = d.prm[gs].w;
    if (q == 0.f || !sys_active(d, d.slot_sys[gs])) continue;
    const SysDev& S = d.sys[d.slot_sys[gs]];
    Spline sp;
    spline_for(S, d.px[a], d.py[a], d.pz[a], sp, true);
    const int Kx = S.grid[0], Ky = S.grid[1], Kz = S.grid[2];
    const float* grid = d.phi + S.grid_off;
    float ga = 0.f, gb = 0.f, gc = 0.f;
    for (int ix = 0; ix < kPmeOrder; ++ix) {
      int gx = sp.base[0] + ix;
      if (gx >= Kx) gx -= Kx;
      for (int iy = 0; iy < kPmeOrder; ++iy) {
        int gy = sp.base[1] + iy;
        if (gy >= Ky) gy -= Ky;
        const float* row = grid + (static_cast<long long>(gx) * Ky + gy) * Kz;
        const float wxy = sp.th[0][ix] * sp.th[1][iy];
        const float dxy = sp.dth[0][ix] * sp.th[1][iy];
        const float xdy = sp.th[0][ix] * sp.dth[1][iy];
#pragma unroll
        for (int iz = 0; iz < kPmeOrder; ++iz) {
          int gz = sp.base[2] + iz;
          if (gz >= Kz) gz -= Kz;
          const float p = row[gz];
          ga = fmaf(p * dxy, sp.th[2][iz], ga);
          gb = fmaf(p * xdy, sp.th[2][iz], gb);
          gc = fmaf(p * wxy, sp.dth[2][iz], gc);
        }
      }
    }
    // F_v = -q sum_u (dE/du_u) K_u M[v][u]  (pme.ts:252-259)
    const float* U = S.umat_f;
    const float fx = -q * (ga * U[0] + gb * U[1] + gc * U[2]);
    const float fy = -q * (ga * U[3] + gb * U[4] + gc * U[5]);
    const float fz = -q * (ga * U[6] + gb * U[7] + gc * U[8]);
    add_fixed(&d.fx[gs], fx);
    add_fixed(&d.fy[gs], fy);
    add_fixed(&d.fz[gs], fz);
  }
}

int grid_blocks(int n) {
  int b = (n + kThreads - 1) / kThreads;
  if (b > 148 * 16) b = 148 * 16;
  return b < 1 ? 1 : b;
}

}  // namespace

// Shared-memory bytes for the largest work item of each pass, set by the host.
struct PmeSmem { int z, y, x, p; };
static PmeSmem g_smem{0, 0, 0, 0};
void set_pme_smem(int z, int y, int x, int plane) {
  g_smem = {z, y, x, plane};
  if (plane > 0) {
    cudaFuncSetAttribute(k_fft_zy_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, plane);
    cudaFuncSetAttribute(k_fft_yz_inverse, cudaFuncAttributeMaxDynamicSharedMemorySize, plane);
  }
  cudaFuncSetAttribute(k_fft_z_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, z);
  cudaFuncSetAttribute(k_fft_z_inverse, cudaFuncAttributeMaxDynamicSharedMemorySize, z);
  cudaFuncSetAttribute(k_fft_y, cudaFuncAttributeMaxDynamicSharedMemorySize, y);
  cudaFuncSetAttribute(k_fft_x_convolve<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, x);
  cudaFuncSetAttribute(k_fft_x_convolve<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, x);
}

// Engines with at least one block of 128 slots per SM spread by slot: the
// 27k-atom octahedron (205 blocks) spreads in 25.5 us by slot against 27.5 us
// by atom, the 12k-atom peptide (96 blocks) in 15.5 us against 13.7 us.
bool spread_by_slot(int n_slots) { return (n_slots + kPatchSlots - 1) / kPatchSlots >= 148; }

void launch_pme_spread(const Dev& d, cudaStream_t st) {
  if (d.n_fft_z == 0) return;
  if (d.spread_sorted) {
    launch_chained(k_spread_sorted, (d.n_slots + kPatchSlots - 1) / kPatchSlots, kThreads, 0, st, d);
    return;
  }
  // about one block per two SMs, up to kSplineAtoms atoms each: small systems
  // get short blocks (latency), large ones full ones (fewer SMs taken from the
  // pair kernel running beside)
  const int per = std::max(16, std::min(kSplineAtoms, (d.n_atoms + 73) / 74));
  launch_chained(k_spread, std::max(1, std::min((d.n_atoms + per - 1) / per, 148 * 8)), kThreads, 0, st, d, per);
}

void launch_pme_fft(const Dev& d, bool energy, cudaStream_t st) {
  if (d.n_fft_z == 0) return;
  if (d.fft_planes) launch_chained(k_fft_zy_forward, d.n_fft_p, kPlaneThreads, g_smem.p, st, d);
  else {
    launch_chained(k_fft_z_forward, d.n_fft_z, kThreads, g_smem.z, st, d);
    launch_chained(k_fft_y, d.n_fft_y, kThreads, g_smem.y, st, d, -1);
  }
  if (energy) launch_chained(k_fft_x_convolve<true>, d.n_fft_x, kThreads, g_smem.x, st, d);
  else launch_chained(k_fft_x_convolve<false>, d.n_fft_x, kThreads, g_smem.x, st, d);
  if (d.fft_planes) launch_chained(k_fft_yz_inverse, d.n_fft_p, kPlaneThreads, g_smem.p, st, d);
  else {
    launch_chained(k_fft_y, d.n_fft_y, kThreads, g_smem.y, st, d, +1);
    launch_chained(k_fft_z_inverse, d.n_fft_z, kThreads, g_smem.z, st, d);
  }
}

void launch_influence(const Dev& d, int s, cudaStream_t st) {
  if (d.n_fft_x == 0) return;
  k_influence<<<d.n_fft_x, kThreads, 0, st>>>(d, s);
}

void launch_pme_gather(const Dev& d, cudaStream_t st) {
  if (d.n_fft_z == 0) return;
  // a thread per slot; blocks of 64 so that even 10k atoms spread over every SM
  launch_chained(k_gather, std::max(1, std::min((d.n_slots + 63) / 64, 148 * 16)), 64, 0, st, d);
}

void launch_pme(const Dev& d, bool energy, cudaStream_t st) {
  launch_pme_spread(d, st);
  launch_pme_fft(d, energy, st);
  launch_pme_gather(d, st);
}

}  // namespace mdb

// ===========================================================================
// Reciprocal-space PME with no allocation: for callers that cannot allocate
// device memory themselves -- code running inside another framework's memory
// pool, a host whose only device memory is what its own allocator hands out,
// or a real-time loop that forbids allocation after start-up.  The caller
// passes its own device buffers for the inputs and outputs; every
// intermediate (charge grid, half spectrum, potential, B-spline moduli,
// twiddles, energy partials) lives in one file-scope device array of fixed
// size, so this path never calls cudaMalloc, cudaFree or any allocating
// library routine.
//
// Limits: at most kNoAllocMaxMeshPoints mesh points (64^3), kNoAllocMaxAxis
// points per axis and at least kPmeOrder.  Every call uses the same array and leaves
// its contents behind; the charge grid is cleared at the start of each call.
// Two calls whose device work overlaps (different streams, or different host
// threads on one device) race on the array and must be serialised by the
// caller.
// ===========================================================================
namespace mdb {
namespace {

constexpr long long kNoAllocMaxMeshPoints = 64ll * 64 * 64;
constexpr int kNoAllocMaxAxis = 128;
constexpr int kNoAllocMaxPartials = kNoAllocMaxAxis * ((kNoAllocMaxAxis / 2 + 1 + 15) / 16);

// Byte offsets of the pieces inside the scratch array.
constexpr size_t kNaGrid = 0;                                           // int64 x K
constexpr size_t kNaSpectrum = kNaGrid + 8 * kNoAllocMaxMeshPoints;     // float2 x Kh (<= K)
constexpr size_t kNaPotential = kNaSpectrum + 8 * kNoAllocMaxMeshPoints;  // f32 x K
constexpr size_t kNaModuli = kNaPotential + 4 * kNoAllocMaxMeshPoints;  // f32 x 3 axes
constexpr size_t kNaTwiddles = kNaModuli + 4 * 3 * kNoAllocMaxAxis;     // float2 x 3 axes
constexpr size_t kNaPartials = kNaTwiddles + 8 * 3 * kNoAllocMaxAxis;   // f64 per x-pass CTA
constexpr size_t kNaBytes = kNaPartials + 8 * kNoAllocMaxPartials;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNaBytes];

struct NaPtrs {
  unsigned long long* grid;
  float2* spectrum;
  float* potential;
  float* moduli;
  float2* twiddles;
  double* partials;
};

// Moduli |b(m)|^2 of the order-5 spline (bspline.ts:102) and the twiddles
// exp(-2 pi i j / K) of each axis, computed on the device in FP64; and the
// charge grid cleared, because the array keeps the previous call's contents.
__global__ void k_na_setup(SysDev S, NaPtrs p) {
  const long long K = static_cast<long long>(S.grid[0]) * S.grid[1] * S.grid[2];
  for (long long i = blockIdx.x * blockDim.x + threadIdx.x; i < K; i += gridDim.x * blockDim.x) p.grid[i] = 0ull;
  if (blockIdx.x != 0) return;
  const double knots[4] = {1.0 / 24, 11.0 / 24, 11.0 / 24, 1.0 / 24};
  for (int axis = 0; axis < 3; ++axis) {
    const int n = S.grid[axis];
    float* mod = p.moduli + axis * kNoAllocMaxAxis;
    for (int m = threadIdx.x; m < n; m += blockDim.x) {
      double re = 0, im = 0;
      for (int k = 0; k < 4 && k < n; ++k) {
        double s, c;
        sincospi(2.0 * double((static_cast<long long>(m) * k) % n) / n, &s, &c);
        re += knots[k] * c;
        im += knots[k] * s;
      }
      mod[m] = float(re * re + im * im);
      double s, c;
      sincospi(-2.0 * m / n, &s, &c);
      p.twiddles[axis * kNoAllocMaxAxis + m] = make_float2(float(c), float(s));
    }
  }
  __syncthreads();
  // bspline.ts:126 -- replace a vanishing modulus by its neighbours' mean
  for (int axis = 0; axis < 3; ++axis) {
    const int n = S.grid[axis];
    float* mod = p.moduli + axis * kNoAllocMaxAxis;
    if (threadIdx.x == 0)
      for (int m = 0; m < n; ++m)
        if (mod[m] < 1e-7f) mod[m] = 0.5f * (mod[(m - 1 + n) % n] + mod[(m + 1) % n]);
  }
}

__device__ __forceinline__ long long fixed_from_double(double x) { return __double2ll_rn(x * 4294967296.0); }

__global__ void k_na_spread(SysDev S, NaPtrs p, int n, const double* pos, const double* charge) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float q = float(charge[i]);
    if (q == 0.f) continue;
    Spline sp;
    spline_for(S, fixed_from_double(pos[3 * i]), fixed_from_double(pos[3 * i + 1]),
               fixed_from_double(pos[3 * i + 2]), sp, false);
    const int Kx = S.grid[0], Ky = S.grid[1], Kz = S.grid[2];
    for (int ix = 0; ix < kPmeOrder; ++ix) {
      int gx = sp.base[0] + ix;
      if (gx >= Kx) gx -= Kx;
      const float wx = q * sp.th[0][ix];
      for (int iy = 0; iy < kPmeOrder; ++iy) {
        int gy = sp.base[1] + iy;
        if (gy >= Ky) gy -= Ky;
        const float wxy = wx * sp.th[1][iy];
        unsigned long long* row = p.grid + (static_cast<long long>(gx) * Ky + gy) * Kz;
        for (int iz = 0; iz < kPmeOrder; ++iz) {
          int gz = sp.base[2] + iz;
          if (gz >= Kz) gz -= Kz;
          add_fixed(&row[gz], wxy * sp.th[2][iz]);
        }
      }
    }
  }
}

__global__ void k_na_z_forward(SysDev S, NaPtrs p, int lines_per_block) {
  extern __shared__ float2 smem[];
  const int Kx = S.grid[0], Ky = S.grid[1], Kz = S.grid[2], kzh = S.kzh;
  const int line0 = blockIdx.x * lines_per_block;
  const int nl = min(lines_per_block, Kx * Ky - line0);
  if (nl <= 0) return;
  float2* A = smem;
  float2* B = smem + nl * Kz;
  unsigned long long* grid = p.grid + static_cast<long long>(line0) * Kz;
  for (int i = threadIdx.x; i < nl * Kz; i += blockDim.x) {
    A[i] = make_float2(from_fixed(static_cast<long long>(grid[i])), 0.f);
    grid[i] = 0ull;
  }
  __syncthreads();
  const float2* R = fft_lines(A, B, Kz, nl, S.radices[2], S.nradix[2], p.twiddles + 2 * kNoAllocMaxAxis, -1);
  float2* out = p.spectrum + static_cast<long long>(line0) * kzh;
  for (int i = threadIdx.x; i < nl * kzh; i += blockDim.x) {
    const int line = i / kzh, k = i - line * kzh;
    out[i] = R[line * Kz + k];
  }
}

__global__ void k_na_y(SysDev S, NaPtrs p, int sign) {
  extern __shared__ float2 smem[];
  const int Ky = S.grid[1], kzh = S.kzh;
  const int tiles = (kzh + 15) / 16;
  const int x = blockIdx.x / tiles, kz0 = (blockIdx.x % tiles) * 16;
  const int nk = min(16, kzh - kz0);
  float2* A = smem;
  float2* B = smem + nk * Ky;
  float2* base = p.spectrum + static_cast<long long>(x) * Ky * kzh + kz0;
  for (int i = threadIdx.x; i < nk * Ky; i += blockDim.x) {
    const int y = i / nk, l = i - y * nk;
    A[l * Ky + y] = base[static_cast<long long>(y) * kzh + l];
  }
  __syncthreads();
  const float2* R = fft_lines(A, B, Ky, nk, S.radices[1], S.nradix[1], p.twiddles + kNoAllocMaxAxis, sign);
  for (int i = threadIdx.x; i < nk * Ky; i += blockDim.x) {
    const int y = i / nk, l = i - y * nk;
    base[static_cast<long long>(y) * kzh + l] = R[l * Ky + y];
  }
}

__global__ void k_na_x_convolve(SysDev S, NaPtrs p) {
  extern __shared__ float2 smem[];
  __shared__ double partial[kThreads / 32];
  const int Kx = S.grid[0], Ky = S.grid[1], Kz = S.grid[2], kzh = S.kzh;
  const int tiles = (kzh + 15) / 16;
  const int my = blockIdx.x / tiles, kz0 = (blockIdx.x % tiles) * 16;
  const int nk = min(16, kzh - kz0);
  float2* A = smem;
  float2* B = smem + nk * Kx;
  const long long stride = static_cast<long long>(Ky) * kzh;
  float2* base = p.spectrum + static_cast<long long>(my) * kzh + kz0;
  for (int i = threadIdx.x; i < nk * Kx; i += blockDim.x) {
    const int x = i / nk, l = i - x * nk;
    A[l * Kx + x] = base[x * stride + l];
  }
  __syncthreads();
  float2* R = fft_lines(A, B, Kx, nk, S.radices[0], S.nradix[0], p.twiddles, -1);
  float2* other = R == A ? B : A;
  const int mb = my <= Ky / 2 ? my : my - Ky;
  const float* modx = p.moduli;
  const float* mody = p.moduli + kNoAllocMaxAxis;
  const float* modz = p.moduli + 2 * kNoAllocMaxAxis;
  double energy = 0.0;
  for (int i = threadIdx.x; i < nk * Kx; i += blockDim.x) {
    const int l = i / Kx, mx = i - l * Kx;
    const int kz = kz0 + l;
    float2 v = R[i];
    float kx, ky, kzv, k2;
    const float factor = influence(S, modx, mody, modz, Kx, mx, mb, my, kz, kx, ky, kzv, k2);
    const double weight = (kz == 0 || (2 * kz == Kz)) ? 1.0 : 2.0;
    energy += weight * double(factor) * (double(v.x) * v.x + double(v.y) * v.y);
    v.x *= 2.f * factor;
    v.y *= 2.f * factor;
    R[i] = v;
  }
  __syncthreads();
  const float2* Q = fft_lines(R, other, Kx, nk, S.radices[0], S.nradix[0], p.twiddles, +1);
  for (int i = threadIdx.x; i < nk * Kx; i += blockDim.x) {
    const int x = i / nk, l = i - x * nk;
    base[x * stride + l] = Q[l * Kx + x];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) energy += __shfl_xor_sync(0xffffffffu, energy, o);
  if ((threadIdx.x & 31) == 0) partial[threadIdx.x >> 5] = energy;
  __syncthreads();
  if (threadIdx.x == 0) {
    double total = 0.0;
    for (int k = 0; k < (blockDim.x >> 5); ++k) total += partial[k];
    p.partials[blockIdx.x] = total;
  }
}

__global__ void k_na_z_inverse(SysDev S, NaPtrs p, int lines_per_block) {
  extern __shared__ float2 smem[];
  const int Kx = S.grid[0], Ky = S.grid[1], Kz = S.grid[2], kzh = S.kzh;
  const int line0 = blockIdx.x * lines_per_block;
  const int nl = min(lines_per_block, Kx * Ky - line0);
  if (nl <= 0) return;
  float2* A = smem;
  float2* B = smem + nl * Kz;
  const float2* in = p.spectrum + static_cast<long long>(line0) * kzh;
  for (int i = threadIdx.x; i < nl * kzh; i += blockDim.x) {
    const int line = i / kzh, k = i - line * kzh;
    A[line * Kz + k] = in[i];
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nl * (Kz - kzh); i += blockDim.x) {
    const int line = i / (Kz - kzh), k = kzh + (i - line * (Kz - kzh));
    const float2 c = A[line * Kz + (Kz - k)];
    A[line * Kz + k] = make_float2(c.x, -c.y);
  }
  __syncthreads();
  const float2* R = fft_lines(A, B, Kz, nl, S.radices[2], S.nradix[2], p.twiddles + 2 * kNoAllocMaxAxis, +1);
  float* out = p.potential + static_cast<long long>(line0) * Kz;
  for (int i = threadIdx.x; i < nl * Kz; i += blockDim.x) out[i] = R[i].x;
}

__global__ void k_na_gather(SysDev S, NaPtrs p, int n, const double* pos, const double* charge, double* forces) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float q = float(charge[i]);
    if (q == 0.f) {
      forces[3 * i] = forces[3 * i + 1] = forces[3 * i + 2] = 0.0;
      continue;
    }
    Spline sp;
    spline_for(S, fixed_from_double(pos[3 * i]), fixed_from_double(pos[3 * i + 1]),
               fixed_from_double(pos[3 * i + 2]), sp, true);
    const int Kx = S.grid[0], Ky = S.grid[1], Kz = S.grid[2];
    float ga = 0.f, gb = 0.f, gc = 0.f;
    for (int ix = 0; ix < kPmeOrder; ++ix) {
      int gx = sp.base[0] + ix;
      if (gx >= Kx) gx -= Kx;
      for (int iy = 0; iy < kPmeOrder; ++iy) {
        int gy = sp.base[1] + iy;
        if (gy >= Ky) gy -= Ky;
        const float* row = p.potential + (static_cast<long long>(gx) * Ky + gy) * Kz;
        const float wxy = sp.th[0][ix] * sp.th[1][iy];
        const float dxy = sp.dth[0][ix] * sp.th[1][iy];
        const float xdy = sp.th[0][ix] * sp.dth[1][iy];
        for (int iz = 0; iz < kPmeOrder; ++iz) {
          int gz = sp.base[2] + iz;
          if (gz >= Kz) gz -= Kz;
          const float v = row[gz];
          ga = fmaf(v * dxy, sp.th[2][iz], ga);
          gb = fmaf(v * xdy, sp.th[2][iz], gb);
          gc = fmaf(v * wxy, sp.dth[2][iz], gc);
        }
      }
    }
    const float* U = S.umat_f;
    forces[3 * i] = -q * (ga * U[0] + gb * U[1] + gc * U[2]);
    forces[3 * i + 1] = -q * (ga * U[3] + gb * U[4] + gc * U[5]);
    forces[3 * i + 2] = -q * (ga * U[6] + gb * U[7] + gc * U[8]);
  }
}

__global__ void k_na_energy(NaPtrs p, int count, double* energy) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double total = 0.0;
    for (int k = 0; k < count; ++k) total += p.partials[k];
    *energy = total;
  }
}

// The scratch array's device address, looked up with the device current.  In
// host code `g_noalloc_scratch` names a host-side stand-in, never device
// memory, so kernels must be given this address instead.  A call on a stream
// that is not capturing looks the address up again (cheap), so a device reset,
// which reloads the module at a new address, is picked up by the next such
// call; a call inside a stream capture uses the address the last call outside
// one found, and fails if there is none yet.
std::mutex g_noalloc_mutex;
std::array<unsigned char*, 64> g_noalloc_address{};

int noalloc_scratch(int device, bool capturing, unsigned char** out) {
  if (device < 0 || device >= int(g_noalloc_address.size())) return MDB_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!capturing) {
    void* ptr = nullptr;
    if (cudaGetSymbolAddress(&ptr, g_noalloc_scratch) != cudaSuccess || ptr == nullptr) return MDB_ERR_DEVICE;
    g_noalloc_address[device] = static_cast<unsigned char*>(ptr);
  }
  if (!g_noalloc_address[device]) return MDB_ERR_INVALID_ARGUMENT;
  *out = g_noalloc_address[device];
  return MDB_OK;
}

}  // namespace
}  // namespace mdb

extern "C" int mdb_reciprocal_noalloc(int32_t n, const double* positions, const double* charges,
                                      const double box[9], double alpha, const int32_t mesh[3], double* forces,
                                      double* energy, void* stream) {
  using namespace mdb;
  if (n < 0 || !box || !mesh || !energy || !(alpha > 0) || (n > 0 && (!positions || !charges || !forces)))
    return MDB_ERR_INVALID_ARGUMENT;
  long long points = 1;
  for (int k = 0; k < 3; ++k) {
    // an order-5 spline spans 5 mesh points, wrapped once into the mesh
    if (mesh[k] < kPmeOrder) return MDB_ERR_INVALID_ARGUMENT;
    if (mesh[k] > kNoAllocMaxAxis) return MDB_ERR_CAPACITY;
    points *= mesh[k];
  }
  if (points > kNoAllocMaxMeshPoints) return MDB_ERR_CAPACITY;
  SysDev S;
  std::memset(&S, 0, sizeof(S));
  for (int k = 0; k < 3; ++k) {
    S.grid[k] = mesh[k];
    if (!plan_radices(mesh[k], S.radices[k], &S.nradix[k])) return MDB_ERR_NOT_SMOOTH;
  }
  S.kzh = mesh[2] / 2 + 1;
  double B[9], M[9];
  if (!reduce_box(box, B)) return MDB_ERR_INVALID_ARGUMENT;
  inverse_box(B, M);
  for (int i = 0; i < 9; ++i) S.inv_f[i] = float(M[i]);
  const double um[6] = {mesh[0] * M[0], mesh[0] * M[3], mesh[0] * M[6], mesh[1] * M[4], mesh[1] * M[7], mesh[2] * M[8]};
  for (int i = 0; i < 6; ++i) S.umat[i] = std::llround(um[i] * 4294967296.0);
  for (int v = 0; v < 3; ++v)
    for (int u = 0; u < 3; ++u) S.umat_f[v * 3 + u] = float(mesh[u] * M[v * 3 + u]);
  S.pme_pref = float(kOne4PiEps0 * 2 * 3.14159265358979323846 / box_volume(B));
  S.exp_scale = float(-1.0 / (4 * alpha * alpha));

  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess) return MDB_ERR_NO_DEVICE;
  // An error left by the caller's earlier work is theirs: report it without
  // consuming it, so that only this call's own launches set what
  // cudaGetLastError returns below.
  if (cudaPeekAtLastError() != cudaSuccess) return MDB_ERR_DEVICE;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &capture) != cudaSuccess) return MDB_ERR_DEVICE;
  unsigned char* base = nullptr;
  const int status = noalloc_scratch(device, capture != cudaStreamCaptureStatusNone, &base);
  if (status != MDB_OK) return status;
  NaPtrs p;
  p.grid = reinterpret_cast<unsigned long long*>(base + kNaGrid);
  p.spectrum = reinterpret_cast<float2*>(base + kNaSpectrum);
  p.potential = reinterpret_cast<float*>(base + kNaPotential);
  p.moduli = reinterpret_cast<float*>(base + kNaModuli);
  p.twiddles = reinterpret_cast<float2*>(base + kNaTwiddles);
  p.partials = reinterpret_cast<double*>(base + kNaPartials);

  const int lines = std::max(1, 2048 / mesh[2]);
  const int z_blocks = int((mesh[0] * mesh[1] + lines - 1) / lines);
  const int tiles = (S.kzh + 15) / 16;
  const int z_smem = 2 * lines * mesh[2] * int(sizeof(float2));
  const int y_smem = 2 * 16 * mesh[1] * int(sizeof(float2));
  const int x_smem = 2 * 16 * mesh[0] * int(sizeof(float2));
  const int atom_blocks = std::max(1, std::min((n + kThreads - 1) / kThreads, 148 * 8));
  k_na_setup<<<std::max(1, int(std::min<long long>((points + kThreads - 1) / kThreads, 148 * 8))), kThreads, 0, st>>>(S, p);
  if (n > 0) k_na_spread<<<atom_blocks, kThreads, 0, st>>>(S, p, n, positions, charges);
  k_na_z_forward<<<z_blocks, kThreads, z_smem, st>>>(S, p, lines);
  k_na_y<<<mesh[0] * tiles, kThreads, y_smem, st>>>(S, p, -1);
  k_na_x_convolve<<<mesh[1] * tiles, kThreads, x_smem, st>>>(S, p);
  k_na_y<<<mesh[0] * tiles, kThreads, y_smem, st>>>(S, p, +1);
  k_na_z_inverse<<<z_blocks, kThreads, z_smem, st>>>(S, p, lines);
  if (n > 0) k_na_gather<<<atom_blocks, kThreads, 0, st>>>(S, p, n, positions, charges, forces);
  k_na_energy<<<1, 32, 0, st>>>(p, mesh[1] * tiles, energy);
  return cudaGetLastError() == cudaSuccess ? MDB_OK : MDB_ERR_DEVICE;
}
