// k_nonbonded.cu -- real-space Ewald + Lennard-Jones over the tile list.
//
// The physics is the reference's pair term (src/gpu/kernels/nonbonded-pairs.wgsl
// `accumulate_pair`, :193; oracle src/reference/forces/nonbonded.ts:279):
//   E  = qq erfc(a r)/r + 4 eps ((s/r)^12 - (s/r)^6),  s = (si+sj)/2, eps = sqrt(ei ej)
// evaluated in f32 on the exact fixed-point pair vector, excluded pairs
// skipped (the exceptions kernel takes their reciprocal part back out).
//
// The B200 shape is different.  Atoms are sorted into clusters of C (8 or 32)
// consecutive slots along a space-filling curve and the list holds cluster
// pairs (tiles).  A warp runs 32/C tiles at once, one per group of C lanes:
// lane l of a group keeps atom i of cluster I in registers and holds atom j of
// cluster J; after every pair the j data and the j-force accumulator rotate
// one lane down inside the group (`__shfl_sync` of width C), so each pair is
// evaluated exactly once (Newton's third law, half the arithmetic of the
// reference's gather) with no shared memory and no atomics inside a tile.
// Smaller clusters are tighter, so 8x8 tiles cover the cutoff sphere with
// about half the pair slots of 32x32 ones at the price of more j-force
// atomics per slot.  Per tile the f32 partial sums become int64 fixed point:
// the j side with one atomic per component, the i side in registers across
// the consecutive tiles of its row.  Integer addition makes the totals
// independent of the order tiles finish in, so repeat runs are bit-identical.
#include "device_state.h"

namespace mdb {
namespace {

constexpr int kThreads = 256;
constexpr unsigned kFull = 0xffffffffu;
// Tiles per warp (a template argument, TPW): blocks take fixed chunks of the
// list and retire as they finish, so the PME stream's kernels can take SMs
// while the pair kernel runs.  Short lists balance best with short chunks;
// long ones save the per-chunk work (the system lookup, the row and energy
// flushes) with long ones.  Measured: the 12k and 27k single systems (lists of
// 0.14 and 0.30 M tiles) are fastest at 8 (16: octahedron step 0.144 against
// 0.141 ms); the 100k box (2 M tiles) at 16 (pair kernel 0.209 against 0.220
// ms); the 64-system ensemble (9 M tiles) at 64 (pair kernel 1.81 ms; 32:
// 1.83, 16: 1.90, 8: 2.03, 4: 2.18).
constexpr long long kChunk16Tiles = 1ll << 20;  // a typical list at least this long takes chunks of 16
constexpr long long kChunk64Tiles = 1ll << 22;  // and from here chunks of 64

// The three special functions of a pair, as the flush-to-zero forms of the
// PTX approximations.  None of their operands or results can be subnormal
// here: r^2 is at least the square of the closest unexcluded approach (about
// 0.01 nm^2), the reciprocal's operand lies in [1, 1 + alpha cutoff / 2], and
// the exponent of the Gaussian is at least -(alpha cutoff)^2 log2(e) (-10 at
// an Ewald tolerance of 5e-4; below -126 only where erfc(alpha r) is itself
// below 1e-38), so the results are the ones the subnormal-preserving forms
// give, without their range fix-ups.
__device__ __forceinline__ float rsqrt_ftz(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float rcp_ftz(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float exp2_ftz(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// erfc(x) = exp(-x^2) P(u): P fits erfcx on x in [0, 3.6] as a degree-7
// polynomial in u = 3.111 t - 2.111, t = 1/(1 + x/2) (fit_erfcx.py in this
// directory derives the coefficients).  The kernel then needs one exponential
// per pair, shared with the Gaussian term of the force.
__device__ __forceinline__ float erfcx_poly(float x) {
  const float t = rcp_ftz(fmaf(0.5f, x, 1.0f));
  const float u = fmaf(t, 3.1111111111111116f, -2.1111111111111116f);
  float p = 2.8532681218254e-05f;
  p = fmaf(p, u, 7.591772236827632e-05f);
  p = fmaf(p, u, -0.0007059478100949549f);
  p = fmaf(p, u, -0.0015110844839526505f);
  p = fmaf(p, u, 0.01997081313517268f);
  p = fmaf(p, u, 0.1346654154149635f);
  p = fmaf(p, u, 0.40507415765174865f);
  p = fmaf(p, u, 0.4424026315060776f);
  return p;
}

// The pair arithmetic, shared by the force and the energy variants and written
// without contractible expressions (every product and sum is an explicit
// rounding or fused step), so both variants produce the same bits for the
// same pair whatever the compiler does around them.
__device__ __forceinline__ float pair_r2(float rx, float ry, float rz) {
  return fmaf(rz, rz, fmaf(ry, ry, __fmul_rn(rx, rx)));
}

// (dE/dr)/r of one pair at r2 < cutoff^2; with ENERGY also its Coulomb and LJ
// energies.  The Gaussian exp(-(alpha r)^2) is 2^(r^2 gscale), gscale =
// -alpha^2 log2(e): one product from r^2, not from alpha r.  With P = erfcx(x),
// x = alpha r, and g the Gaussian, the Coulomb part of (dE/dr)/r is
// -qq g (P / r + a2sp) / r^2, and the parameters carry sqrt(24 eps), so the
// pair's product is 24 eps and the LJ part is 24 eps (s6 - 2 s12) / r^2.
template <bool ENERGY>
__device__ __forceinline__ float pair_force(float r2, float4 qi, float4 qj, float alpha, float a2sp, float gscale,
                                            float& coul_e, float& lj_e) {
  const float rinv = rsqrt_ftz(r2);
  const float rinv2 = __fmul_rn(rinv, rinv);
  const float x = __fmul_rn(alpha, __fmul_rn(r2, rinv));
  const float gauss = exp2_ftz(__fmul_rn(r2, gscale));
  const float p = erfcx_poly(x);
  const float qg = __fmul_rn(__fmul_rn(qi.x, qj.x), gauss);
  const float eps24 = __fmul_rn(qi.z, qj.z);
  const float sig = __fadd_rn(qi.y, qj.y);
  const float s2 = __fmul_rn(__fmul_rn(sig, sig), rinv2);
  const float s6 = __fmul_rn(__fmul_rn(s2, s2), s2);
  const float s12 = __fmul_rn(s6, s6);
  if (ENERGY) {
    coul_e = __fmul_rn(__fmul_rn(qg, p), rinv);
    // 4 eps (s12 - s6)
    lj_e = __fmul_rn(__fmul_rn(eps24, 1.0f / 6.0f), __fsub_rn(s12, s6));
  }
  const float coul_f = __fmul_rn(qg, fmaf(p, rinv, a2sp));
  return __fmul_rn(rinv2, fmaf(eps24, fmaf(-2.0f, s12, s6), -coul_f));
}

// A system's pair energies, pair count and pair virial (xx yy zz xy xz yz)
// into its energy words; the virial slots are row-major 3x3, the symmetric
// tensor written to both halves.
__device__ __forceinline__ void add_pair_energies(unsigned long long* e, long long c, long long lj, long long p,
                                                  const long long* v) {
  if (c) add_fixed64(&e[kECoulomb], c);
  if (lj) add_fixed64(&e[kELj], lj);
  if (p) add_fixed64(&e[kEPairs], p);
  const int slot[6] = {0, 4, 8, 1, 2, 5}, mirror[6] = {-1, -1, -1, 3, 6, 7};
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    if (!v[k]) continue;
    add_fixed64(&e[kEVirial0 + slot[k]], v[k]);
    if (mirror[k] >= 0) add_fixed64(&e[kEVirial0 + mirror[k]], v[k]);
  }
}

// Lanes of the group that holds `lane`, as a shuffle mask.
template <int C>
__device__ __forceinline__ unsigned group_mask(int lane) {
  return C == 32 ? kFull : (((1u << C) - 1u) << (lane & ~(C - 1)));
}

template <int C>
__device__ __forceinline__ long long group_sum64(long long v, unsigned mask) {
#pragma unroll
  for (int o = C / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o, C);
  return v;
}

// IMAGE: take the minimum image of every pair; otherwise pj already carries
// the tile's lattice shift and the plain difference is the separation.
// `mask` arrives rotated: bit k is the pair of step k (j = l + k mod C).  A
// tile's pairs get the same separations and arithmetic in either image loop,
// whatever its neighbours in the warp, so a tile's result does not depend on
// where in the list it sits.  Measured and not
// kept: evaluating every slot and selecting zeros (no branch) costs 28% more
// on 32x32 tiles, whose warps often have no pair inside at a step; screening
// all slots first and evaluating only the pairs inside, 32 at a time through
// shared memory, gave the same bits but 5-15% more time (7% fewer
// instructions, longer shared-memory dependency chains).
// The system's constants arrive in registers (`SysConst`): read from global
// memory in every tile, they cost the loop a load each.
struct SysConst {
  float alpha, a2sp, gscale, cut2u, inv;  // cut2u: the cutoff squared in pair-coordinate units
  long long tile_base;  // the system's first tile in the list, minus its first tile index
  int next;             // the next system's first tile index
};

__device__ __forceinline__ SysConst sys_const(const Dev& d, int s) {
  const SysDev& S = d.sys[s];
  const int first = d.tile_prefix[s];
  return SysConst{S.alpha, S.alpha_2_sqrtpi, S.gauss_scale, S.cut2u, S.pc_inv, S.tile_off - static_cast<long long>(first),
                  d.tile_prefix[s + 1]};
}

template <int C, bool ENERGY, bool TRICLINIC, bool IMAGE>
__device__ __forceinline__ void tile_pairs(const SysDev& S, const SysConst& K, int4 pi, float4 qi, int4 pj,
                                           float4 qj, unsigned int mask, int l, float& fix,
                                           float& fiy, float& fiz, float& fjx, float& fjy, float& fjz, float& ecoul,
                                           float& elj, int& pairs, float* vir) {
  const float alpha = K.alpha, a2sp = K.a2sp, gscale = K.gscale, inv = K.inv;
  // The separation stays in pair-coordinate units (u = float(d)) until it is
  // needed in nm: inv = 2^-shift is a power of two, so every scaling below is
  // exact and r2 = r2u inv^2, fs rx = (fs inv) ux and r2 < cut2 <=>
  // r2u < cut2 / inv^2 hold bit for bit.
  const float inv2 = __fmul_rn(inv, inv), cut2u = K.cut2u;
  const int src = (l + 1) & (C - 1);
  constexpr int kUnroll = C == 8 ? 8 : 4;
#pragma unroll kUnroll
  for (int k = 0; k < C; ++k) {
    int dx = int(unsigned(pj.x) - unsigned(pi.x)), dy = int(unsigned(pj.y) - unsigned(pi.y)),
        dz = int(unsigned(pj.z) - unsigned(pi.z));
    if (IMAGE) min_image<TRICLINIC>(S, dx, dy, dz);
    const float ux = float(dx), uy = float(dy), uz = float(dz);
    const float r2u = pair_r2(ux, uy, uz);
    if (((mask >> k) & 1u) && r2u < cut2u) {
      float coul = 0.f, lj = 0.f;
      const float r2 = __fmul_rn(r2u, inv2);
      const float fs = pair_force<ENERGY>(r2, qi, qj, alpha, a2sp, gscale, coul, lj);
      const float fsu = __fmul_rn(fs, inv);
      fix = fmaf(fsu, ux, fix);
      fiy = fmaf(fsu, uy, fiy);
      fiz = fmaf(fsu, uz, fiz);
      fjx = fmaf(-fsu, ux, fjx);
      fjy = fmaf(-fsu, uy, fjy);
      fjz = fmaf(-fsu, uz, fjz);
      if (ENERGY) {
        const float rx = __fmul_rn(ux, inv), ry = __fmul_rn(uy, inv), rz = __fmul_rn(uz, inv);
        ecoul += coul;
        elj += lj;
        pairs += 1;
        // virial (r_i - r_j) (x) F_i = -fs r (x) r, symmetric: xx yy zz xy xz yz
        vir[0] -= fs * rx * rx;
        vir[1] -= fs * ry * ry;
        vir[2] -= fs * rz * rz;
        vir[3] -= fs * rx * ry;
        vir[4] -= fs * rx * rz;
        vir[5] -= fs * ry * rz;
      }
    }
    pj.x = __shfl_sync(kFull, pj.x, src, C);
    pj.y = __shfl_sync(kFull, pj.y, src, C);
    pj.z = __shfl_sync(kFull, pj.z, src, C);
    qj.x = __shfl_sync(kFull, qj.x, src, C);
    qj.y = __shfl_sync(kFull, qj.y, src, C);
    qj.z = __shfl_sync(kFull, qj.z, src, C);
    fjx = __shfl_sync(kFull, fjx, src, C);
    fjy = __shfl_sync(kFull, fjy, src, C);
    fjz = __shfl_sync(kFull, fjz, src, C);
  }
}

// A warp takes chunks of TPW consecutive tiles of the list (chunk
// w, then w + warps, ...) and walks each 32/C tiles at a time; group g of the
// warp runs tile t + g.  Every lane keeps its own row and system, because the
// groups of one warp may be at different ones.  The grid is sized for a
// typical list, so most warps take one chunk and then retire.
template <int C, int TPW, bool ENERGY, bool TRICLINIC>
__global__ void __launch_bounds__(kThreads, ENERGY ? 1 : 4) k_nonbonded(Dev d) {
  wait_for_predecessor();  // no early release: later waves would share their SMs with the next kernel
  constexpr int G = 32 / C;
  const int lane = threadIdx.x & 31;
  const int g = lane / C, l = lane & (C - 1);
  const unsigned gmask = group_mask<C>(lane);
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const int total = d.tile_prefix[d.S];
  // Energy launches: the groups' sums for the system of the block's first
  // chunk meet in shared memory and reach the system's energy words once per
  // block.  Every group adding into the same dozen words of global memory
  // serialises on them (a 100k-atom box: some 3 M same-address atomics per
  // evaluation).  The sums are integers, so the totals do not change.
  __shared__ unsigned long long blk_acc[9];  // coulomb, LJ, pairs, virial xx yy zz xy xz yz
  __shared__ int blk_sys;
  if (ENERGY) {
    if (threadIdx.x < 9) blk_acc[threadIdx.x] = 0ull;
    if (threadIdx.x == 0) {
      const int t_first = blockIdx.x * (blockDim.x >> 5) * TPW;
      blk_sys = t_first < total ? find_system(d.tile_prefix, d.S, t_first) : -1;
    }
    __syncthreads();
  }
  for (int t0 = warp * TPW; t0 < total; t0 += nwarps * TPW) {
    const int tend = min(total, t0 + TPW);
    int s = find_system(d.tile_prefix, d.S, min(t0 + g, tend - 1));
    if (ENERGY && d.active) {
      // an evaluation of some systems only (energy evaluations; a step's
      // force launches compute every system): a chunk that lies inside one
      // skipped system is skipped by the whole warp; in a mixed chunk the
      // skipped system's tiles run with an empty mask
      const int first = find_system(d.tile_prefix, d.S, t0), last = find_system(d.tile_prefix, d.S, tend - 1);
      if (first == last && !d.active[first]) continue;
    }

    long long aix = 0, aiy = 0, aiz = 0;
    int cur_row = -1;
    long long ecoul64 = 0, elj64 = 0, pairs64 = 0;
    long long vir64[6] = {0, 0, 0, 0, 0, 0};

    auto flush_row = [&]() {
      if (cur_row >= 0) {
        const int gi = cur_row * C + l;
        if (aix | aiy | aiz) {
          add_fixed64(&d.fx[gi], aix);
          add_fixed64(&d.fy[gi], aiy);
          add_fixed64(&d.fz[gi], aiz);
        }
      }
      aix = aiy = aiz = 0;
    };
    // energies of the group's tiles so far, into system `sys` (every lane of the
    // group calls it together)
    auto flush_energy = [&](int sys) {
      if (ENERGY) {
        const long long c = group_sum64<C>(ecoul64, gmask), lj = group_sum64<C>(elj64, gmask),
                        p = group_sum64<C>(pairs64, gmask);
        long long v[6];
  #pragma unroll
        for (int k = 0; k < 6; ++k) v[k] = group_sum64<C>(vir64[k], gmask);
        if (l == 0 && sys == blk_sys) {
          if (c) atomicAdd(&blk_acc[0], static_cast<unsigned long long>(c));
          if (lj) atomicAdd(&blk_acc[1], static_cast<unsigned long long>(lj));
          if (p) atomicAdd(&blk_acc[2], static_cast<unsigned long long>(p));
  #pragma unroll
          for (int k = 0; k < 6; ++k)
            if (v[k]) atomicAdd(&blk_acc[3 + k], static_cast<unsigned long long>(v[k]));
        } else if (l == 0) {
          add_pair_energies(&d.energy[d.sys[sys].energy_base], c, lj, p, v);
        }
        ecoul64 = elj64 = pairs64 = 0;
  #pragma unroll
        for (int k = 0; k < 6; ++k) vir64[k] = 0;
      }
    };

    SysConst K = sys_const(d, s);
    int4 pi_row = make_int4(0, 0, 0, 0);
    float4 qi_row = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int base = t0; base < tend; base += G) {
      const int t = base + g;
      const bool active = t < tend;  // the same for every lane of a group
      unsigned int mask = 0u;
      int4 pi = make_int4(0, 0, 0, 0), pj = pi;
      float4 qi = make_float4(0.f, 0.f, 0.f, 0.f), qj = qi;
      int gj = -1;
      bool per_pair = false;
      if (active) {
        if (t >= K.next) {
          while (t >= d.tile_prefix[s + 1]) {
            flush_energy(s);
            ++s;
          }
          K = sys_const(d, s);
        }
        const long long ti = K.tile_base + t;
        mask = !ENERGY || sys_active(d, s) ? row_bits<C>(d.masks, ti, l) : 0u;
        const int2 tile = d.tiles[ti];
        if (tile.x != cur_row) {
          flush_row();
          cur_row = tile.x;
          // the row's atom stays in registers across the row's tiles
          pi_row = d.pc[tile.x * C + l];
          qi_row = d.prm[tile.x * C + l];
        }
        gj = tile.y * C + l;
        pi = pi_row;
        qi = qi_row;
        pj = d.pc[gj];
        qj = d.prm[gj];
        const int4 sh = d.tile_shift[ti];
        per_pair = tile_per_pair(sh.w);
        if (!per_pair) {
          pj.x = int(unsigned(pj.x) + unsigned(sh.x));
          pj.y = int(unsigned(pj.y) + unsigned(sh.y));
          pj.z = int(unsigned(pj.z) + unsigned(sh.z));
        }
      }
      float fix = 0.f, fiy = 0.f, fiz = 0.f, fjx = 0.f, fjy = 0.f, fjz = 0.f, ec = 0.f, el = 0.f;
      float vir[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      int np = 0;
      mask = C == 32 ? __funnelshift_r(mask, mask, l) : ((mask >> l) | (mask << ((C - l) & (C - 1)))) & 0xFFu;
      // The minimum image, for every lane of the warp when any of its tiles
      // needs it: one warp-wide decision instead of a divergent branch per
      // slot.  A tile that does not need it holds every pair under its
      // nearest image already, and the reduction leaves such a separation
      // unchanged when it is inside the cutoff and longer than the cutoff
      // when it is not, so both loops give the same pairs and the same bits.
      if (__any_sync(kFull, per_pair))
        tile_pairs<C, ENERGY, TRICLINIC, true>(d.sys[s], K, pi, qi, pj, qj, mask, l, fix, fiy, fiz, fjx, fjy, fjz, ec,
                                               el, np, vir);
      else
        tile_pairs<C, ENERGY, TRICLINIC, false>(d.sys[s], K, pi, qi, pj, qj, mask, l, fix, fiy, fiz, fjx, fjy, fjz,
                                                ec, el, np, vir);
      if (!active) continue;
      aix += to_fixed(fix);
      aiy += to_fixed(fiy);
      aiz += to_fixed(fiz);
      if (fjx != 0.f || fjy != 0.f || fjz != 0.f) {
        add_fixed(&d.fx[gj], fjx);
        add_fixed(&d.fy[gj], fjy);
        add_fixed(&d.fz[gj], fjz);
      }
      if (ENERGY) {
        ecoul64 += to_fixed(ec);
        elj64 += to_fixed(el);
        pairs64 += np;
  #pragma unroll
        for (int k = 0; k < 6; ++k) vir64[k] += to_fixed(vir[k]);
      }
    }
    flush_row();
    flush_energy(s);
  }
  if (ENERGY) {
    __syncthreads();
    if (threadIdx.x == 0 && blk_sys >= 0) {
      long long v[6];
  #pragma unroll
      for (int k = 0; k < 6; ++k) v[k] = static_cast<long long>(blk_acc[3 + k]);
      add_pair_energies(&d.energy[d.sys[blk_sys].energy_base], static_cast<long long>(blk_acc[0]),
                        static_cast<long long>(blk_acc[1]), static_cast<long long>(blk_acc[2]), v);
    }
  }
}

template <int C, int TPW>
void launch_shape(const Dev& d, bool energy, bool triclinic, cudaStream_t st) {
  // one chunk per warp for a list of ~160 tiles per cluster (8x8 tiles in
  // water run 90-150); a longer list makes warps take further chunks
  const int warps_per_block = kThreads / 32;
  const long long typical = static_cast<long long>(d.n_blocks) * (C == 8 ? 160 : 100);
  const int blocks = static_cast<int>(std::max<long long>(
      1, std::min<long long>((typical + TPW * warps_per_block - 1) / (TPW * warps_per_block),
                             (d.tile_cap_total + TPW * warps_per_block - 1) / (TPW * warps_per_block))));
  if (energy) {
    if (triclinic) launch_chained(k_nonbonded<C, TPW, true, true>, blocks, kThreads, 0, st, d);
    else launch_chained(k_nonbonded<C, TPW, true, false>, blocks, kThreads, 0, st, d);
  } else {
    if (triclinic) launch_chained(k_nonbonded<C, TPW, false, true>, blocks, kThreads, 0, st, d);
    else launch_chained(k_nonbonded<C, TPW, false, false>, blocks, kThreads, 0, st, d);
  }
}

template <int C>
void launch_size(const Dev& d, bool energy, bool triclinic, cudaStream_t st) {
  const long long typical = static_cast<long long>(d.n_blocks) * (C == 8 ? 160 : 100);
  if (typical >= kChunk64Tiles) launch_shape<C, 64>(d, energy, triclinic, st);
  else if (typical >= kChunk16Tiles) launch_shape<C, 16>(d, energy, triclinic, st);
  else launch_shape<C, 8>(d, energy, triclinic, st);
}

}  // namespace

void launch_nonbonded(const Dev& d, bool energy, cudaStream_t st) {
  Dev list = d;
  if (d.inner) {  // the inner list has the outer list's layout: per-system regions, offsets by prefix
    list.tiles = d.in_tiles;
    list.masks = d.in_masks;
    list.tile_shift = d.in_shift;
    list.tile_prefix = d.in_prefix;
  }
  if (d.cluster == 8) launch_size<8>(list, energy, d.any_triclinic != 0, st);
  else launch_size<32>(list, energy, d.any_triclinic != 0, st);
}

}  // namespace mdb
