// k_nonbonded.cu -- real-space Ewald + Lennard-Jones over the tile list.
//
// The physics is the reference's pair term (src/gpu/kernels/nonbonded-pairs.wgsl
// `accumulate_pair`, :193; oracle src/reference/forces/nonbonded.ts:279):
//   E  = qq erfc(a r)/r + 4 eps ((s/r)^12 - (s/r)^6),  s = (si+sj)/2, eps = sqrt(ei ej)
// evaluated in f32 on the exact fixed-point pair vector, excluded pairs
// skipped (the exceptions kernel takes their reciprocal part back out).
//
// The B200 shape is different: one warp owns one 32x32 tile of the list.  Lane
// l keeps atom i of block I in registers and holds atom j of block J; after
// every pair the j data and the j-force accumulator rotate one lane down with
// `__shfl_sync`, so each pair is evaluated exactly once (Newton's third law,
// half the arithmetic of the reference's gather) and no shared memory or
// atomics are needed inside the tile.  Per tile the f32 partial sums become
// int64 fixed point: the j side with one atomic per component, the i side in
// registers across the consecutive tiles of its row.  Integer addition makes
// the totals independent of the order tiles finish in, so repeat runs are
// bit-identical.
#include "device_state.h"

namespace mdb {
namespace {

constexpr int kThreads = 256;
constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ long long warp_sum64(long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

template <bool TRICLINIC>
__device__ __forceinline__ void min_image(const SysDev& S, int& dx, int& dy, int& dz) {
  if (!TRICLINIC) {
    if (dx > S.pc_half[0]) dx -= S.pc_box[0];
    if (dx < -S.pc_half[0]) dx += S.pc_box[0];
    if (dy > S.pc_half[1]) dy -= S.pc_box[4];
    if (dy < -S.pc_half[1]) dy += S.pc_box[4];
    if (dz > S.pc_half[2]) dz -= S.pc_box[8];
    if (dz < -S.pc_half[2]) dz += S.pc_box[8];
  } else {
    // Sequential reduction against c, b, a (nonbonded.ts:241), the count
    // estimated in f32 and applied in integers.
    const int kc = __float2int_rn(dz * S.pc_inv_diag[2]);
    dz -= kc * S.pc_box[8];
    dy -= kc * S.pc_box[7];
    dx -= kc * S.pc_box[6];
    const int kb = __float2int_rn(dy * S.pc_inv_diag[1]);
    dy -= kb * S.pc_box[4];
    dx -= kb * S.pc_box[3];
    const int ka = __float2int_rn(dx * S.pc_inv_diag[0]);
    dx -= ka * S.pc_box[0];
  }
}

// erfc(x) = exp(-x^2) P(u): P fits erfcx on x in [0, 3.6] as a degree-7
// polynomial in u = 3.111 t - 2.111, t = 1/(1 + x/2) (fit_erfcx.py in this
// directory derives the coefficients).  The kernel then needs one exponential
// per pair, shared with the Gaussian term of the force.
__device__ __forceinline__ float erfcx_poly(float x) {
  const float t = __fdividef(1.0f, fmaf(0.5f, x, 1.0f));
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

template <bool ENERGY, bool TRICLINIC>
__device__ __forceinline__ void tile_pairs(const SysDev& S, int4 pi, float4 qi, int4 pj, float4 qj,
                                           unsigned int mask, int lane, float& fix, float& fiy,
                                           float& fiz, float& fjx, float& fjy, float& fjz,
                                           float& ecoul, float& elj, int& pairs, float* vir) {
  const float alpha = S.alpha, a2sp = S.alpha_2_sqrtpi, cut2 = S.cut2, inv = S.pc_inv;
#pragma unroll 4
  for (int k = 0; k < 32; ++k) {
    const int jl = (lane + k) & 31;
    int dx = pj.x - pi.x, dy = pj.y - pi.y, dz = pj.z - pi.z;
    min_image<TRICLINIC>(S, dx, dy, dz);
    const float rx = dx * inv, ry = dy * inv, rz = dz * inv;
    const float r2 = rx * rx + ry * ry + rz * rz;
    if (((mask >> jl) & 1u) && r2 < cut2) {
      const float rinv = rsqrtf(r2);
      const float rinv2 = rinv * rinv;
      const float r = r2 * rinv;
      const float qq = qi.x * qj.x;
      const float x = alpha * r;
      const float gauss = __expf(-x * x);
      const float screened = gauss * erfcx_poly(x);
      const float coul = qq * screened * rinv;
      const float eps = qi.z * qj.z;
      const float sig = qi.y + qj.y;
      const float s2 = sig * sig * rinv2;
      const float s6 = s2 * s2 * s2;
      const float s12 = s6 * s6;
      // (dE/dr)/r
      const float fs = rinv2 * (-coul - qq * a2sp * gauss + eps * (24.0f * s6 - 48.0f * s12));
      fix = fmaf(fs, rx, fix);
      fiy = fmaf(fs, ry, fiy);
      fiz = fmaf(fs, rz, fiz);
      fjx = fmaf(-fs, rx, fjx);
      fjy = fmaf(-fs, ry, fjy);
      fjz = fmaf(-fs, rz, fjz);
      if (ENERGY) {
        ecoul += coul;
        elj += 4.0f * eps * (s12 - s6);
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
    const int src = (lane + 1) & 31;
    pj.x = __shfl_sync(kFull, pj.x, src);
    pj.y = __shfl_sync(kFull, pj.y, src);
    pj.z = __shfl_sync(kFull, pj.z, src);
    qj.x = __shfl_sync(kFull, qj.x, src);
    qj.y = __shfl_sync(kFull, qj.y, src);
    qj.z = __shfl_sync(kFull, qj.z, src);
    fjx = __shfl_sync(kFull, fjx, src);
    fjy = __shfl_sync(kFull, fjy, src);
    fjz = __shfl_sync(kFull, fjz, src);
  }
}

template <bool ENERGY>
__global__ void __launch_bounds__(kThreads) k_nonbonded(Dev d) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const int total = d.tile_prefix[d.S];
  const int per = (total + nwarps - 1) / nwarps;
  int t = warp * per;
  const int tend = min(total, t + per);
  if (t >= tend) return;
  int s = find_system(d.tile_prefix, d.S, t);

  long long aix = 0, aiy = 0, aiz = 0;
  int cur_row = -1;
  long long ecoul64 = 0, elj64 = 0, pairs64 = 0;
  long long vir64[6] = {0, 0, 0, 0, 0, 0};

  auto flush_row = [&]() {
    if (cur_row >= 0) {
      const int gi = cur_row * 32 + lane;
      if (aix | aiy | aiz) {
        add_fixed64(&d.fx[gi], aix);
        add_fixed64(&d.fy[gi], aiy);
        add_fixed64(&d.fz[gi], aiz);
      }
    }
    aix = aiy = aiz = 0;
  };
  auto base_of = [&](int sys) { return d.sys[sys].energy_base; };
  auto flush_energy = [&](int sys) {
    if (ENERGY) {
      const long long c = warp_sum64(ecoul64), l = warp_sum64(elj64), p = warp_sum64(pairs64);
      if (lane == 0) {
        const int base = d.sys[sys].energy_base;
        add_fixed64(&d.energy[base + kECoulomb], c);
        add_fixed64(&d.energy[base + kELj], l);
        add_fixed64(&d.energy[base + kEPairs], p);
      }
      // slots: row-major 3x3, the symmetric pair tensor written to both halves
      const int slot[6] = {0, 4, 8, 1, 2, 5}, mirror[6] = {-1, -1, -1, 3, 6, 7};
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        const long long v = warp_sum64(vir64[k]);
        if (lane == 0) {
          add_fixed64(&d.energy[base_of(sys) + kEVirial0 + slot[k]], v);
          if (mirror[k] >= 0) add_fixed64(&d.energy[base_of(sys) + kEVirial0 + mirror[k]], v);
        }
        vir64[k] = 0;
      }
      ecoul64 = elj64 = pairs64 = 0;
    }
  };

  for (; t < tend; ++t) {
    while (t >= d.tile_prefix[s + 1]) {
      flush_energy(s);
      ++s;
    }
    const SysDev& S = d.sys[s];
    const long long ti = S.tile_off + (t - d.tile_prefix[s]);
    const int2 tile = d.tiles[ti];
    if (tile.x != cur_row) {
      flush_row();
      cur_row = tile.x;
    }
    const int gi = tile.x * 32 + lane, gj = tile.y * 32 + lane;
    const int4 pi = d.pc[gi];
    const float4 qi = d.prm[gi];
    const int4 pj = d.pc[gj];
    const float4 qj = d.prm[gj];
    const unsigned int mask = d.masks[ti * 32 + lane];
    float fix = 0.f, fiy = 0.f, fiz = 0.f, fjx = 0.f, fjy = 0.f, fjz = 0.f, ec = 0.f, el = 0.f;
    float vir[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    int np = 0;
    if (S.triclinic)
      tile_pairs<ENERGY, true>(S, pi, qi, pj, qj, mask, lane, fix, fiy, fiz, fjx, fjy, fjz, ec, el, np, vir);
    else
      tile_pairs<ENERGY, false>(S, pi, qi, pj, qj, mask, lane, fix, fiy, fiz, fjx, fjy, fjz, ec, el, np, vir);
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

}  // namespace

void launch_nonbonded(const Dev& d, bool energy, cudaStream_t st) {
  // Persistent-style: a fixed grid of 148 SMs x 8 blocks of 8 warps, each warp
  // taking a contiguous run of tiles so consecutive tiles of a row share i.
  const int blocks = 148 * 8;
  if (energy) k_nonbonded<true><<<blocks, kThreads, 0, st>>>(d);
  else k_nonbonded<false><<<blocks, kThreads, 0, st>>>(d);
}

}  // namespace mdb
