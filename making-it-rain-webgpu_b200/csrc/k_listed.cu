// k_listed.cu -- every listed interaction in one launch: harmonic bonds,
// harmonic angles, periodic torsions (src/gpu/kernels/bonded.wgsl:31/51/86;
// oracle src/reference/forces/bonded.ts:39/71/133), the nonbonded exceptions
// (nonbonded-exceptions.wgsl:74; oracle nonbonded.ts:330) and position
// restraints (restraint.wgsl:81; oracle forces/restraint.ts:38).
//
// One thread per term over the concatenation [bonds | angles | torsions |
// exceptions | restraints] of all systems.  Vectors are differenced exactly in
// 64-bit fixed point and only then converted, so nothing is rounded while it
// is still box-sized (fixed64.wgsl:166-233).  Bonded terms take no minimum
// image, as in OpenMM; exceptions and restraints do.  Forces are scattered as
// int64 fixed-point atomics into the slot-ordered force arrays.
#include "device_state.h"

namespace mdb {
namespace {

constexpr int kThreads = 256;

struct Ctx {
  const Dev& d;
};

__device__ __forceinline__ float3 diff(const Dev& d, int a, int b) {
  return make_float3(from_fixed(d.px[b] - d.px[a]), from_fixed(d.py[b] - d.py[a]),
                     from_fixed(d.pz[b] - d.pz[a]));
}

// Minimum image of an exact fixed-point difference: the box count is estimated
// in f32 and removed in integers, c then b then a (nonbonded.ts:241).
__device__ __forceinline__ float3 min_image_fixed(const SysDev& S, long long dx, long long dy, long long dz) {
  const long long kc = __float2ll_rn(from_fixed(dz) * S.inv_f[8]);
  dz -= kc * S.box_fx[8];
  dy -= kc * S.box_fx[7];
  dx -= kc * S.box_fx[6];
  const long long kb = __float2ll_rn(from_fixed(dy) * S.inv_f[4]);
  dy -= kb * S.box_fx[4];
  dx -= kb * S.box_fx[3];
  const long long ka = __float2ll_rn(from_fixed(dx) * S.inv_f[0]);
  dx -= ka * S.box_fx[0];
  return make_float3(from_fixed(dx), from_fixed(dy), from_fixed(dz));
}

__device__ __forceinline__ void add_force(const Dev& d, const SysDev& S, int atom, float x, float y, float z) {
  const int gs = S.slot_off + d.rank[atom];
  add_fixed(&d.fx[gs], x);
  add_fixed(&d.fy[gs], y);
  add_fixed(&d.fz[gs], z);
}

// Energy launches: a thread's energy and virial words in registers (2^32
// fixed point, every slot up to the virial's last), summed over the warp
// before they reach the system's words in global memory.  A thread per term
// adding straight into the same dozen words serialises on them (100k waters:
// about 1.1 M same-address atomics per evaluation); integer sums make the
// totals the same whatever the grouping.
struct EnergySums {
  long long v[kEPairs];
};

template <bool ENERGY>
__device__ __forceinline__ void add_energy(EnergySums& acc, int slot, float e) {
  if (ENERGY) acc.v[slot] += to_fixed(e);
}

// Virial contribution r (x) F of one atom of a term, r measured from the
// term's first atom (energy evaluations only; a 3x3 row-major tensor).
template <bool ENERGY>
__device__ __forceinline__ void add_virial(EnergySums& acc, float3 r, float fx, float fy, float fz) {
  if (!ENERGY) return;
  const float rr[3] = {r.x, r.y, r.z}, ff[3] = {fx, fy, fz};
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) acc.v[kEVirial0 + 3 * a + b] += to_fixed(rr[a] * ff[b]);
}

// One thread's sums into system s's words, and cleared.
__device__ __forceinline__ void flush_sums(const Dev& d, EnergySums& acc, int s) {
  unsigned long long* e = &d.energy[d.sys[s].energy_base];
#pragma unroll
  for (int k = 0; k < kEPairs; ++k) {
    if (acc.v[k]) add_fixed64(&e[k], acc.v[k]);
    acc.v[k] = 0;
  }
}

// The warp's sums at the end of the kernel (every lane present): one add per
// word when every lane that has sums has them for the same system, else one
// per lane.
__device__ __forceinline__ void flush_warp(const Dev& d, EnergySums& acc, int s) {
  const unsigned full = 0xffffffffu;
  const int lead = __reduce_max_sync(full, s);
  if (lead < 0) return;
  if (__all_sync(full, s == lead || s < 0)) {
    unsigned long long* e = &d.energy[d.sys[lead].energy_base];
#pragma unroll
    for (int k = 0; k < kEPairs; ++k) {
      long long v = acc.v[k];
      if (!__any_sync(full, v != 0)) continue;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(full, v, o);
      if ((threadIdx.x & 31) == 0 && v) add_fixed64(&e[k], v);
    }
  } else if (s >= 0) {
    flush_sums(d, acc, s);
  }
}

// Error-free transformations on f32 (Knuth's TwoSum; the fma product error).
// The _rn intrinsics keep the compiler from contracting them into fma.
__device__ __forceinline__ float two_sum(float a, float b, float& err) {
  const float s = __fadd_rn(a, b), bb = __fsub_rn(s, a);
  err = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
  return s;
}

// The stretch r - r0 of one bond, to about 1e-12 nm where plain f32 gives
// r0 * 2^-24 (~7e-9 nm, or ~3e-3 kJ/mol/nm of force at k = 4.8e5 on a C=O
// bond).  The exact integer separation is split into f32 hi + lo parts,
// r^2 - r0^2 is accumulated with TwoSum and fma product errors, and divided by
// r + r0.  Still f32 arithmetic throughout.
__device__ __forceinline__ float bond_stretch(const Dev& d, const BondDev& t, float3& v, float& r) {
  const long long D[3] = {d.px[t.b] - d.px[t.a], d.py[t.b] - d.py[t.a], d.pz[t.b] - d.pz[t.a]};
  float hi[3], lo[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float h = __ll2float_rn(D[k]);
    hi[k] = h * 2.3283064365386963e-10f;
    lo[k] = __ll2float_rn(D[k] - __float2ll_rn(h)) * 2.3283064365386963e-10f;
  }
  float p[3], tail = 0.f;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    p[k] = __fmul_rn(hi[k], hi[k]);
    tail += fmaf(hi[k], hi[k], -p[k]) + (2.f * hi[k] + lo[k]) * lo[k];
  }
  float e1, e2;
  const float s1 = two_sum(p[0], p[1], e1);
  const float s2 = two_sum(s1, p[2], e2);
  const float delta = __fsub_rn(s2, t.r0sq_hi) + (e1 + e2 + tail - t.r0sq_lo);
  v = make_float3(hi[0] + lo[0], hi[1] + lo[1], hi[2] + lo[2]);
  r = sqrtf(s2);
  return delta / (r + t.r0);
}

template <bool ENERGY>
__device__ void bond(const Dev& d, const BondDev& t, EnergySums& acc) {
  const SysDev& S = d.sys[t.sys];
  float3 v;
  float r;
  const float dr = bond_stretch(d, t, v, r);
  add_energy<ENERGY>(acc, kEBond, 0.5f * t.k * dr * dr);
  const float sc = t.k * dr / r;
  add_force(d, S, t.a, sc * v.x, sc * v.y, sc * v.z);
  add_force(d, S, t.b, -sc * v.x, -sc * v.y, -sc * v.z);
  add_virial<ENERGY>(acc, v, -sc * v.x, -sc * v.y, -sc * v.z);
}

template <bool ENERGY>
__device__ void angle(const Dev& d, const AngleDev& t, EnergySums& acc) {
  const SysDev& S = d.sys[t.sys];
  const float3 v1 = diff(d, t.b, t.a), v2 = diff(d, t.b, t.c);
  const float r1 = v1.x * v1.x + v1.y * v1.y + v1.z * v1.z;
  const float r2 = v2.x * v2.x + v2.y * v2.y + v2.z * v2.z;
  const float dot = v1.x * v2.x + v1.y * v2.y + v1.z * v2.z;
  const float cs = fminf(1.f, fmaxf(-1.f, dot * rsqrtf(r1 * r2)));
  const float nx = v1.y * v2.z - v1.z * v2.y, ny = v1.z * v2.x - v1.x * v2.z, nz = v1.x * v2.y - v1.y * v2.x;
  const float nn = fmaxf(sqrtf(nx * nx + ny * ny + nz * nz), 1e-6f);
  // theta from atan2(|n|, dot) keeps its precision near 0 and pi, where acos does not.
  const float theta = atan2f(sqrtf(nx * nx + ny * ny + nz * nz), dot);
  (void)cs;
  const float dth = theta - t.theta0;
  add_energy<ENERGY>(acc, kEAngle, 0.5f * t.k * dth * dth);
  const float dE = t.k * dth;
  const float tA = dE / (r1 * nn), tC = -dE / (r2 * nn);
  const float f1x = -tA * (v1.y * nz - v1.z * ny), f1y = -tA * (v1.z * nx - v1.x * nz),
              f1z = -tA * (v1.x * ny - v1.y * nx);
  const float f3x = -tC * (v2.y * nz - v2.z * ny), f3y = -tC * (v2.z * nx - v2.x * nz),
              f3z = -tC * (v2.x * ny - v2.y * nx);
  add_force(d, S, t.a, f1x, f1y, f1z);
  add_force(d, S, t.c, f3x, f3y, f3z);
  add_force(d, S, t.b, -f1x - f3x, -f1y - f3y, -f1z - f3z);
  add_virial<ENERGY>(acc, v1, f1x, f1y, f1z);
  add_virial<ENERGY>(acc, v2, f3x, f3y, f3z);
}

template <bool ENERGY>
__device__ void torsion(const Dev& d, const TorsionDev& t, EnergySums& acc) {
  const SysDev& S = d.sys[t.sys];
  const float3 b1 = diff(d, t.a, t.b), b2 = diff(d, t.b, t.c), b3 = diff(d, t.c, t.d);
  const float n1x = b1.y * b2.z - b1.z * b2.y, n1y = b1.z * b2.x - b1.x * b2.z, n1z = b1.x * b2.y - b1.y * b2.x;
  const float n2x = b2.y * b3.z - b2.z * b3.y, n2y = b2.z * b3.x - b2.x * b3.z, n2z = b2.x * b3.y - b2.y * b3.x;
  const float n1 = n1x * n1x + n1y * n1y + n1z * n1z, n2 = n2x * n2x + n2y * n2y + n2z * n2z;
  const float b2n = sqrtf(b2.x * b2.x + b2.y * b2.y + b2.z * b2.z);
  const float X = n1x * n2x + n1y * n2y + n1z * n2z;
  const float Y = b2n * (b1.x * n2x + b1.y * n2y + b1.z * n2z);
  const float phi = atan2f(Y, X);
  const float arg = t.periodicity * phi - t.phase;
  float sn, cn;
  sincosf(arg, &sn, &cn);
  add_energy<ENERGY>(acc, kETorsion, t.k * (1.f + cn));
  if (n1 == 0.f || n2 == 0.f) return;
  const float dEdPhi = -t.k * t.periodicity * sn;
  const float s1 = dEdPhi * b2n / n1, s4 = -dEdPhi * b2n / n2;
  const float f1x = s1 * n1x, f1y = s1 * n1y, f1z = s1 * n1z;
  const float f4x = s4 * n2x, f4y = s4 * n2y, f4z = s4 * n2z;
  const float b2sq = b2n * b2n;
  const float ss = (b1.x * b2.x + b1.y * b2.y + b1.z * b2.z) / b2sq;
  const float tt = (b3.x * b2.x + b3.y * b2.y + b3.z * b2.z) / b2sq;
  add_force(d, S, t.a, f1x, f1y, f1z);
  add_force(d, S, t.b, -(1.f + ss) * f1x + tt * f4x, -(1.f + ss) * f1y + tt * f4y, -(1.f + ss) * f1z + tt * f4z);
  add_force(d, S, t.c, ss * f1x - (1.f + tt) * f4x, ss * f1y - (1.f + tt) * f4y, ss * f1z - (1.f + tt) * f4z);
  add_force(d, S, t.d, f4x, f4y, f4z);
  if (ENERGY) {
    const float3 rc = make_float3(b1.x + b2.x, b1.y + b2.y, b1.z + b2.z);
    const float3 rd = make_float3(rc.x + b3.x, rc.y + b3.y, rc.z + b3.z);
    add_virial<ENERGY>(acc, b1, -(1.f + ss) * f1x + tt * f4x, -(1.f + ss) * f1y + tt * f4y,
                       -(1.f + ss) * f1z + tt * f4z);
    add_virial<ENERGY>(acc, rc, ss * f1x - (1.f + tt) * f4x, ss * f1y - (1.f + tt) * f4y,
                       ss * f1z - (1.f + tt) * f4z);
    add_virial<ENERGY>(acc, rd, f4x, f4y, f4z);
  }
}

template <bool ENERGY>
__device__ void exception(const Dev& d, const ExceptionDev& t, EnergySums& acc) {
  const SysDev& S = d.sys[t.sys];
  const float3 v = min_image_fixed(S, d.px[t.b] - d.px[t.a], d.py[t.b] - d.py[t.a], d.pz[t.b] - d.pz[t.a]);
  const float r2 = v.x * v.x + v.y * v.y + v.z * v.z;
  const float rinv = rsqrtf(r2);
  const float r = r2 * rinv;
  float dEdR = 0.f, correction = 0.f, own = 0.f;
  if (t.qq_particles != 0.f) {
    const float x = S.alpha * r;
    const float ef = erff(x);
    correction = -t.qq_particles * ef * rinv;
    dEdR += t.qq_particles * (ef * rinv * rinv - S.alpha_2_sqrtpi * __expf(-x * x) * rinv);
  }
  if (t.qq_own != 0.f) {
    own += t.qq_own * rinv;
    dEdR -= t.qq_own * rinv * rinv;
  }
  if (t.eps4 != 0.f) {
    const float s2 = t.sigma * t.sigma * rinv * rinv;
    const float s6 = s2 * s2 * s2, s12 = s6 * s6;
    own += t.eps4 * (s12 - s6);
    dEdR += t.eps4 * rinv * (6.f * s6 - 12.f * s12);
  }
  add_energy<ENERGY>(acc, kEExclusion, correction);
  add_energy<ENERGY>(acc, kEException, own);
  if (dEdR != 0.f) {
    const float sc = dEdR * rinv;
    add_force(d, S, t.a, sc * v.x, sc * v.y, sc * v.z);
    add_force(d, S, t.b, -sc * v.x, -sc * v.y, -sc * v.z);
    add_virial<ENERGY>(acc, v, -sc * v.x, -sc * v.y, -sc * v.z);
  }
}

template <bool ENERGY>
__device__ void restraint(const Dev& d, const RestraintDev& t, EnergySums& acc) {
  const SysDev& S = d.sys[t.sys];
  const float3 v = min_image_fixed(S, d.px[t.p] - t.x0, d.py[t.p] - t.y0, d.pz[t.p] - t.z0);
  add_energy<ENERGY>(acc, kERestraint, t.k * (v.x * v.x + v.y * v.y + v.z * v.z));
  add_force(d, S, t.p, -2.f * t.k * v.x, -2.f * t.k * v.y, -2.f * t.k * v.z);
}

template <bool ENERGY>
__global__ void __launch_bounds__(kThreads) k_listed(Dev d) {
  const int n0 = d.n_bonds, n1 = n0 + d.n_angles, n2 = n1 + d.n_torsions, n3 = n2 + d.n_exceptions,
            n4 = n3 + d.n_restraints;
  EnergySums acc;
  int acc_sys = -1;  // the system acc holds sums for
  if (ENERGY) {
#pragma unroll
    for (int k = 0; k < kEPairs; ++k) acc.v[k] = 0;
  }
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += gridDim.x * blockDim.x) {
    const int sys = i < n0   ? d.bonds[i].sys
                    : i < n1 ? d.angles[i - n0].sys
                    : i < n2 ? d.torsions[i - n1].sys
                    : i < n3 ? d.exceptions[i - n2].sys
                             : d.restraints[i - n3].sys;
    if (!sys_active(d, sys)) continue;
    if (ENERGY && sys != acc_sys) {
      if (acc_sys >= 0) flush_sums(d, acc, acc_sys);
      acc_sys = sys;
    }
    if (i < n0) bond<ENERGY>(d, d.bonds[i], acc);
    else if (i < n1) angle<ENERGY>(d, d.angles[i - n0], acc);
    else if (i < n2) torsion<ENERGY>(d, d.torsions[i - n1], acc);
    else if (i < n3) exception<ENERGY>(d, d.exceptions[i - n2], acc);
    else restraint<ENERGY>(d, d.restraints[i - n3], acc);
  }
  if (ENERGY) flush_warp(d, acc, acc_sys);
}

}  // namespace

void launch_listed(const Dev& d, bool energy, cudaStream_t st) {
  const int n = d.n_bonds + d.n_angles + d.n_torsions + d.n_exceptions + d.n_restraints;
  if (n == 0) return;
  int blocks = (n + kThreads - 1) / kThreads;
  if (blocks > 148 * 16) blocks = 148 * 16;
  if (energy) k_listed<true><<<blocks, kThreads, 0, st>>>(d);
  else k_listed<false><<<blocks, kThreads, 0, st>>>(d);
}

}  // namespace mdb
