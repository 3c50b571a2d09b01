// k_integrate.cu -- one fused launch for the whole integrator step.
//
// The reference splits LFMiddle into kick -> RATTLE/SETTLE-v -> drift ->
// SHAKE/SETTLE -> finish, one dispatch each, because its constraint solvers
// are separate passes (src/gpu/kernels/integrate.wgsl:140-203, settle.wgsl,
// shake.wgsl; oracle src/reference/integrator.ts:140-220).  Constraints never
// couple two clusters, so here one thread owns one *integration unit* -- a
// SETTLE water, a SHAKE cluster (<= 8 atoms, <= 8 constraints), or a free atom
// -- and carries it through every phase in registers:
//
//   COM removal (com-motion.ts:48, on removesOnStep)
//   kick          v += dt F / m
//   SETTLE-v / RATTLE
//   drift         x' = x + v dt/2 (+ residual); v = e^{-g dt} v + noise; x' += v dt/2
//   SETTLE / SHAKE (Jacobi, reference bond vectors, FP64 convergence test)
//   finish        v += (x'' - x')/dt; x = x''
//
// and then the things the next step needs: the displacement test that asks for
// a neighbour-list rebuild (verlet.wgsl:57), the momentum for the next COM
// removal (a fixed-order FP64 reduction, so it is deterministic), the step
// counter, and the rebuild decision, all by the last block to finish.
// Positions are int64 fixed point with residual feedback (integrate.wgsl:40),
// velocities f32, thermostat noise Threefry-2x32-20 (random.wgsl:78).
#include "device_state.h"

namespace mdb {
namespace {

// 128 threads for 32 units a block; 64 / 16 and 256 / 32-or-64 measured no faster
constexpr int kThreads = 128;

struct Atom {
  long long x, y, z;  // start-of-step position (reference for the constraints)
  float vx, vy, vz;
  float im;
  float rx, ry, rz;
  float fx, fy, fz;
};

__device__ __forceinline__ float3 rel(const Atom& a, const Atom& o) {
  return make_float3(from_fixed(a.x - o.x), from_fixed(a.y - o.y), from_fixed(a.z - o.z));
}

// src/reference/settle.ts:198 -- exact 3x3 impulse solve for the velocities.
__device__ __forceinline__ void settle_velocities(Atom* at) {
  const float mA = at[0].im > 0 ? 1.f / at[0].im : 0.f, mB = at[1].im > 0 ? 1.f / at[1].im : 0.f,
              mC = at[2].im > 0 ? 1.f / at[2].im : 0.f;
  const float3 pB = rel(at[1], at[0]), pC = rel(at[2], at[0]);
  auto unit = [](float3 v) {
    const float inv = rsqrtf(v.x * v.x + v.y * v.y + v.z * v.z);
    return make_float3(v.x * inv, v.y * inv, v.z * inv);
  };
  const float3 eAB = unit(pB);
  const float3 eBC = unit(make_float3(pC.x - pB.x, pC.y - pB.y, pC.z - pB.z));
  const float3 eCA = unit(make_float3(-pC.x, -pC.y, -pC.z));
  auto relv = [&](int from, int to, float3 e) {
    return (at[to].vx - at[from].vx) * e.x + (at[to].vy - at[from].vy) * e.y + (at[to].vz - at[from].vz) * e.z;
  };
  const float vAB = relv(0, 1, eAB), vBC = relv(1, 2, eBC), vCA = relv(2, 0, eCA);
  auto dot = [](float3 p, float3 q) { return p.x * q.x + p.y * q.y + p.z * q.z; };
  const float cA = -dot(eAB, eCA), cB = -dot(eAB, eBC), cC = -dot(eBC, eCA);
  const float s2A = 1.f - cA * cA, s2B = 1.f - cB * cB, s2C = 1.f - cC * cC;
  const float mi = 1.f / (mA * mB * mC);
  const float den = (((s2A * mB + s2B * mA) * mC + (s2A * mB * mB + 2.f * (cA * cB * cC + 1.f) * mA * mB + s2B * mA * mA)) * mC +
                     s2C * mA * mB * (mA + mB)) * mi;
  const float tab = ((cB * cC * mA - cA * mB - cA * mC) * vCA + (cA * cC * mB - cB * mC - cB * mA) * vBC +
                     (s2C * mA * mA * mB * mB * mi + (mA + mB + mC)) * vAB) / den;
  const float tbc = ((cA * cB * mC - cC * mB - cC * mA) * vCA + (s2A * mB * mB * mC * mC * mi + (mA + mB + mC)) * vBC +
                     (cA * cC * mB - cB * mA - cB * mC) * vAB) / den;
  const float tca = ((s2B * mA * mA * mC * mC * mi + (mA + mB + mC)) * vCA + (cA * cB * mC - cC * mB - cC * mA) * vBC +
                     (cB * cC * mA - cA * mB - cA * mC) * vAB) / den;
  at[0].vx += (eAB.x * tab - eCA.x * tca) * at[0].im;
  at[0].vy += (eAB.y * tab - eCA.y * tca) * at[0].im;
  at[0].vz += (eAB.z * tab - eCA.z * tca) * at[0].im;
  at[1].vx += (eBC.x * tbc - eAB.x * tab) * at[1].im;
  at[1].vy += (eBC.y * tbc - eAB.y * tab) * at[1].im;
  at[1].vz += (eBC.z * tbc - eAB.z * tab) * at[1].im;
  at[2].vx += (eCA.x * tca - eBC.x * tbc) * at[2].im;
  at[2].vy += (eCA.y * tca - eBC.y * tbc) * at[2].im;
  at[2].vz += (eCA.z * tca - eBC.z * tbc) * at[2].im;
}

// src/reference/settle.ts:31 -- Miyamoto & Kollman in the reference frame.
// `dp` holds each atom's trial displacement from its start position on input
// and its constrained displacement on output.
__device__ __forceinline__ void settle_positions(const Atom* at, float3* dp, float d1, float d2) {
  const float m0 = 1.f / at[0].im, m1 = 1.f / at[1].im, m2 = 1.f / at[2].im;
  const float3 b0 = rel(at[1], at[0]), c0 = rel(at[2], at[0]);
  const float xb0 = b0.x, yb0 = b0.y, zb0 = b0.z, xc0 = c0.x, yc0 = c0.y, zc0 = c0.z;
  const float itm = 1.f / (m0 + m1 + m2);
  const float xcom = (dp[0].x * m0 + (xb0 + dp[1].x) * m1 + (xc0 + dp[2].x) * m2) * itm;
  const float ycom = (dp[0].y * m0 + (yb0 + dp[1].y) * m1 + (yc0 + dp[2].y) * m2) * itm;
  const float zcom = (dp[0].z * m0 + (zb0 + dp[1].z) * m1 + (zc0 + dp[2].z) * m2) * itm;
  const float xa1 = dp[0].x - xcom, ya1 = dp[0].y - ycom, za1 = dp[0].z - zcom;
  const float xb1 = xb0 + dp[1].x - xcom, yb1 = yb0 + dp[1].y - ycom, zb1 = zb0 + dp[1].z - zcom;
  const float xc1 = xc0 + dp[2].x - xcom, yc1 = yc0 + dp[2].y - ycom, zc1 = zc0 + dp[2].z - zcom;
  const float xZ = yb0 * zc0 - zb0 * yc0, yZ = zb0 * xc0 - xb0 * zc0, zZ = xb0 * yc0 - yb0 * xc0;
  const float xX = ya1 * zZ - za1 * yZ, yX = za1 * xZ - xa1 * zZ, zX = xa1 * yZ - ya1 * xZ;
  const float xY = yZ * zX - zZ * yX, yY = zZ * xX - xZ * zX, zY = xZ * yX - yZ * xX;
  const float ilx = rsqrtf(xX * xX + yX * yX + zX * zX);
  const float ily = rsqrtf(xY * xY + yY * yY + zY * zY);
  const float ilz = rsqrtf(xZ * xZ + yZ * yZ + zZ * zZ);
  const float t11 = xX * ilx, t21 = yX * ilx, t31 = zX * ilx;
  const float t12 = xY * ily, t22 = yY * ily, t32 = zY * ily;
  const float t13 = xZ * ilz, t23 = yZ * ilz, t33 = zZ * ilz;
  const float xb0d = t11 * xb0 + t21 * yb0 + t31 * zb0, yb0d = t12 * xb0 + t22 * yb0 + t32 * zb0;
  const float xc0d = t11 * xc0 + t21 * yc0 + t31 * zc0, yc0d = t12 * xc0 + t22 * yc0 + t32 * zc0;
  const float za1d = t13 * xa1 + t23 * ya1 + t33 * za1;
  const float xb1d = t11 * xb1 + t21 * yb1 + t31 * zb1, yb1d = t12 * xb1 + t22 * yb1 + t32 * zb1;
  const float zb1d = t13 * xb1 + t23 * yb1 + t33 * zb1;
  const float xc1d = t11 * xc1 + t21 * yc1 + t31 * zc1, yc1d = t12 * xc1 + t22 * yc1 + t32 * zc1;
  const float zc1d = t13 * xc1 + t23 * yc1 + t33 * zc1;
  const float rc = 0.5f * d2;
  float rb = sqrtf(d1 * d1 - rc * rc);
  const float ra = rb * (m1 + m2) * itm;
  rb -= ra;
  const float sinphi = za1d / ra, cosphi = sqrtf(fmaxf(0.f, 1.f - sinphi * sinphi));
  const float sinpsi = (zb1d - zc1d) / (2.f * rc * cosphi), cospsi = sqrtf(fmaxf(0.f, 1.f - sinpsi * sinpsi));
  const float ya2d = ra * cosphi;
  float xb2d = -rc * cospsi;
  const float yb2d = -rb * cosphi - rc * sinpsi * sinphi, yc2d = -rb * cosphi + rc * sinpsi * sinphi;
  const float xb2d2 = xb2d * xb2d;
  const float hh2 = 4.f * xb2d2 + (yb2d - yc2d) * (yb2d - yc2d) + (zb1d - zc1d) * (zb1d - zc1d);
  const float deltx = 2.f * xb2d + sqrtf(fmaxf(0.f, 4.f * xb2d2 - hh2 + d2 * d2));
  xb2d -= deltx * 0.5f;
  const float al = xb2d * (xb0d - xc0d) + yb0d * yb2d + yc0d * yc2d;
  const float be = xb2d * (yc0d - yb0d) + xb0d * yb2d + xc0d * yc2d;
  const float ga = xb0d * yb1d - xb1d * yb0d + xc0d * yc1d - xc1d * yc0d;
  const float a2b2 = al * al + be * be;
  const float sinth = (al * ga - be * sqrtf(fmaxf(0.f, a2b2 - ga * ga))) / a2b2;
  const float costh = sqrtf(fmaxf(0.f, 1.f - sinth * sinth));
  const float xa3d = -ya2d * sinth, ya3d = ya2d * costh, za3d = za1d;
  const float xb3d = xb2d * costh - yb2d * sinth, yb3d = xb2d * sinth + yb2d * costh, zb3d = zb1d;
  const float xc3d = -xb2d * costh - yc2d * sinth, yc3d = -xb2d * sinth + yc2d * costh, zc3d = zc1d;
  dp[0] = make_float3(xcom + t11 * xa3d + t12 * ya3d + t13 * za3d, ycom + t21 * xa3d + t22 * ya3d + t23 * za3d,
                      zcom + t31 * xa3d + t32 * ya3d + t33 * za3d);
  dp[1] = make_float3(xcom + t11 * xb3d + t12 * yb3d + t13 * zb3d - xb0, ycom + t21 * xb3d + t22 * yb3d + t23 * zb3d - yb0,
                      zcom + t31 * xb3d + t32 * yb3d + t33 * zb3d - zb0);
  dp[2] = make_float3(xcom + t11 * xc3d + t12 * yc3d + t13 * zc3d - xc0, ycom + t21 * xc3d + t22 * yc3d + t23 * zc3d - yc0,
                      zcom + t31 * xc3d + t32 * yc3d + t33 * zc3d - zc0);
}

// src/reference/constraints.ts:195 -- RATTLE, Jacobi, over one cluster.  The
// solve runs in FP64: its absolute 1e-6 convergence test sits at the rounding
// noise of an f32 velocity difference along a bond, where an f32 iteration
// stalls short of the tolerance and runs to the 150-iteration cap.
__device__ __noinline__ bool rattle(Atom* at, const UnitDev& u, float tol) {
  double rv[kMaxClusterConstraints][3];
  double rl[kMaxClusterConstraints], rm[kMaxClusterConstraints], delta[kMaxClusterConstraints];
  double v[kMaxClusterAtoms][3];
  for (int k = 0; k < u.na; ++k) {
    v[k][0] = at[k].vx; v[k][1] = at[k].vy; v[k][2] = at[k].vz;
  }
  for (int c = 0; c < u.nc; ++c) {
    const float3 r = rel(at[u.ci[c]], at[u.cj[c]]);
    rv[c][0] = r.x; rv[c][1] = r.y; rv[c][2] = r.z;
    rl[c] = rv[c][0] * rv[c][0] + rv[c][1] * rv[c][1] + rv[c][2] * rv[c][2];
    const double sum = double(at[u.ci[c]].im) + at[u.cj[c]].im;
    rm[c] = sum == 0.0 ? 0.0 : 0.5 / sum;
  }
  bool ok = false;
  for (int it = 0; it < kMaxShakeIterations; ++it) {
    int conv = 0;
    for (int c = 0; c < u.nc; ++c) {
      const int i = u.ci[c], j = u.cj[c];
      const double proj = (v[i][0] - v[j][0]) * rv[c][0] + (v[i][1] - v[j][1]) * rv[c][1] + (v[i][2] - v[j][2]) * rv[c][2];
      delta[c] = rl[c] == 0.0 ? 0.0 : (-2.0 * rm[c] * proj) / rl[c];
      conv += fabs(delta[c]) <= tol;
    }
    if (conv == u.nc) { ok = true; break; }
    for (int c = 0; c < u.nc; ++c) {
      const int i = u.ci[c], j = u.cj[c];
      const double ii = at[i].im, jj = at[j].im;
      for (int x = 0; x < 3; ++x) {
        const double dr = rv[c][x] * delta[c];
        v[i][x] += dr * ii;
        v[j][x] -= dr * jj;
      }
    }
  }
  for (int k = 0; k < u.na; ++k) {
    at[k].vx = float(v[k][0]); at[k].vy = float(v[k][1]); at[k].vz = float(v[k][2]);
  }
  return ok;
}

// src/reference/constraints.ts:130 -- SHAKE, Jacobi along the reference bond
// vectors, over one cluster, in FP64 (convergence window and updates).  The
// trial bond vector is the exact reference vector plus the difference of the
// two displacements.
__device__ __noinline__ bool shake(const Atom* at, float3* dp, const UnitDev& u, float tol) {
  double rv[kMaxClusterConstraints][3];
  double rm[kMaxClusterConstraints], delta[kMaxClusterConstraints];
  double q[kMaxClusterAtoms][3];
  for (int k = 0; k < u.na; ++k) {
    q[k][0] = dp[k].x; q[k][1] = dp[k].y; q[k][2] = dp[k].z;
  }
  for (int c = 0; c < u.nc; ++c) {
    const float3 r = rel(at[u.ci[c]], at[u.cj[c]]);
    rv[c][0] = r.x; rv[c][1] = r.y; rv[c][2] = r.z;
    const double sum = double(at[u.ci[c]].im) + at[u.cj[c]].im;
    rm[c] = sum == 0.0 ? 0.0 : 0.5 / sum;
  }
  const double lo = 1.0 - 2.0 * tol + double(tol) * tol, hi = 1.0 + 2.0 * tol + double(tol) * tol;
  bool ok = false;
  for (int it = 0; it < kMaxShakeIterations; ++it) {
    int conv = 0;
    for (int c = 0; c < u.nc; ++c) {
      const int i = u.ci[c], j = u.cj[c];
      const double x = rv[c][0] + q[i][0] - q[j][0], y = rv[c][1] + q[i][1] - q[j][1], z = rv[c][2] + q[i][2] - q[j][2];
      const double l2 = x * x + y * y + z * z;
      const double d2 = double(u.dist[c]) * u.dist[c];
      const double proj = x * rv[c][0] + y * rv[c][1] + z * rv[c][2];
      delta[c] = proj == 0.0 ? 0.0 : rm[c] * (d2 - l2) / proj;
      conv += (l2 >= lo * d2 && l2 <= hi * d2);
    }
    if (conv == u.nc) { ok = true; break; }
    for (int c = 0; c < u.nc; ++c) {
      const int i = u.ci[c], j = u.cj[c];
      const double ii = at[i].im, jj = at[j].im;
      for (int x = 0; x < 3; ++x) {
        const double dr = rv[c][x] * delta[c];
        q[i][x] += dr * ii;
        q[j][x] -= dr * jj;
      }
    }
  }
  for (int k = 0; k < u.na; ++k) dp[k] = make_float3(float(q[k][0]), float(q[k][1]), float(q[k][2]));
  return ok;
}

__device__ __forceinline__ long long displace(float wanted, float& left_over) {
  const long long taken = to_fixed(wanted);
  left_over = wanted - from_fixed(taken);
  return taken;
}

// ------------------------------------------------------- star clusters ----
// Most SHAKE clusters are an X-H_n star (every constraint joins the centre,
// atom 0, to one spoke, atom c + 1): C-H, CH2, CH3, N-H, NH3+.  Written for
// that shape with the constraint count known at compile time, the FP64 solves
// stay in registers; the general `rattle`/`shake` above index their arrays at
// run time and spill to local memory.  Same Jacobi iterations, same order.
template <int NC>
__device__ bool rattle_star(const long long* x, const long long* y, const long long* z, float* vx, float* vy,
                            float* vz, const float* im, float tol) {
  constexpr int NA = NC + 1;
  double v[NA][3];
#pragma unroll
  for (int k = 0; k < NA; ++k) {
    v[k][0] = vx[k]; v[k][1] = vy[k]; v[k][2] = vz[k];
  }
  // the reference bond vectors are f32 values (from_fixed) and the inverse
  // masses f32: kept as f32 and widened where used, to save registers
  float rv[NC][3];
  double rl[NC], rm[NC], delta[NC];
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    rv[c][0] = from_fixed(x[0] - x[c + 1]);
    rv[c][1] = from_fixed(y[0] - y[c + 1]);
    rv[c][2] = from_fixed(z[0] - z[c + 1]);
    rl[c] = double(rv[c][0]) * rv[c][0] + double(rv[c][1]) * rv[c][1] + double(rv[c][2]) * rv[c][2];
    const double sum = double(im[0]) + double(im[c + 1]);
    rm[c] = sum == 0.0 ? 0.0 : 0.5 / sum;
  }
  bool ok = false;
  for (int it = 0; it < kMaxShakeIterations; ++it) {
    int conv = 0;
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      const double proj = (v[0][0] - v[c + 1][0]) * rv[c][0] + (v[0][1] - v[c + 1][1]) * rv[c][1] +
                          (v[0][2] - v[c + 1][2]) * rv[c][2];
      delta[c] = rl[c] == 0.0 ? 0.0 : (-2.0 * rm[c] * proj) / rl[c];
      conv += fabs(delta[c]) <= tol;
    }
    if (conv == NC) { ok = true; break; }
#pragma unroll
    for (int c = 0; c < NC; ++c)
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const double dr = rv[c][k] * delta[c];
        v[0][k] += dr * double(im[0]);
        v[c + 1][k] -= dr * double(im[c + 1]);
      }
  }
#pragma unroll
  for (int k = 0; k < NA; ++k) {
    vx[k] = float(v[k][0]); vy[k] = float(v[k][1]); vz[k] = float(v[k][2]);
  }
  return ok;
}

// `dp` holds the trial displacements on input and the constrained ones on output.
template <int NC>
__device__ bool shake_star(const long long* x, const long long* y, const long long* z, const float* im,
                           const float* dist, float3* dp, float tol) {
  constexpr int NA = NC + 1;
  double q[NA][3];
#pragma unroll
  for (int k = 0; k < NA; ++k) {
    q[k][0] = dp[k].x; q[k][1] = dp[k].y; q[k][2] = dp[k].z;
  }
  float rv[NC][3];  // f32 values (from_fixed), widened where used
  double rm[NC], delta[NC];
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    rv[c][0] = from_fixed(x[0] - x[c + 1]);
    rv[c][1] = from_fixed(y[0] - y[c + 1]);
    rv[c][2] = from_fixed(z[0] - z[c + 1]);
    const double sum = double(im[0]) + double(im[c + 1]);
    rm[c] = sum == 0.0 ? 0.0 : 0.5 / sum;
  }
  const double lo = 1.0 - 2.0 * tol + double(tol) * tol, hi = 1.0 + 2.0 * tol + double(tol) * tol;
  bool ok = false;
  for (int it = 0; it < kMaxShakeIterations; ++it) {
    int conv = 0;
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      const double d2 = double(dist[c]) * dist[c];
      const double ex = rv[c][0] + q[0][0] - q[c + 1][0], ey = rv[c][1] + q[0][1] - q[c + 1][1],
                   ez = rv[c][2] + q[0][2] - q[c + 1][2];
      const double l2 = ex * ex + ey * ey + ez * ez;
      const double proj = ex * rv[c][0] + ey * rv[c][1] + ez * rv[c][2];
      delta[c] = proj == 0.0 ? 0.0 : rm[c] * (d2 - l2) / proj;
      conv += (l2 >= lo * d2 && l2 <= hi * d2);
    }
    if (conv == NC) { ok = true; break; }
#pragma unroll
    for (int c = 0; c < NC; ++c)
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const double dr = rv[c][k] * delta[c];
        q[0][k] += dr * double(im[0]);
        q[c + 1][k] -= dr * double(im[c + 1]);
      }
  }
#pragma unroll
  for (int k = 0; k < NA; ++k) dp[k] = make_float3(float(q[k][0]), float(q[k][1]), float(q[k][2]));
  return ok;
}

__device__ void block_sum3(double* v, double (*red)[kThreads / 32]) {
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
  if ((threadIdx.x & 31) == 0)
    for (int k = 0; k < 3; ++k) red[k][threadIdx.x >> 5] = v[k];
  __syncthreads();
  if (threadIdx.x == 0)
    for (int k = 0; k < 3; ++k) {
      double t = 0;
      for (int w = 0; w < kThreads / 32; ++w) t += red[k][w];
      v[k] = t;
    }
}

// The last block of a system turns the block momenta into the next step's
// COM velocity (a fixed-order block reduction, so runs stay bit-identical) and
// advances the step; the last block of the launch snapshots the rebuild
// requests for the next step's list kernels.
__device__ void finish_block(const Dev& d, int s, const SysDev& S, bool advance, double (*red)[kThreads / 32]) {
  __shared__ int last_of_system, last_of_launch;
  __threadfence();
  if (threadIdx.x == 0) last_of_system = atomicAdd(&d.done_count[s], 1) == S.n_iblk - 1;
  __syncthreads();
  if (last_of_system) {
    __threadfence();
    double p[3] = {0, 0, 0};
    for (int i = threadIdx.x; i < S.n_iblk; i += kThreads)
      for (int k = 0; k < 3; ++k) p[k] += __ldcg(&d.mom_partial[(S.iblk_off + i) * 3 + k]);
    block_sum3(p, red);
    if (threadIdx.x == 0) {
      const double m = S.total_mass > 0 ? S.total_mass : 1.0;
      d.vcom[s] = make_float4(float(p[0] / m), float(p[1] / m), float(p[2] / m), 0.f);
      if (advance) d.step[s] += 1;
      d.done_count[s] = 0;
    }
  }
  if (!advance) return;
  __threadfence();
  if (threadIdx.x == 0) last_of_launch = atomicAdd(d.global_ticket, 1) == int(gridDim.x) - 1;
  __syncthreads();
  if (last_of_launch && threadIdx.x == 0) {
    __threadfence();
    int any = 0, any_prune = 0;
    for (int k = 0; k < d.S; ++k) {
      const int f = __ldcg(&d.rebuild_flag[k]) | d.run.always_rebuild;
      d.rebuild_now[k] = f;
      d.rebuild_flag[k] = 0;
      any |= f;
      if (d.inner) {
        const int p = __ldcg(&d.prune_flag[k]);
        d.prune_now[k] = p;
        d.prune_flag[k] = 0;
        any_prune |= p;
      }
    }
    *d.any_rebuild = any;
    if (d.inner) *d.any_prune = any_prune;
    *d.global_ticket = 0;
  }
}

// One integrate block: up to kIntegrateUnits units and their atoms, staged in
// shared memory between phases that alternate between one thread per atom
// (loads, kick, noise, drift, finish: the bulk of the arithmetic and every
// global access) and one thread per unit (the constraint solves).
struct Stage {
  long long x[kIntegrateTable], y[kIntegrateTable], z[kIntegrateTable];     // start-of-step positions
  long long tx[kIntegrateTable], ty[kIntegrateTable], tz[kIntegrateTable];  // unconstrained drift
  long long cx[kIntegrateTable], cy[kIntegrateTable], cz[kIntegrateTable];  // constrained drift
  float vx[kIntegrateTable], vy[kIntegrateTable], vz[kIntegrateTable], im[kIntegrateTable];
  float rx[kIntegrateTable], ry[kIntegrateTable], rz[kIntegrateTable];     // drift residuals
};

constexpr int kPerThread = kIntegrateTable / kThreads;

__device__ __forceinline__ Atom staged_atom(const Stage& sh, int e) {
  Atom A;
  A.x = sh.x[e]; A.y = sh.y[e]; A.z = sh.z[e];
  A.vx = sh.vx[e]; A.vy = sh.vy[e]; A.vz = sh.vz[e];
  A.im = sh.im[e];
  return A;
}

__device__ __noinline__ void cluster_velocities(Stage& sh, const UnitDev& u, float tol, bool& bad) {
  const int e = u.base;
  Atom at[kMaxClusterAtoms];
  for (int k = 0; k < u.na; ++k) at[k] = staged_atom(sh, e + k);
  bad |= !rattle(at, u, tol);
  for (int k = 0; k < u.na; ++k) { sh.vx[e + k] = at[k].vx; sh.vy[e + k] = at[k].vy; sh.vz[e + k] = at[k].vz; }
}

// Velocity constraints of one unit (LFMiddle, after the kick).
__device__ void unit_velocities(Stage& sh, const UnitDev& u, float tol, bool& bad) {
  const int e = u.base;
  if (u.kind == kUnitSettle) {
    Atom at[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) at[k] = staged_atom(sh, e + k);
    settle_velocities(at);
#pragma unroll
    for (int k = 0; k < 3; ++k) { sh.vx[e + k] = at[k].vx; sh.vy[e + k] = at[k].vy; sh.vz[e + k] = at[k].vz; }
  } else if (u.kind == kUnitStar) {
    switch (u.nc) {
      case 1: bad |= !rattle_star<1>(sh.x + e, sh.y + e, sh.z + e, sh.vx + e, sh.vy + e, sh.vz + e, sh.im + e, tol); break;
      case 2: bad |= !rattle_star<2>(sh.x + e, sh.y + e, sh.z + e, sh.vx + e, sh.vy + e, sh.vz + e, sh.im + e, tol); break;
      default: bad |= !rattle_star<3>(sh.x + e, sh.y + e, sh.z + e, sh.vx + e, sh.vy + e, sh.vz + e, sh.im + e, tol); break;
    }
  } else if (u.kind == kUnitShake) {
    cluster_velocities(sh, u, tol, bad);
  }
}

__device__ __forceinline__ void store_constrained(Stage& sh, int e, float3 dp) {
  if (sh.im[e] == 0.f) {
    sh.cx[e] = sh.tx[e]; sh.cy[e] = sh.ty[e]; sh.cz[e] = sh.tz[e];
  } else {
    sh.cx[e] = to_fixed(dp.x); sh.cy[e] = to_fixed(dp.y); sh.cz[e] = to_fixed(dp.z);
  }
}

__device__ __forceinline__ float3 staged_drift(const Stage& sh, int e) {
  return make_float3(from_fixed(sh.tx[e]), from_fixed(sh.ty[e]), from_fixed(sh.tz[e]));
}

template <int NC>
__device__ __forceinline__ void star_positions(Stage& sh, const UnitDev& u, float tol, bool& bad) {
  const int e = u.base;
  float3 dp[NC + 1];
#pragma unroll
  for (int k = 0; k <= NC; ++k) dp[k] = staged_drift(sh, e + k);
  bad |= !shake_star<NC>(sh.x + e, sh.y + e, sh.z + e, sh.im + e, u.dist, dp, tol);
#pragma unroll
  for (int k = 0; k <= NC; ++k) store_constrained(sh, e + k, dp[k]);
}

__device__ __noinline__ void cluster_positions(Stage& sh, const UnitDev& u, float tol, bool& bad) {
  const int e = u.base;
  Atom at[kMaxClusterAtoms];
  float3 dp[kMaxClusterAtoms];
  for (int k = 0; k < u.na; ++k) {
    at[k] = staged_atom(sh, e + k);
    dp[k] = staged_drift(sh, e + k);
  }
  bad |= !shake(at, dp, u, tol);
  for (int k = 0; k < u.na; ++k) store_constrained(sh, e + k, dp[k]);
}

// Position constraints of one unit: cx = constrained drift (the unconstrained
// drift for free and massless atoms).
__device__ void unit_positions(Stage& sh, const UnitDev& u, float tol, bool& bad) {
  const int e = u.base;
  if (u.kind == kUnitFree) {
    sh.cx[e] = sh.tx[e]; sh.cy[e] = sh.ty[e]; sh.cz[e] = sh.tz[e];
  } else if (u.kind == kUnitSettle) {
    Atom at[3];
    float3 dp[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      at[k] = staged_atom(sh, e + k);
      dp[k] = staged_drift(sh, e + k);
    }
    settle_positions(at, dp, u.dist[0], u.dist[1]);
#pragma unroll
    for (int k = 0; k < 3; ++k) store_constrained(sh, e + k, dp[k]);
  } else if (u.kind == kUnitStar) {
    switch (u.nc) {
      case 1: star_positions<1>(sh, u, tol, bad); break;
      case 2: star_positions<2>(sh, u, tol, bad); break;
      default: star_positions<3>(sh, u, tol, bad); break;
    }
  } else {
    cluster_positions(sh, u, tol, bad);
  }
}

__global__ void __launch_bounds__(kThreads) k_integrate(Dev d) {
  __shared__ Stage sh;
  __shared__ double red[3][kThreads / 32];
  wait_for_predecessor();
  const int b = blockIdx.x;
  const int s = d.iblk_sys[b];
  const SysDev& S = d.sys[s];
  if (*d.halt) {
    // a list overflowed this step (every block sees the same word): the
    // forces came from a cut list, so nothing advances; only the force
    // slots are cleared for the next step, which the host runs after it has
    // grown and rebuilt the list
    for (int e = threadIdx.x; e < d.iblk_natom[b]; e += kThreads) {
      const int gs = S.slot_off + d.rank[d.iatom[d.iblk_atom0[b] + e]];
      d.fx[gs] = 0ull; d.fy[gs] = 0ull; d.fz[gs] = 0ull;
    }
    return;
  }
  const RunDev& R = d.run;
  const long long step = d.step[s];
  const bool com = S.com_freq > 0 && (step % S.com_freq) == 0;
  const float4 vc = com ? d.vcom[s] : make_float4(0.f, 0.f, 0.f, 0.f);
  const int natom = d.iblk_natom[b], atom0 = d.iblk_atom0[b], nunit = d.iblk_nunit[b];
  const UnitDev* units = d.units + d.iblk_unit0[b];
  const float dt = R.dt;
  const bool lfm = R.integrator == 0;

  // Every phase keeps its per-atom state in the shared table, not in
  // registers across the barriers, so the kernel needs few registers and
  // many blocks fit on an SM; an atom phase reads its atom's index again.

  // ---- atoms: load, clear the force slot, COM removal, kick
#pragma unroll
  for (int j = 0; j < kPerThread; ++j) {
    const int e = threadIdx.x + j * kThreads;
    if (e >= natom) continue;
    const int a = d.iatom[atom0 + e];
    float vx = d.vx[a], vy = d.vy[a], vz = d.vz[a];
    const float im = d.invm[a];
    const int gs = S.slot_off + d.rank[a];
    const float fx = from_fixed(static_cast<long long>(d.fx[gs]));
    const float fy = from_fixed(static_cast<long long>(d.fy[gs]));
    const float fz = from_fixed(static_cast<long long>(d.fz[gs]));
    d.fx[gs] = 0ull; d.fy[gs] = 0ull; d.fz[gs] = 0ull;  // consumer clears
    if (com && im > 0.f) { vx -= vc.x; vy -= vc.y; vz -= vc.z; }
    if (im != 0.f) {
      if (lfm) {
        vx += dt * im * fx; vy += dt * im * fy; vz += dt * im * fz;
      } else {
        vx += im * fx * dt; vy += im * fy * dt; vz += im * fz * dt;
      }
    }
    sh.x[e] = d.px[a]; sh.y[e] = d.py[a]; sh.z[e] = d.pz[a];
    sh.vx[e] = vx; sh.vy[e] = vy; sh.vz[e] = vz;
    sh.rx[e] = d.rx[a]; sh.ry[e] = d.ry[a]; sh.rz[e] = d.rz[a];
    sh.im[e] = im;
  }
  __syncthreads();

  // ---- units: SETTLE-v / RATTLE (LFMiddle)
  bool bad = false;
  if (lfm && threadIdx.x < nunit) unit_velocities(sh, units[threadIdx.x], R.tolerance, bad);
  __syncthreads();

  // ---- atoms: drift (fixed point, residual feedback) with the thermostat
  // between the halves; the thermostatted velocity and the new residual go
  // back to the table (the position constraints read neither)
  const float half = 0.5f * dt;
#pragma unroll
  for (int j = 0; j < kPerThread; ++j) {
    const int e = threadIdx.x + j * kThreads;
    if (e >= natom) continue;
    const float im = sh.im[e];
    long long tx = 0, ty = 0, tz = 0;
    if (im != 0.f) {
      float vx = sh.vx[e], vy = sh.vy[e], vz = sh.vz[e];
      float rx = sh.rx[e], ry = sh.ry[e], rz = sh.rz[e];
      if (lfm) {
        float n0 = 0.f, n1 = 0.f, n2 = 0.f;
        if (R.draw_noise) {
          const unsigned p = static_cast<unsigned>(d.iatom[atom0 + e] - S.atom_off);
          const uint2 key = make_uint2(R.seed, kThermostatDomain);
          const float2 g0 = normal_pair(make_uint2(p * 2u, static_cast<unsigned>(step)), key);
          const float2 g1 = normal_pair(make_uint2(p * 2u + 1u, static_cast<unsigned>(step)), key);
          n0 = g0.x; n1 = g0.y; n2 = g1.x;
        }
        const float noise = R.noise_scale * sqrtf(R.kt * im);
        float lo;
        tx = displace(vx * half + rx, lo);
        vx = R.velocity_scale * vx + noise * n0;
        tx += displace(vx * half + lo, rx);
        ty = displace(vy * half + ry, lo);
        vy = R.velocity_scale * vy + noise * n1;
        ty += displace(vy * half + lo, ry);
        tz = displace(vz * half + rz, lo);
        vz = R.velocity_scale * vz + noise * n2;
        tz += displace(vz * half + lo, rz);
      } else {
        tx = displace(vx * dt + rx, rx);
        ty = displace(vy * dt + ry, ry);
        tz = displace(vz * dt + rz, rz);
      }
      sh.vx[e] = vx; sh.vy[e] = vy; sh.vz[e] = vz;
      sh.rx[e] = rx; sh.ry[e] = ry; sh.rz[e] = rz;
    }
    sh.tx[e] = tx; sh.ty[e] = ty; sh.tz[e] = tz;
  }
  __syncthreads();

  // ---- units: SETTLE / SHAKE on the drifted positions
  if (threadIdx.x < nunit) unit_positions(sh, units[threadIdx.x], R.tolerance, bad);
  __syncthreads();

  // ---- atoms: velocity correction, store, rebuild test, momentum
  const float idt = 1.f / dt;
  double mom[3] = {0, 0, 0};
  bool moved = false, strayed = false;
#pragma unroll
  for (int j = 0; j < kPerThread; ++j) {
    const int e = threadIdx.x + j * kThreads;
    if (e >= natom) continue;
    const int a = d.iatom[atom0 + e];
    const float im = sh.im[e];
    const long long cx = sh.cx[e], cy = sh.cy[e], cz = sh.cz[e];
    long long px = sh.x[e], py = sh.y[e], pz = sh.z[e];
    float vx = sh.vx[e], vy = sh.vy[e], vz = sh.vz[e];
    if (im != 0.f) {
      if (lfm) {
        vx += idt * from_fixed(cx - sh.tx[e]);
        vy += idt * from_fixed(cy - sh.ty[e]);
        vz += idt * from_fixed(cz - sh.tz[e]);
      } else {
        vx = idt * from_fixed(cx);
        vy = idt * from_fixed(cy);
        vz = idt * from_fixed(cz);
      }
      px += cx; py += cy; pz += cz;
      d.px[a] = px; d.py[a] = py; d.pz[a] = pz;
      d.vx[a] = vx; d.vy[a] = vy; d.vz[a] = vz;
      d.rx[a] = sh.rx[e]; d.ry[a] = sh.ry[e]; d.rz[a] = sh.rz[e];
      const double m = 1.0 / im;
      mom[0] += m * vx; mom[1] += m * vy; mom[2] += m * vz;
      bad |= !isfinite(vx + vy + vz);
    } else if (com) {
      d.vx[a] = vx; d.vy[a] = vy; d.vz[a] = vz;
    }
    {
      // the next step's pair coordinates under this list's fold, so the list
      // kernel need not wrap again unless a rebuild or a prune is due
      const int gs = S.slot_off + d.rank[a];
      long long na, nb, nc;
      unpack_fold(d.fold[gs], na, nb, nc);
      d.pc[gs] = pair_coordinate(S, px, py, pz, na, nb, nc);
      if (d.spread_sorted) d.spread_atom[gs] = a;  // the next step's spread reads this, not the order a rebuild rewrites
    }
    const float ex = from_fixed(px - d.refx[a]), ey = from_fixed(py - d.refy[a]),
                ez = from_fixed(pz - d.refz[a]);
    moved |= ex * ex + ey * ey + ez * ez > S.half_skin2;
    if (d.inner) {
      const float qx = from_fixed(px - d.prx[a]), qy = from_fixed(py - d.pry[a]),
                  qz = from_fixed(pz - d.prz[a]);
      strayed |= qx * qx + qy * qy + qz * qz > S.half_inner2;
    }
  }
  if (moved) atomicOr(&d.rebuild_flag[s], 1);
  if (strayed) atomicOr(&d.prune_flag[s], 1);
  if (bad) atomicAdd(&d.shake_failures[s], 1);
  block_sum3(mom, red);
  if (threadIdx.x == 0)
    for (int k = 0; k < 3; ++k) d.mom_partial[b * 3 + k] = mom[k];
  finish_block(d, s, S, true, red);
}

// The momentum of the current velocities, for the first COM removal after the
// host set them.
__global__ void __launch_bounds__(kThreads) k_momentum(Dev d) {
  __shared__ double red[3][kThreads / 32];
  const int b = blockIdx.x;
  const int s = d.iblk_sys[b];
  const SysDev& S = d.sys[s];
  double mom[3] = {0, 0, 0};
  for (int e = threadIdx.x; e < d.iblk_natom[b]; e += kThreads) {
    const int a = d.iatom[d.iblk_atom0[b] + e];
    const float im = d.invm[a];
    if (im == 0.f) continue;
    const double m = 1.0 / im;
    mom[0] += m * d.vx[a]; mom[1] += m * d.vy[a]; mom[2] += m * d.vz[a];
  }
  block_sum3(mom, red);
  if (threadIdx.x == 0)
    for (int k = 0; k < 3; ++k) d.mom_partial[b * 3 + k] = mom[k];
  finish_block(d, s, S, false, red);
}

}  // namespace

void launch_integrate(const Dev& d, cudaStream_t st) {
  launch_chained(k_integrate, d.n_iblk, kThreads, 0, st, d);
}

void launch_momentum(const Dev& d, cudaStream_t st) {
  k_momentum<<<d.n_iblk, kThreads, 0, st>>>(d);
}

}  // namespace mdb
