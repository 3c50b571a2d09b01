// oracle.cpp -- TEST INFRASTRUCTURE: the CPU f64 restatement of the
// reference's own f64 oracle (src/reference/** of making-it-rain-webgpu).
//
// This is the checker the B200 engine is measured against, and the timed CPU
// baseline in bench.py.  It is never linked into, loaded by or called from the
// engine.  Every function cites the reference file:line whose algorithm it
// restates; the arithmetic is the same, the code is this project's own.
//
// Parity is pinned against the reference's golden data (see oracle.h).
#include "oracle.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <functional>
#include <numeric>
#include <unordered_set>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

using Vec3 = std::array<double, 3>;
using Box = std::array<double, 9>;

// src/engine/units.ts:15-21
constexpr double kBoltzmann = 0.008314462618153242;
constexpr double kOne4PiEps0 = 138.93545764498457;
constexpr double kPi = 3.14159265358979323846;
constexpr int kPmeOrder = 5;  // src/reference/forces/pme.ts:60

// ---------------------------------------------------------------- erf -----
// src/reference/erf.ts:29-91: erfc(x) = Q(1/2, x^2) by the series below the
// crossover x^2 < 1.5 and by the modified-Lentz continued fraction above it.
constexpr double kLnSqrtPi = 0.5723649429247001;
constexpr int kMaxGammaIterations = 300;

double lower_gamma_series(double a, double x) {
  double term = 1.0 / a, sum = term, ap = a;
  for (int i = 0; i < kMaxGammaIterations; ++i) {
    ap += 1.0;
    term *= x / ap;
    sum += term;
    if (std::fabs(term) < std::fabs(sum) * 2.220446049250313e-16) break;
  }
  return sum * std::exp(-x + a * std::log(x) - kLnSqrtPi);
}

double upper_gamma_fraction(double a, double x) {
  const double tiny = 1e-300;
  double b = x + 1.0 - a, c = 1.0 / tiny, d = 1.0 / b, h = d;
  for (int i = 1; i <= kMaxGammaIterations; ++i) {
    const double an = -i * (i - a);
    b += 2.0;
    d = an * d + b;
    if (std::fabs(d) < tiny) d = tiny;
    c = b + an / c;
    if (std::fabs(c) < tiny) c = tiny;
    d = 1.0 / d;
    const double delta = d * c;
    h *= delta;
    if (std::fabs(delta - 1.0) <= 2.220446049250313e-16) break;
  }
  return std::exp(-x + a * std::log(x) - kLnSqrtPi) * h;
}

double erfc_ref(double x) {
  if (x == 0) return 1.0;
  if (std::isinf(x)) return x > 0 ? 0.0 : 2.0;
  const double m = std::fabs(x), x2 = m * m;
  const double v = x2 < 1.5 ? 1.0 - lower_gamma_series(0.5, x2) : upper_gamma_fraction(0.5, x2);
  return x >= 0 ? v : 2.0 - v;
}

double erf_ref(double x) {
  if (x == 0) return 0.0;
  const double m = std::fabs(x), x2 = m * m;
  const double v = x2 < 1.5 ? lower_gamma_series(0.5, x2) : 1.0 - upper_gamma_fraction(0.5, x2);
  return x >= 0 ? v : -v;
}

// erf.ts:100
double erf_derivative(double x) { return 2.0 * 0.5641895835477563 * std::exp(-x * x); }

// ---------------------------------------------------------- triclinic -----
// src/reference/triclinic.ts:38-470.  Boxes are row-major a, b, c.
double box_volume(const double* b) {
  return std::fabs(b[0] * (b[4] * b[8] - b[5] * b[7]) - b[1] * (b[3] * b[8] - b[5] * b[6]) +
                   b[2] * (b[3] * b[7] - b[4] * b[6]));
}

Vec3 perpendicular_widths(const double* b) {
  auto cross = [](const double* u, const double* v) {
    return Vec3{u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0]};
  };
  auto norm = [](const Vec3& u) { return std::sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]); };
  const double v = box_volume(b);
  return {v / norm(cross(b + 3, b + 6)), v / norm(cross(b + 6, b)), v / norm(cross(b, b + 3))};
}

// triclinic.ts:93 -- ties to even, c against b, then c and b against a.
Box reduce_box(const double* in) {
  Box v;
  std::copy(in, in + 9, v.begin());
  auto reduce_by = [](double ratio) {
    const double nearest = std::round(ratio);
    const bool tie = std::fabs(ratio - std::trunc(ratio)) == 0.5;
    if (tie && std::fmod(std::fabs(nearest), 2.0) != 0.0) return nearest - (ratio > 0 ? 1.0 : -1.0);
    return nearest;
  };
  auto sub = [&](int t, int s, double times) {
    for (int k = 0; k < 3; ++k) v[t * 3 + k] -= times * v[s * 3 + k];
  };
  sub(2, 1, reduce_by(v[7] / v[4]));
  sub(2, 0, reduce_by(v[6] / v[0]));
  sub(1, 0, reduce_by(v[3] / v[0]));
  return v;
}

bool is_reduced(const double* b, double tol = 1e-9) {
  if (std::fabs(b[1]) > tol || std::fabs(b[2]) > tol || std::fabs(b[5]) > tol) return false;
  if (b[0] <= 0 || b[4] <= 0 || b[8] <= 0) return false;
  return std::fabs(b[3]) <= 0.5 * b[0] + tol && std::fabs(b[6]) <= 0.5 * b[0] + tol &&
         std::fabs(b[7]) <= 0.5 * b[4] + tol;
}

// triclinic.ts:394 -- f = r . M, M lower triangular.
std::array<double, 9> inverse_box(const double* b) {
  const double ax = b[0], bx = b[3], by = b[4], cx = b[6], cy = b[7], cz = b[8];
  return {1 / ax, 0, 0, -bx / (ax * by), 1 / by, 0, ((bx * cy) / (by * cz) - cx / cz) / ax,
          -cy / (by * cz), 1 / cz};
}

Vec3 fractional_of(double x, double y, double z, const std::array<double, 9>& m) {
  return {x * m[0] + y * m[3] + z * m[6], x * m[1] + y * m[4] + z * m[7],
          x * m[2] + y * m[5] + z * m[8]};
}

// triclinic.ts:441 -- k = 2 pi m B^-T.
Vec3 reciprocal_vector(double ma, double mb, double mc, const std::array<double, 9>& m) {
  const double tp = 2 * kPi;
  return {tp * ma * m[0], tp * (ma * m[3] + mb * m[4]), tp * (ma * m[6] + mb * m[7] + mc * m[8])};
}

// src/reference/forces/nonbonded.ts:241 -- sequential reduction c, b, a.
inline void nearest_image(const double* b, double& dx, double& dy, double& dz) {
  const double kc = std::round(dz / b[8]);
  dx -= kc * b[6];
  dy -= kc * b[7];
  dz -= kc * b[8];
  const double kb = std::round(dy / b[4]);
  dx -= kb * b[3];
  dy -= kb * b[4];
  dx -= std::round(dx / b[0]) * b[0];
}

// ------------------------------------------------------------ splines -----
// src/reference/forces/bspline.ts:20-55 (weights) and :55 (with derivatives).
void bspline_weights(double w, int order, double* theta) {
  for (int i = 0; i < order; ++i) theta[i] = 0;
  theta[1] = w;
  theta[0] = 1 - w;
  for (int k = 3; k <= order - 1; ++k) {
    const double d = 1.0 / (k - 1);
    theta[k - 1] = d * w * theta[k - 2];
    for (int j = 1; j < k - 1; ++j)
      theta[k - j - 1] = d * ((w + j) * theta[k - j - 2] + (k - j - w) * theta[k - j - 1]);
    theta[0] = d * (1 - w) * theta[0];
  }
  const double d = 1.0 / (order - 1);
  theta[order - 1] = d * w * theta[order - 2];
  for (int j = 1; j < order - 1; ++j)
    theta[order - j - 1] =
        d * ((w + j) * theta[order - j - 2] + (order - j - w) * theta[order - j - 1]);
  theta[0] = d * (1 - w) * theta[0];
}

void bspline_with_derivatives(double w, double* weights, double* derivs) {
  const int order = kPmeOrder;
  double lower[kPmeOrder] = {0, 0, 0, 0, 0};
  lower[1] = w;
  lower[0] = 1 - w;
  for (int k = 3; k <= order - 1; ++k) {
    const double d = 1.0 / (k - 1);
    lower[k - 1] = d * w * lower[k - 2];
    for (int j = 1; j < k - 1; ++j)
      lower[k - j - 1] = d * ((w + j) * lower[k - j - 2] + (k - j - w) * lower[k - j - 1]);
    lower[0] = d * (1 - w) * lower[0];
  }
  derivs[0] = -lower[0];
  for (int j = 1; j < order; ++j) derivs[j] = lower[j - 1] - lower[j];
  for (int j = 0; j < order; ++j) weights[j] = lower[j];
  const double d = 1.0 / (order - 1);
  weights[order - 1] = d * w * weights[order - 2];
  for (int j = 1; j < order - 1; ++j)
    weights[order - j - 1] =
        d * ((w + j) * weights[order - j - 2] + (order - j - w) * weights[order - j - 1]);
  weights[0] = d * (1 - w) * weights[0];
}

// bspline.ts:102 -- 1/|b(m)|^2 ... stored as |b(m)|^2, divided by in the kernel.
std::vector<double> bspline_moduli(int n) {
  std::vector<double> data(n, 0.0), mod(n, 0.0);
  double knots[kPmeOrder];
  bspline_weights(0.0, kPmeOrder, knots);
  for (int i = 0; i < kPmeOrder && i < n; ++i) data[i] = knots[i];
  for (int m = 0; m < n; ++m) {
    double re = 0, im = 0;
    for (int k = 0; k < n; ++k) {
      const double a = 2 * kPi * m * k / n;
      re += data[k] * std::cos(a);
      im += data[k] * std::sin(a);
    }
    mod[m] = re * re + im * im;
  }
  for (int m = 0; m < n; ++m)
    if (mod[m] < 1e-7) mod[m] = 0.5 * (mod[(m - 1 + n) % n] + mod[(m + 1) % n]);
  return mod;
}

// ---------------------------------------------------------------- FFT -----
// src/reference/fft.ts:54-248: Stockham autosort, radices 7, 5, 3, 2 largest
// first, unnormalised; src/reference/dft.ts is the direct transform used when a
// length is not 2/3/5/7-smooth (OpenMM's Reference platform grids, e.g. 22).
using cplx = std::complex<double>;

struct Stage { int radix, ns; };

bool plan_fft(int n, std::vector<Stage>& stages) {
  stages.clear();
  int rem = n, ns = 1;
  for (int r : {7, 5, 3, 2}) {
    while (rem % r == 0) {
      stages.push_back({r, ns});
      ns *= r;
      rem /= r;
    }
  }
  return rem == 1;
}

// One line of length n at `stride`, transformed in place; `sign` -1 forward.
void transform_line(cplx* base, int n, long stride, int sign, std::vector<cplx>& a,
                    std::vector<cplx>& b) {
  a.resize(n);
  b.resize(n);
  for (int i = 0; i < n; ++i) a[i] = base[i * stride];
  std::vector<Stage> stages;
  if (plan_fft(n, stages)) {
    cplx* from = a.data();
    cplx* to = b.data();
    cplx v[7];
    for (const Stage& st : stages) {
      const int r = st.radix, ns = st.ns, bf = n / r;
      for (int j = 0; j < bf; ++j) {
        const int tw = j % ns;
        for (int q = 0; q < r; ++q) {
          cplx x = from[j + q * bf];
          if (q != 0 && tw != 0) {
            const double ang = sign * 2 * kPi * double(tw) * q / double(ns * r);
            x *= cplx(std::cos(ang), std::sin(ang));
          }
          v[q] = x;
        }
        const int dest = (j / ns) * ns * r + tw;
        for (int k = 0; k < r; ++k) {
          cplx s(0, 0);
          for (int m = 0; m < r; ++m) {
            const double ang = sign * 2 * kPi * double(k) * m / r;
            s += v[m] * cplx(std::cos(ang), std::sin(ang));
          }
          to[dest + k * ns] = s;
        }
      }
      std::swap(from, to);
    }
    for (int i = 0; i < n; ++i) base[i * stride] = from[i];
  } else {
    for (int k = 0; k < n; ++k) {
      cplx s(0, 0);
      for (int j = 0; j < n; ++j) {
        const double ang = sign * 2 * kPi * double((long(k) * j) % n) / n;
        s += a[j] * cplx(std::cos(ang), std::sin(ang));
      }
      b[k] = s;
    }
    for (int i = 0; i < n; ++i) base[i * stride] = b[i];
  }
}

// fft.ts:217 -- axes z, y, x over a [nx][ny][nz] grid, z fastest.
void fft3d(std::vector<cplx>& g, int nx, int ny, int nz, int sign, int threads) {
  (void)threads;
#pragma omp parallel num_threads(threads > 1 ? threads : 1)
  {
    std::vector<cplx> a, b;
#pragma omp for collapse(2) schedule(static)
    for (int x = 0; x < nx; ++x)
      for (int y = 0; y < ny; ++y) transform_line(&g[(long(x) * ny + y) * nz], nz, 1, sign, a, b);
#pragma omp for collapse(2) schedule(static)
    for (int x = 0; x < nx; ++x)
      for (int z = 0; z < nz; ++z) transform_line(&g[long(x) * ny * nz + z], ny, nz, sign, a, b);
#pragma omp for collapse(2) schedule(static)
    for (int y = 0; y < ny; ++y)
      for (int z = 0; z < nz; ++z) transform_line(&g[long(y) * nz + z], nx, long(ny) * nz, sign, a, b);
  }
}

// ----------------------------------------------------------- helpers ------
double ewald_alpha(double cutoff, double tol) { return (1.0 / cutoff) * std::sqrt(-std::log(2 * tol)); }

int pme_min_grid(double alpha, double length, double tol) {
  return std::max(6, int(std::ceil((2 * alpha * length) / (3 * std::pow(tol, 0.2)))));
}

int smooth_size(int minimum) {
  for (int n = std::max(1, minimum);; ++n) {
    int r = n;
    for (int p : {2, 3, 5, 7})
      while (r % p == 0) r /= p;
    if (r == 1) return n;
  }
}

double splitting_parameter(const mdb_system_desc* s) {
  return s->alpha != 0 ? s->alpha : ewald_alpha(s->cutoff, s->ewald_tolerance);
}

// potential.ts:79 -- from the box *diagonal*.
std::array<int, 3> default_grid(const mdb_system_desc* s, const double* box, double alpha) {
  return {smooth_size(pme_min_grid(alpha, box[0], s->ewald_tolerance)),
          smooth_size(pme_min_grid(alpha, box[4], s->ewald_tolerance)),
          smooth_size(pme_min_grid(alpha, box[8], s->ewald_tolerance))};
}

// Exclusions as a hash set of (min, max) pairs (nonbonded.ts:189).
std::unordered_set<uint64_t> exclusion_set(const mdb_system_desc* s) {
  std::unordered_set<uint64_t> set;
  set.reserve(size_t(s->n_exceptions) * 2 + 1);
  for (int e = 0; e < s->n_exceptions; ++e) {
    const uint64_t a = std::min(s->exception_p1[e], s->exception_p2[e]);
    const uint64_t b = std::max(s->exception_p1[e], s->exception_p2[e]);
    set.insert(a * 2097152ull + b);
  }
  return set;
}

// --------------------------------------------------------- nonbonded ------
// src/reference/forces/nonbonded.ts:279 -- one non-excluded pair.
// Virial tensor W[3a+b] = sum r_a F_b over every interaction (r the
// separation, F the force on the atom it points from) = -dU/d eps_ab for the
// affine strain x -> (1 + eps) x of positions and box.  Filled only while
// orc_potential_virial runs; position restraints are left out (their anchors
// do not move with the box).  No reference counterpart: the reference has no
// virial.
double* g_virial = nullptr;

inline void add_virial(double* w, double rx, double ry, double rz, double fx, double fy, double fz) {
  const double r[3] = {rx, ry, rz}, f[3] = {fx, fy, fz};
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) w[3 * a + b] += r[a] * f[b];
}

struct PairAcc { double coulomb = 0, lj = 0; int64_t pairs = 0; double vir[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}; };

// erfc-Coulomb plus Lorentz-Berthelot LJ of one pair at squared distance r2
// (nonbonded.ts:330): the energies, and dE/dr as the return value.
inline double pair_terms(const mdb_system_desc* s, double alpha, int i, int j, double r2, double& coulomb,
                         double& lj) {
  const double r = std::sqrt(r2);
  const double qq = kOne4PiEps0 * s->charge[i] * s->charge[j];
  const double ar = alpha * r;
  const double ec = erfc_ref(ar);
  coulomb = qq * ec / r;
  double dEdR = qq * (-ec / r2 - alpha * erf_derivative(ar) / r);
  lj = 0;
  const double eps = std::sqrt(s->epsilon[i] * s->epsilon[j]);
  if (eps != 0) {
    const double sig = 0.5 * (s->sigma[i] + s->sigma[j]);
    const double s6 = std::pow(sig * sig / r2, 3);
    const double s12 = s6 * s6;
    lj = 4 * eps * (s12 - s6);
    dEdR += (4 * eps / r) * (6 * s6 - 12 * s12);
  }
  return dEdR;
}

inline void pair_interaction(const mdb_system_desc* s, const double* pos, const double* box,
                             double alpha, double cut2, int i, int j, double* forces,
                             PairAcc& acc) {
  double dx = pos[3 * j] - pos[3 * i], dy = pos[3 * j + 1] - pos[3 * i + 1],
         dz = pos[3 * j + 2] - pos[3 * i + 2];
  nearest_image(box, dx, dy, dz);
  const double r2 = dx * dx + dy * dy + dz * dz;
  if (r2 >= cut2) return;
  const double r = std::sqrt(r2);
  double coulomb, lj;
  const double dEdR = pair_terms(s, alpha, i, j, r2, coulomb, lj);
  if (forces) {
    const double sc = dEdR / r;
    forces[3 * i] += sc * dx;
    forces[3 * i + 1] += sc * dy;
    forces[3 * i + 2] += sc * dz;
    forces[3 * j] -= sc * dx;
    forces[3 * j + 1] -= sc * dy;
    forces[3 * j + 2] -= sc * dz;
  }
  if (g_virial) {
    // pair (i, j): r_i - r_j = -d, force on i = (dEdR / r) d
    const double sc = dEdR / r;
    add_virial(acc.vir, -dx, -dy, -dz, sc * dx, sc * dy, sc * dz);
  }
  if (coulomb != 0 || lj != 0) acc.pairs++;
  acc.coulomb += coulomb;
  acc.lj += lj;
}

// nonbonded.ts:330 -- every exception, at any distance.
void exception_terms(const mdb_system_desc* s, const double* pos, const double* box, double alpha,
                     double* forces, double& correction, double& exceptions) {
  correction = 0;
  exceptions = 0;
  for (int e = 0; e < s->n_exceptions; ++e) {
    const int i = s->exception_p1[e], j = s->exception_p2[e];
    double dx = pos[3 * j] - pos[3 * i], dy = pos[3 * j + 1] - pos[3 * i + 1],
           dz = pos[3 * j + 2] - pos[3 * i + 2];
    nearest_image(box, dx, dy, dz);
    const double r2 = dx * dx + dy * dy + dz * dz, r = std::sqrt(r2), ar = alpha * r;
    double dEdR = 0;
    const double pp = kOne4PiEps0 * s->charge[i] * s->charge[j];
    if (pp != 0) {
      const double ef = erf_ref(ar);
      correction -= pp * ef / r;
      dEdR += pp * (ef / r2 - alpha * erf_derivative(ar) / r);
    }
    const double cp = kOne4PiEps0 * s->exception_charge_prod[e];
    if (cp != 0) {
      exceptions += cp / r;
      dEdR += -cp / r2;
    }
    const double eps = s->exception_epsilon[e];
    if (eps != 0) {
      const double sig = s->exception_sigma[e];
      const double s6 = std::pow(sig * sig / r2, 3), s12 = s6 * s6;
      exceptions += 4 * eps * (s12 - s6);
      dEdR += (4 * eps / r) * (6 * s6 - 12 * s12);
    }
    if (g_virial && dEdR != 0) {
      const double sc = dEdR / r;
      add_virial(g_virial, -dx, -dy, -dz, sc * dx, sc * dy, sc * dz);
    }
    if (forces && dEdR != 0) {
      const double sc = dEdR / r;
      forces[3 * i] += sc * dx;
      forces[3 * i + 1] += sc * dy;
      forces[3 * i + 2] += sc * dz;
      forces[3 * j] -= sc * dx;
      forces[3 * j + 1] -= sc * dy;
      forces[3 * j + 2] -= sc * dz;
    }
  }
}

// nonbonded.ts:107 -- grouped by (sigma, epsilon) class, pairs including i==j.
double dispersion_correction(const mdb_system_desc* s, double volume) {
  const int n = s->n_particles;
  if (n == 0) return 0;
  std::vector<double> sig, eps;
  std::vector<double> cnt;
  for (int i = 0; i < n; ++i) {
    size_t c = 0;
    for (; c < sig.size(); ++c)
      if (sig[c] == s->sigma[i] && eps[c] == s->epsilon[i]) break;
    if (c == sig.size()) {
      sig.push_back(s->sigma[i]);
      eps.push_back(s->epsilon[i]);
      cnt.push_back(0);
    }
    cnt[c] += 1;
  }
  double s6 = 0, s12 = 0;
  for (size_t c = 0; c < sig.size(); ++c)
    for (size_t d = c; d < sig.size(); ++d) {
      const double sg = 0.5 * (sig[c] + sig[d]), ep = std::sqrt(eps[c] * eps[d]);
      const double sg6 = std::pow(sg, 6);
      const double mult = c == d ? cnt[c] * (cnt[c] + 1) / 2 : cnt[c] * cnt[d];
      s6 += mult * ep * sg6;
      s12 += mult * ep * sg6 * sg6;
    }
  const double pairs = double(n) * (n + 1) / 2, rc = s->cutoff;
  return (8 * kPi * double(n) * n / volume) *
         ((s12 / pairs) / (9 * std::pow(rc, 9)) - (s6 / pairs) / (3 * std::pow(rc, 3)));
}

// nonbonded.ts:594, :610
double net_charge_correction(const mdb_system_desc* s, double alpha, double volume) {
  double q = 0;
  for (int i = 0; i < s->n_particles; ++i) q += s->charge[i];
  return (-kPi * q * q * kOne4PiEps0) / (2 * alpha * alpha * volume);
}

double self_energy(const mdb_system_desc* s, double alpha) {
  double q2 = 0;
  for (int i = 0; i < s->n_particles; ++i) q2 += s->charge[i] * s->charge[i];
  return (-kOne4PiEps0 * alpha * q2) / std::sqrt(kPi);
}

// nonbonded.ts:394 (naive) and :447 (cell list), threaded over i with private
// force arrays; the sums are the same pairs in a different order.
void direct_pairs(const mdb_system_desc* s, const double* pos, const double* box, double alpha,
                  double* forces, PairAcc& total, int threads, bool naive) {
  const int n = s->n_particles;
  const double cut = s->cutoff, cut2 = cut * cut;
  const auto excluded = exclusion_set(s);
  const Vec3 widths = perpendicular_widths(box);
  int counts[3];
  for (int a = 0; a < 3; ++a) counts[a] = std::max(1, int(std::floor(widths[a] / cut)));
  if (counts[0] < 3 || counts[1] < 3 || counts[2] < 3) naive = true;
  const int nt = threads > 1 ? threads : 1;
  std::vector<std::vector<double>> tf(nt);
  std::vector<PairAcc> ta(nt);

  std::vector<int> order, start;
  std::vector<int> cell_of;
  if (!naive) {
    const int ncell = counts[0] * counts[1] * counts[2];
    const auto inv = inverse_box(box);
    cell_of.resize(n);
    start.assign(ncell + 1, 0);
    auto bucket = [](double f, int div) {
      const double w = f - std::floor(f);
      const int idx = int(std::floor(w * div));
      return idx == div ? div - 1 : idx;
    };
    for (int i = 0; i < n; ++i) {
      const Vec3 f = fractional_of(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], inv);
      const int c = (bucket(f[0], counts[0]) * counts[1] + bucket(f[1], counts[1])) * counts[2] +
                    bucket(f[2], counts[2]);
      cell_of[i] = c;
      start[c + 1]++;
    }
    for (int c = 0; c < ncell; ++c) start[c + 1] += start[c];
    order.resize(n);
    std::vector<int> cur(start.begin(), start.end() - 1);
    for (int i = 0; i < n; ++i) order[cur[cell_of[i]]++] = i;
  }

#pragma omp parallel num_threads(nt)
  {
    int t = 0;
#ifdef _OPENMP
    t = omp_get_thread_num();
#endif
    double* f = nullptr;
    if (forces) {
      tf[t].assign(size_t(3) * n, 0.0);
      f = tf[t].data();
    }
    PairAcc acc;
    if (naive) {
#pragma omp for schedule(dynamic, 16)
      for (int i = 0; i < n; ++i)
        for (int j = i + 1; j < n; ++j) {
          if (excluded.count(uint64_t(i) * 2097152ull + j)) continue;
          pair_interaction(s, pos, box, alpha, cut2, i, j, f, acc);
        }
    } else {
      const int ncell = counts[0] * counts[1] * counts[2];
#pragma omp for schedule(dynamic, 4)
      for (int cell = 0; cell < ncell; ++cell) {
        const int cz = cell % counts[2], cy = (cell / counts[2]) % counts[1],
                  cx = cell / (counts[1] * counts[2]);
        for (int ddx = -1; ddx <= 1; ++ddx)
          for (int ddy = -1; ddy <= 1; ++ddy)
            for (int ddz = -1; ddz <= 1; ++ddz) {
              const int nx = (cx + ddx + counts[0]) % counts[0];
              const int ny = (cy + ddy + counts[1]) % counts[1];
              const int nz = (cz + ddz + counts[2]) % counts[2];
              const int nb = (nx * counts[1] + ny) * counts[2] + nz;
              if (nb < cell) continue;
              for (int a = start[cell]; a < start[cell + 1]; ++a) {
                const int i = order[a];
                const int from = nb == cell ? a + 1 : start[nb];
                for (int b = from; b < start[nb + 1]; ++b) {
                  const int j = order[b];
                  const int lo = std::min(i, j), hi = std::max(i, j);
                  if (excluded.count(uint64_t(lo) * 2097152ull + hi)) continue;
                  pair_interaction(s, pos, box, alpha, cut2, lo, hi, f, acc);
                }
              }
            }
      }
    }
    ta[t] = acc;
  }
  for (int t = 0; t < nt; ++t) {
    total.coulomb += ta[t].coulomb;
    total.lj += ta[t].lj;
    total.pairs += ta[t].pairs;
    for (int k = 0; k < 9; ++k) total.vir[k] += ta[t].vir[k];
    if (forces)
      for (size_t k = 0; k < size_t(3) * n; ++k) forces[k] += tf[t][k];
  }
}

// ---------------------------------------------------------------- PME -----
// src/reference/forces/pme.ts:93-263: order-5 spread, transform, convolve with
// exp(-k^2/4a^2)/(k^2 |b|^2), transform back, interpolate the gradient.
double reciprocal_space(const mdb_system_desc* s, const double* pos, const double* box,
                        double alpha, const int* grid, double* forces, int threads) {
  const int nx = grid[0], ny = grid[1], nz = grid[2], n = s->n_particles;
  const auto inv = inverse_box(box);
  std::vector<cplx> g(size_t(nx) * ny * nz, cplx(0, 0));
  struct Spline { int base[3]; double w[3][kPmeOrder], d[3][kPmeOrder]; };
  std::vector<Spline> sp(n);
  const int dims[3] = {nx, ny, nz};
  for (int i = 0; i < n; ++i) {
    const Vec3 f = fractional_of(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], inv);
    for (int a = 0; a < 3; ++a) {
      const double frac = f[a] - std::floor(f[a]);
      const double scaled = frac * dims[a];
      const double cell = std::floor(scaled);
      bspline_with_derivatives(scaled - cell, sp[i].w[a], sp[i].d[a]);
      sp[i].base[a] = int(cell) - kPmeOrder + 1;
    }
  }
  for (int i = 0; i < n; ++i) {
    const double q = s->charge[i];
    if (q == 0) continue;
    const Spline& S = sp[i];
    for (int a = 0; a < kPmeOrder; ++a) {
      const int gx = (((S.base[0] + a) % nx) + nx) % nx;
      const double wx = q * S.w[0][a];
      for (int b = 0; b < kPmeOrder; ++b) {
        const int gy = (((S.base[1] + b) % ny) + ny) % ny;
        const double wxy = wx * S.w[1][b];
        for (int c = 0; c < kPmeOrder; ++c) {
          const int gz = (((S.base[2] + c) % nz) + nz) % nz;
          g[(size_t(gx) * ny + gy) * nz + gz] += wxy * S.w[2][c];
        }
      }
    }
  }
  fft3d(g, nx, ny, nz, -1, threads);
  const auto mx_ = bspline_moduli(nx), my_ = bspline_moduli(ny), mz_ = bspline_moduli(nz);
  const double volume = box_volume(box);
  const double pref = (kOne4PiEps0 * 2 * kPi) / volume;
  const double expScale = -1 / (4 * alpha * alpha);
  double energy = 0;
  for (int x = 0; x < nx; ++x) {
    const int ma = x <= nx / 2 ? x : x - nx;
    for (int y = 0; y < ny; ++y) {
      const int mb = y <= ny / 2 ? y : y - ny;
      for (int z = 0; z < nz; ++z) {
        cplx& v = g[(size_t(x) * ny + y) * nz + z];
        if (x == 0 && y == 0 && z == 0) {
          v = 0;
          continue;
        }
        const int mc = z <= nz / 2 ? z : z - nz;
        const Vec3 k = reciprocal_vector(ma, mb, mc, inv);
        const double k2 = k[0] * k[0] + k[1] * k[1] + k[2] * k[2];
        const double modulus = mx_[x] * my_[y] * mz_[z];
        const double factor = (pref * std::exp(k2 * expScale)) / (k2 * modulus);
        energy += factor * std::norm(v);
        if (g_virial) {
          // -dE_k/d eps_ab = E_k (delta_ab - 2 k_a k_b (1/k^2 + 1/(4 alpha^2)))
          const double ek = factor * std::norm(v), c = 2 * (1 / k2 - expScale);
          for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) g_virial[3 * a + b] += ek * ((a == b ? 1.0 : 0.0) - c * k[a] * k[b]);
        }
        v *= 2 * factor;
      }
    }
  }
  if (!forces) return energy;
  fft3d(g, nx, ny, nz, +1, threads);
#pragma omp parallel for num_threads(threads > 1 ? threads : 1) schedule(static)
  for (int i = 0; i < n; ++i) {
    const double q = s->charge[i];
    if (q == 0) continue;
    const Spline& S = sp[i];
    double fx = 0, fy = 0, fz = 0;
    for (int a = 0; a < kPmeOrder; ++a) {
      const int gx = (((S.base[0] + a) % nx) + nx) % nx;
      for (int b = 0; b < kPmeOrder; ++b) {
        const int gy = (((S.base[1] + b) % ny) + ny) % ny;
        for (int c = 0; c < kPmeOrder; ++c) {
          const int gz = (((S.base[2] + c) % nz) + nz) % nz;
          const double p = g[(size_t(gx) * ny + gy) * nz + gz].real();
          fx += p * S.d[0][a] * S.w[1][b] * S.w[2][c];
          fy += p * S.w[0][a] * S.d[1][b] * S.w[2][c];
          fz += p * S.w[0][a] * S.w[1][b] * S.d[2][c];
        }
      }
    }
    const double df[3] = {-q * fx * nx, -q * fy * ny, -q * fz * nz};
    for (int ax = 0; ax < 3; ++ax)
      forces[3 * i + ax] += df[0] * inv[ax * 3 + 0] + df[1] * inv[ax * 3 + 1] + df[2] * inv[ax * 3 + 2];
  }
  return energy;
}

// ------------------------------------------------------------- bonded -----
// src/reference/forces/bonded.ts:39 (bond), :71 (angle), :133 (torsion).
double harmonic_bonds(const mdb_system_desc* s, const double* pos, double* f) {
  double e = 0;
  for (int t = 0; t < s->n_bonds; ++t) {
    const int a = 3 * s->bond_p1[t], b = 3 * s->bond_p2[t];
    const double dx = pos[b] - pos[a], dy = pos[b + 1] - pos[a + 1], dz = pos[b + 2] - pos[a + 2];
    const double r = std::sqrt(dx * dx + dy * dy + dz * dz), dr = r - s->bond_length[t];
    const double k = s->bond_k[t];
    e += 0.5 * k * dr * dr;
    if (f) {
      const double sc = k * dr / r;
      f[a] += sc * dx; f[a + 1] += sc * dy; f[a + 2] += sc * dz;
      f[b] -= sc * dx; f[b + 1] -= sc * dy; f[b + 2] -= sc * dz;
      if (g_virial) add_virial(g_virial, dx, dy, dz, -sc * dx, -sc * dy, -sc * dz);
    }
  }
  return e;
}

double harmonic_angles(const mdb_system_desc* s, const double* pos, double* f) {
  double e = 0;
  for (int t = 0; t < s->n_angles; ++t) {
    const int a = 3 * s->angle_p1[t], b = 3 * s->angle_p2[t], c = 3 * s->angle_p3[t];
    const double v1x = pos[a] - pos[b], v1y = pos[a + 1] - pos[b + 1], v1z = pos[a + 2] - pos[b + 2];
    const double v2x = pos[c] - pos[b], v2y = pos[c + 1] - pos[b + 1], v2z = pos[c + 2] - pos[b + 2];
    const double r1 = v1x * v1x + v1y * v1y + v1z * v1z, r2 = v2x * v2x + v2y * v2y + v2z * v2z;
    const double dot = v1x * v2x + v1y * v2y + v1z * v2z;
    const double cs = std::min(1.0, std::max(-1.0, dot / std::sqrt(r1 * r2)));
    const double th = std::acos(cs), k = s->angle_k[t], dth = th - s->angle_theta[t];
    e += 0.5 * k * dth * dth;
    if (!f) continue;
    const double nx = v1y * v2z - v1z * v2y, ny = v1z * v2x - v1x * v2z, nz = v1x * v2y - v1y * v2x;
    const double nn = std::max(std::sqrt(nx * nx + ny * ny + nz * nz), 1e-6);
    const double dE = k * dth;
    const double tA = dE / (r1 * nn), tC = -dE / (r2 * nn);
    const double f1x = -tA * (v1y * nz - v1z * ny), f1y = -tA * (v1z * nx - v1x * nz),
                 f1z = -tA * (v1x * ny - v1y * nx);
    const double f3x = -tC * (v2y * nz - v2z * ny), f3y = -tC * (v2z * nx - v2x * nz),
                 f3z = -tC * (v2x * ny - v2y * nx);
    f[a] += f1x; f[a + 1] += f1y; f[a + 2] += f1z;
    f[c] += f3x; f[c + 1] += f3y; f[c + 2] += f3z;
    f[b] -= f1x + f3x; f[b + 1] -= f1y + f3y; f[b + 2] -= f1z + f3z;
    if (g_virial) {
      add_virial(g_virial, v1x, v1y, v1z, f1x, f1y, f1z);
      add_virial(g_virial, v2x, v2y, v2z, f3x, f3y, f3z);
    }
  }
  return e;
}

double periodic_torsions(const mdb_system_desc* s, const double* pos, double* f) {
  double e = 0;
  for (int t = 0; t < s->n_torsions; ++t) {
    const int a = 3 * s->torsion_p1[t], b = 3 * s->torsion_p2[t], c = 3 * s->torsion_p3[t],
              d = 3 * s->torsion_p4[t];
    const double b1x = pos[b] - pos[a], b1y = pos[b + 1] - pos[a + 1], b1z = pos[b + 2] - pos[a + 2];
    const double b2x = pos[c] - pos[b], b2y = pos[c + 1] - pos[b + 1], b2z = pos[c + 2] - pos[b + 2];
    const double b3x = pos[d] - pos[c], b3y = pos[d + 1] - pos[c + 1], b3z = pos[d + 2] - pos[c + 2];
    const double n1x = b1y * b2z - b1z * b2y, n1y = b1z * b2x - b1x * b2z, n1z = b1x * b2y - b1y * b2x;
    const double n2x = b2y * b3z - b2z * b3y, n2y = b2z * b3x - b2x * b3z, n2z = b2x * b3y - b2y * b3x;
    const double n1 = n1x * n1x + n1y * n1y + n1z * n1z, n2 = n2x * n2x + n2y * n2y + n2z * n2z;
    const double b2n = std::sqrt(b2x * b2x + b2y * b2y + b2z * b2z);
    const double X = n1x * n2x + n1y * n2y + n1z * n2z;
    const double Y = b2n * (b1x * n2x + b1y * n2y + b1z * n2z);
    const double phi = std::atan2(Y, X);
    const double per = s->torsion_periodicity[t], ph = s->torsion_phase[t], k = s->torsion_k[t];
    e += k * (1 + std::cos(per * phi - ph));
    if (!f) continue;
    const double dEdPhi = -k * per * std::sin(per * phi - ph);
    if (n1 == 0 || n2 == 0) continue;
    const double s1 = dEdPhi * b2n / n1, s4 = -dEdPhi * b2n / n2;
    const double f1x = s1 * n1x, f1y = s1 * n1y, f1z = s1 * n1z;
    const double f4x = s4 * n2x, f4y = s4 * n2y, f4z = s4 * n2z;
    const double b2sq = b2n * b2n;
    const double ss = (b1x * b2x + b1y * b2y + b1z * b2z) / b2sq;
    const double tt = (b3x * b2x + b3y * b2y + b3z * b2z) / b2sq;
    f[a] += f1x; f[a + 1] += f1y; f[a + 2] += f1z;
    f[b] += -(1 + ss) * f1x + tt * f4x; f[b + 1] += -(1 + ss) * f1y + tt * f4y;
    f[b + 2] += -(1 + ss) * f1z + tt * f4z;
    f[c] += ss * f1x - (1 + tt) * f4x; f[c + 1] += ss * f1y - (1 + tt) * f4y;
    f[c + 2] += ss * f1z - (1 + tt) * f4z;
    f[d] += f4x; f[d + 1] += f4y; f[d + 2] += f4z;
    if (g_virial) {
      add_virial(g_virial, b1x, b1y, b1z, -(1 + ss) * f1x + tt * f4x, -(1 + ss) * f1y + tt * f4y,
                 -(1 + ss) * f1z + tt * f4z);
      add_virial(g_virial, b1x + b2x, b1y + b2y, b1z + b2z, ss * f1x - (1 + tt) * f4x,
                 ss * f1y - (1 + tt) * f4y, ss * f1z - (1 + tt) * f4z);
      add_virial(g_virial, b1x + b2x + b3x, b1y + b2y + b3y, b1z + b2z + b3z, f4x, f4y, f4z);
    }
  }
  return e;
}

// src/reference/forces/restraint.ts:38 -- k |minimum image(r - r0)|^2.
double position_restraints(const mdb_system_desc* s, const double* pos, const double* box, double* f) {
  double e = 0;
  for (int t = 0; t < s->n_restraints; ++t) {
    const int p = s->restraint_particle[t];
    double dx = pos[3 * p] - s->restraint_x0[t], dy = pos[3 * p + 1] - s->restraint_y0[t],
           dz = pos[3 * p + 2] - s->restraint_z0[t];
    nearest_image(box, dx, dy, dz);
    const double k = s->restraint_k[t];
    e += k * (dx * dx + dy * dy + dz * dz);
    if (f) {
      f[3 * p] -= 2 * k * dx;
      f[3 * p + 1] -= 2 * k * dy;
      f[3 * p + 2] -= 2 * k * dz;
    }
  }
  return e;
}

// -------------------------------------------------------- constraints -----
// src/engine/constraint-clusters.ts:93 -- SETTLE triangles, the rest iterative.
struct Settle { int central, first, second; double d1, d2; };
struct Split {
  std::vector<Settle> settle;
  std::vector<int> iterative;  // constraint indices
  std::vector<std::vector<int>> clusters;
  int largest_atoms = 0, largest_constraints = 0;
  bool too_large = false;
};

Split split_constraints(const mdb_system_desc* s) {
  Split out;
  const int n = s->n_particles, count = s->n_constraints;
  std::vector<int> ccount(n, 0);
  std::vector<char> live(count, 0);
  for (int c = 0; c < count; ++c) {
    const int p1 = s->constraint_p1[c], p2 = s->constraint_p2[c];
    if (s->masses[p1] == 0 && s->masses[p2] == 0) continue;
    live[c] = 1;
    ccount[p1]++;
    ccount[p2]++;
  }
  // partners[a] = list of (b, f32 distance), insertion ordered, for atoms with
  // exactly two constraints at both ends.
  std::vector<std::vector<std::pair<int, float>>> partners(n);
  for (int c = 0; c < count; ++c) {
    if (!live[c]) continue;
    const int p1 = s->constraint_p1[c], p2 = s->constraint_p2[c];
    if (ccount[p1] == 2 && ccount[p2] == 2) {
      const float d = float(s->constraint_distance[c]);
      auto link = [&](int a, int b) {
        for (auto& pr : partners[a])
          if (pr.first == b) { pr.second = d; return; }
        partners[a].push_back({b, d});
      };
      link(p1, p2);
      link(p2, p1);
    }
  }
  auto has = [&](int a, int b) {
    for (auto& pr : partners[a]) if (pr.first == b) return true;
    return false;
  };
  auto dist = [&](int a, int b) {
    for (auto& pr : partners[a]) if (pr.first == b) return pr.second;
    return -1.0f;
  };
  std::vector<char> valid(n, 0);
  for (int a = 0; a < n; ++a) {
    if (partners[a].size() != 2) continue;
    const int f1 = partners[a][0].first, f2 = partners[a][1].first;
    if (partners[f1].size() == 2 && partners[f2].size() == 2 && has(f1, f2)) valid[a] = 1;
  }
  std::vector<char> is_settle(n, 0);
  for (int a = 0; a < n; ++a) {
    if (!valid[a]) continue;
    const int p2 = partners[a][0].first, p3 = partners[a][1].first;
    if (!(a < p2 && a < p3)) continue;
    const float d12 = dist(a, p2), d13 = dist(a, p3), d23 = dist(p2, p3);
    Settle st{};
    bool ok = true;
    if (d12 == d13) st = {a, p2, p3, d12, d23};
    else if (d12 == d23) st = {p2, a, p3, d12, d13};
    else if (d13 == d23) st = {p3, a, p2, d13, d12};
    else ok = false;
    if (!ok) continue;
    out.settle.push_back(st);
    is_settle[a] = is_settle[p2] = is_settle[p3] = 1;
  }
  for (int c = 0; c < count; ++c) {
    if (!live[c]) continue;
    if (is_settle[s->constraint_p1[c]]) continue;
    out.iterative.push_back(c);
  }
  // union-find into connected clusters
  std::vector<int> parent(n);
  std::iota(parent.begin(), parent.end(), 0);
  std::function<int(int)> find = [&](int x) {
    while (parent[x] != x) { parent[x] = parent[parent[x]]; x = parent[x]; }
    return x;
  };
  for (int c : out.iterative) {
    const int a = find(s->constraint_p1[c]), b = find(s->constraint_p2[c]);
    if (a != b) parent[a] = b;
  }
  std::vector<int> label(n, -1);
  std::vector<std::vector<int>> atoms;
  for (int c : out.iterative) {
    const int r = find(s->constraint_p1[c]);
    if (label[r] < 0) {
      label[r] = int(out.clusters.size());
      out.clusters.push_back({});
      atoms.push_back({});
    }
    out.clusters[label[r]].push_back(c);
    auto& at = atoms[label[r]];
    for (int p : {s->constraint_p1[c], s->constraint_p2[c]})
      if (std::find(at.begin(), at.end(), p) == at.end()) at.push_back(p);
  }
  for (size_t k = 0; k < out.clusters.size(); ++k) {
    out.largest_atoms = std::max(out.largest_atoms, int(atoms[k].size()));
    out.largest_constraints = std::max(out.largest_constraints, int(out.clusters[k].size()));
    if (atoms[k].size() > 8 || out.clusters[k].size() > 8) out.too_large = true;
  }
  return out;
}

// src/reference/settle.ts:31 (positions) -- Miyamoto & Kollman, in the frame of
// the reference triangle.
void settle_positions(const mdb_system_desc* s, const std::vector<Settle>& cl, const double* ref,
                      double* trial) {
  for (const Settle& c : cl) {
    const int a0 = 3 * c.central, a1 = 3 * c.first, a2 = 3 * c.second;
    const double m0 = s->masses[c.central], m1 = s->masses[c.first], m2 = s->masses[c.second];
    const double xp0[3] = {trial[a0] - ref[a0], trial[a0 + 1] - ref[a0 + 1], trial[a0 + 2] - ref[a0 + 2]};
    const double xp1[3] = {trial[a1] - ref[a1], trial[a1 + 1] - ref[a1 + 1], trial[a1 + 2] - ref[a1 + 2]};
    const double xp2[3] = {trial[a2] - ref[a2], trial[a2 + 1] - ref[a2 + 1], trial[a2 + 2] - ref[a2 + 2]};
    const double xb0 = ref[a1] - ref[a0], yb0 = ref[a1 + 1] - ref[a0 + 1], zb0 = ref[a1 + 2] - ref[a0 + 2];
    const double xc0 = ref[a2] - ref[a0], yc0 = ref[a2 + 1] - ref[a0 + 1], zc0 = ref[a2 + 2] - ref[a0 + 2];
    const double itm = 1 / (m0 + m1 + m2);
    const double xcom = (xp0[0] * m0 + (xb0 + xp1[0]) * m1 + (xc0 + xp2[0]) * m2) * itm;
    const double ycom = (xp0[1] * m0 + (yb0 + xp1[1]) * m1 + (yc0 + xp2[1]) * m2) * itm;
    const double zcom = (xp0[2] * m0 + (zb0 + xp1[2]) * m1 + (zc0 + xp2[2]) * m2) * itm;
    const double xa1 = xp0[0] - xcom, ya1 = xp0[1] - ycom, za1 = xp0[2] - zcom;
    const double xb1 = xb0 + xp1[0] - xcom, yb1 = yb0 + xp1[1] - ycom, zb1 = zb0 + xp1[2] - zcom;
    const double xc1 = xc0 + xp2[0] - xcom, yc1 = yc0 + xp2[1] - ycom, zc1 = zc0 + xp2[2] - zcom;
    const double xZ = yb0 * zc0 - zb0 * yc0, yZ = zb0 * xc0 - xb0 * zc0, zZ = xb0 * yc0 - yb0 * xc0;
    const double xX = ya1 * zZ - za1 * yZ, yX = za1 * xZ - xa1 * zZ, zX = xa1 * yZ - ya1 * xZ;
    const double xY = yZ * zX - zZ * yX, yY = zZ * xX - xZ * zX, zY = xZ * yX - yZ * xX;
    const double lx = std::sqrt(xX * xX + yX * yX + zX * zX);
    const double ly = std::sqrt(xY * xY + yY * yY + zY * zY);
    const double lz = std::sqrt(xZ * xZ + yZ * yZ + zZ * zZ);
    const double t11 = xX / lx, t21 = yX / lx, t31 = zX / lx;
    const double t12 = xY / ly, t22 = yY / ly, t32 = zY / ly;
    const double t13 = xZ / lz, t23 = yZ / lz, t33 = zZ / lz;
    const double xb0d = t11 * xb0 + t21 * yb0 + t31 * zb0, yb0d = t12 * xb0 + t22 * yb0 + t32 * zb0;
    const double xc0d = t11 * xc0 + t21 * yc0 + t31 * zc0, yc0d = t12 * xc0 + t22 * yc0 + t32 * zc0;
    const double za1d = t13 * xa1 + t23 * ya1 + t33 * za1;
    const double xb1d = t11 * xb1 + t21 * yb1 + t31 * zb1, yb1d = t12 * xb1 + t22 * yb1 + t32 * zb1;
    const double zb1d = t13 * xb1 + t23 * yb1 + t33 * zb1;
    const double xc1d = t11 * xc1 + t21 * yc1 + t31 * zc1, yc1d = t12 * xc1 + t22 * yc1 + t32 * zc1;
    const double zc1d = t13 * xc1 + t23 * yc1 + t33 * zc1;
    const double rc = 0.5 * c.d2;
    double rb = std::sqrt(c.d1 * c.d1 - rc * rc);
    const double ra = rb * (m1 + m2) * itm;
    rb -= ra;
    const double sinphi = za1d / ra, cosphi = std::sqrt(1 - sinphi * sinphi);
    const double sinpsi = (zb1d - zc1d) / (2 * rc * cosphi), cospsi = std::sqrt(1 - sinpsi * sinpsi);
    const double ya2d = ra * cosphi;
    double xb2d = -rc * cospsi;
    const double yb2d = -rb * cosphi - rc * sinpsi * sinphi, yc2d = -rb * cosphi + rc * sinpsi * sinphi;
    const double xb2d2 = xb2d * xb2d;
    const double hh2 = 4 * xb2d2 + (yb2d - yc2d) * (yb2d - yc2d) + (zb1d - zc1d) * (zb1d - zc1d);
    const double deltx = 2 * xb2d + std::sqrt(4 * xb2d2 - hh2 + c.d2 * c.d2);
    xb2d -= deltx * 0.5;
    const double al = xb2d * (xb0d - xc0d) + yb0d * yb2d + yc0d * yc2d;
    const double be = xb2d * (yc0d - yb0d) + xb0d * yb2d + xc0d * yc2d;
    const double ga = xb0d * yb1d - xb1d * yb0d + xc0d * yc1d - xc1d * yc0d;
    const double a2b2 = al * al + be * be;
    const double sinth = (al * ga - be * std::sqrt(a2b2 - ga * ga)) / a2b2;
    const double costh = std::sqrt(1 - sinth * sinth);
    const double xa3d = -ya2d * sinth, ya3d = ya2d * costh, za3d = za1d;
    const double xb3d = xb2d * costh - yb2d * sinth, yb3d = xb2d * sinth + yb2d * costh, zb3d = zb1d;
    const double xc3d = -xb2d * costh - yc2d * sinth, yc3d = -xb2d * sinth + yc2d * costh, zc3d = zc1d;
    const double xa3 = t11 * xa3d + t12 * ya3d + t13 * za3d, ya3 = t21 * xa3d + t22 * ya3d + t23 * za3d,
                 za3 = t31 * xa3d + t32 * ya3d + t33 * za3d;
    const double xb3 = t11 * xb3d + t12 * yb3d + t13 * zb3d, yb3 = t21 * xb3d + t22 * yb3d + t23 * zb3d,
                 zb3 = t31 * xb3d + t32 * yb3d + t33 * zb3d;
    const double xc3 = t11 * xc3d + t12 * yc3d + t13 * zc3d, yc3 = t21 * xc3d + t22 * yc3d + t23 * zc3d,
                 zc3 = t31 * xc3d + t32 * yc3d + t33 * zc3d;
    trial[a0] = ref[a0] + xcom + xa3;
    trial[a0 + 1] = ref[a0 + 1] + ycom + ya3;
    trial[a0 + 2] = ref[a0 + 2] + zcom + za3;
    trial[a1] = ref[a1] + xcom + xb3 - xb0;
    trial[a1 + 1] = ref[a1 + 1] + ycom + yb3 - yb0;
    trial[a1 + 2] = ref[a1 + 2] + zcom + zb3 - zb0;
    trial[a2] = ref[a2] + xcom + xc3 - xc0;
    trial[a2 + 1] = ref[a2 + 1] + ycom + yc3 - yc0;
    trial[a2 + 2] = ref[a2 + 2] + zcom + zc3 - zc0;
  }
}

// settle.ts:198 -- the exact 3x3 impulse solve.
void settle_velocities(const mdb_system_desc* s, const std::vector<Settle>& cl, const double* pos,
                       double* vel) {
  for (const Settle& c : cl) {
    const int a = 3 * c.central, b = 3 * c.first, cc = 3 * c.second;
    const double mA = s->masses[c.central], mB = s->masses[c.first], mC = s->masses[c.second];
    const double iA = mA == 0 ? 0 : 1 / mA, iB = mB == 0 ? 0 : 1 / mB, iC = mC == 0 ? 0 : 1 / mC;
    auto unit = [&](int from, int to) {
      const double x = pos[to] - pos[from], y = pos[to + 1] - pos[from + 1], z = pos[to + 2] - pos[from + 2];
      const double l = std::sqrt(x * x + y * y + z * z);
      return Vec3{x / l, y / l, z / l};
    };
    const Vec3 eAB = unit(a, b), eBC = unit(b, cc), eCA = unit(cc, a);
    auto rel = [&](int from, int to, const Vec3& e) {
      return (vel[to] - vel[from]) * e[0] + (vel[to + 1] - vel[from + 1]) * e[1] +
             (vel[to + 2] - vel[from + 2]) * e[2];
    };
    const double vAB = rel(a, b, eAB), vBC = rel(b, cc, eBC), vCA = rel(cc, a, eCA);
    auto dot = [](const Vec3& p, const Vec3& q) { return p[0] * q[0] + p[1] * q[1] + p[2] * q[2]; };
    const double cA = -dot(eAB, eCA), cB = -dot(eAB, eBC), cC = -dot(eBC, eCA);
    const double s2A = 1 - cA * cA, s2B = 1 - cB * cB, s2C = 1 - cC * cC;
    const double mi = 1 / (mA * mB * mC);
    const double den = (((s2A * mB + s2B * mA) * mC + (s2A * mB * mB + 2 * (cA * cB * cC + 1) * mA * mB +
                                                     s2B * mA * mA)) * mC +
                        s2C * mA * mB * (mA + mB)) * mi;
    const double tab = ((cB * cC * mA - cA * mB - cA * mC) * vCA + (cA * cC * mB - cB * mC - cB * mA) * vBC +
                        (s2C * mA * mA * mB * mB * mi + (mA + mB + mC)) * vAB) / den;
    const double tbc = ((cA * cB * mC - cC * mB - cC * mA) * vCA +
                        (s2A * mB * mB * mC * mC * mi + (mA + mB + mC)) * vBC +
                        (cA * cC * mB - cB * mA - cB * mC) * vAB) / den;
    const double tca = ((s2B * mA * mA * mC * mC * mi + (mA + mB + mC)) * vCA +
                        (cA * cB * mC - cC * mB - cC * mA) * vBC + (cB * cC * mA - cA * mB - cA * mC) * vAB) / den;
    for (int ax = 0; ax < 3; ++ax) {
      vel[a + ax] += (eAB[ax] * tab - eCA[ax] * tca) * iA;
      vel[b + ax] += (eBC[ax] * tbc - eAB[ax] * tab) * iB;
      vel[cc + ax] += (eCA[ax] * tca - eBC[ax] * tbc) * iC;
    }
  }
}

std::vector<double> inverse_masses(const mdb_system_desc* s) {
  std::vector<double> inv(s->n_particles);
  for (int i = 0; i < s->n_particles; ++i) inv[i] = s->masses[i] == 0 ? 0 : 1 / s->masses[i];
  return inv;
}

constexpr int kMaxConstraintIterations = 150;  // constraints.ts:34

// constraints.ts:130 -- Jacobi SHAKE along the reference vectors, all
// iterative constraints together.
bool shake(const mdb_system_desc* s, const std::vector<int>& idx, const double* ref, double* trial,
           double tol) {
  const size_t cnt = idx.size();
  if (cnt == 0) return true;
  const auto inv = inverse_masses(s);
  std::vector<double> rv(3 * cnt), rm(cnt), delta(cnt);
  for (size_t k = 0; k < cnt; ++k) {
    const int c = idx[k], i = 3 * s->constraint_p1[c], j = 3 * s->constraint_p2[c];
    for (int ax = 0; ax < 3; ++ax) rv[3 * k + ax] = ref[i + ax] - ref[j + ax];
    const double sum = inv[s->constraint_p1[c]] + inv[s->constraint_p2[c]];
    rm[k] = sum == 0 ? 0 : 0.5 / sum;
  }
  const double lo = 1 - 2 * tol + tol * tol, hi = 1 + 2 * tol + tol * tol;
  for (int it = 0; it < kMaxConstraintIterations; ++it) {
    size_t conv = 0;
    for (size_t k = 0; k < cnt; ++k) {
      const int c = idx[k], p1 = 3 * s->constraint_p1[c], p2 = 3 * s->constraint_p2[c];
      const double x = trial[p1] - trial[p2], y = trial[p1 + 1] - trial[p2 + 1], z = trial[p1 + 2] - trial[p2 + 2];
      const double l2 = x * x + y * y + z * z, d = s->constraint_distance[c], d2 = d * d;
      const double proj = x * rv[3 * k] + y * rv[3 * k + 1] + z * rv[3 * k + 2];
      delta[k] = proj == 0 ? 0 : rm[k] * (d2 - l2) / proj;
      if (l2 >= lo * d2 && l2 <= hi * d2) conv++;
    }
    if (conv == cnt) return true;
    for (size_t k = 0; k < cnt; ++k) {
      if (delta[k] == 0) continue;
      const int c = idx[k], p1 = s->constraint_p1[c], p2 = s->constraint_p2[c];
      for (int ax = 0; ax < 3; ++ax) {
        const double dr = rv[3 * k + ax] * delta[k];
        trial[3 * p1 + ax] += dr * inv[p1];
        trial[3 * p2 + ax] -= dr * inv[p2];
      }
    }
  }
  return false;
}

// constraints.ts:195 -- RATTLE, dividing by the reference squared length.
bool rattle(const mdb_system_desc* s, const std::vector<int>& idx, const double* pos, double* vel,
            double tol) {
  const size_t cnt = idx.size();
  if (cnt == 0) return true;
  const auto inv = inverse_masses(s);
  std::vector<double> rv(3 * cnt), rl(cnt), rm(cnt), delta(cnt);
  for (size_t k = 0; k < cnt; ++k) {
    const int c = idx[k], i = 3 * s->constraint_p1[c], j = 3 * s->constraint_p2[c];
    for (int ax = 0; ax < 3; ++ax) rv[3 * k + ax] = pos[i + ax] - pos[j + ax];
    rl[k] = rv[3 * k] * rv[3 * k] + rv[3 * k + 1] * rv[3 * k + 1] + rv[3 * k + 2] * rv[3 * k + 2];
    const double sum = inv[s->constraint_p1[c]] + inv[s->constraint_p2[c]];
    rm[k] = sum == 0 ? 0 : 0.5 / sum;
  }
  for (int it = 0; it < kMaxConstraintIterations; ++it) {
    size_t conv = 0;
    for (size_t k = 0; k < cnt; ++k) {
      const int c = idx[k], p1 = 3 * s->constraint_p1[c], p2 = 3 * s->constraint_p2[c];
      const double proj = (vel[p1] - vel[p2]) * rv[3 * k] + (vel[p1 + 1] - vel[p2 + 1]) * rv[3 * k + 1] +
                          (vel[p1 + 2] - vel[p2 + 2]) * rv[3 * k + 2];
      delta[k] = rl[k] == 0 ? 0 : (-2 * rm[k] * proj) / rl[k];
      if (std::fabs(delta[k]) <= tol) conv++;
    }
    if (conv == cnt) return true;
    for (size_t k = 0; k < cnt; ++k) {
      if (delta[k] == 0) continue;
      const int c = idx[k], p1 = s->constraint_p1[c], p2 = s->constraint_p2[c];
      for (int ax = 0; ax < 3; ++ax) {
        const double dr = rv[3 * k + ax] * delta[k];
        vel[3 * p1 + ax] += dr * inv[p1];
        vel[3 * p2 + ax] -= dr * inv[p2];
      }
    }
  }
  return false;
}

// com-motion.ts:48
void remove_com(const mdb_system_desc* s, double* v) {
  double M = 0, px = 0, py = 0, pz = 0;
  for (int i = 0; i < s->n_particles; ++i) {
    const double m = s->masses[i];
    M += m;
    px += m * v[3 * i];
    py += m * v[3 * i + 1];
    pz += m * v[3 * i + 2];
  }
  if (M == 0) return;
  const double vx = px / M, vy = py / M, vz = pz / M;
  for (int i = 0; i < s->n_particles; ++i) {
    if (s->masses[i] == 0) continue;
    v[3 * i] -= vx;
    v[3 * i + 1] -= vy;
    v[3 * i + 2] -= vz;
  }
}

// random.ts:63-111 -- Threefry-2x32 and Box-Muller.
void threefry(uint32_t c0, uint32_t c1, uint32_t k0, uint32_t k1, int rounds, uint32_t* out) {
  static const int rot[8] = {13, 15, 26, 6, 17, 29, 16, 24};
  const uint32_t ks[3] = {k0, k1, 0x1bd11bdau ^ k0 ^ k1};
  uint32_t x0 = c0 + ks[0], x1 = c1 + ks[1];
  for (int r = 0; r < rounds; ++r) {
    x0 += x1;
    const int b = rot[r % 8];
    x1 = ((x1 << b) | (x1 >> (32 - b))) ^ x0;
    if ((r + 1) % 4 == 0) {
      const uint32_t inj = uint32_t((r + 1) / 4);
      x0 += ks[inj % 3];
      x1 += ks[(inj + 1) % 3] + inj;
    }
  }
  out[0] = x0;
  out[1] = x1;
}

double open_unit(uint32_t bits) { return (double(bits >> 9) + 0.5) * std::ldexp(1.0, -23); }

void normal_pair(uint32_t c0, uint32_t c1, uint32_t k0, uint32_t k1, double* out) {
  uint32_t b[2];
  threefry(c0, c1, k0, k1, 20, b);
  const double radius = std::sqrt(-2 * std::log(open_unit(b[0])));
  const double angle = 2 * kPi * open_unit(b[1]);
  out[0] = radius * std::cos(angle);
  out[1] = radius * std::sin(angle);
}

constexpr uint32_t kThermostatDomain = 0x9e3779b9u;  // random.ts:122
constexpr uint32_t kVelocityDomain = 0xbb67ae85u;    // random.ts:154

double thermostat_normal(uint32_t seed, uint32_t step, uint32_t particle, int axis) {
  double p[2];
  normal_pair(particle * 2u + uint32_t(axis >> 1), step, seed, kThermostatDomain, p);
  return p[axis & 1];
}

struct Potential {
  orc_energies e{};
  int status = MDB_OK;
};

Potential evaluate(const mdb_system_desc* s, const double* pos, const double* box_in,
                   const int32_t* grid_in, int threads, bool naive, double* forces) {
  Potential out;
  Box box;
  if (is_reduced(box_in)) std::copy(box_in, box_in + 9, box.begin());
  else box = reduce_box(box_in);
  const int n = s->n_particles;
  if (forces) std::fill(forces, forces + 3 * size_t(n), 0.0);
  orc_energies& e = out.e;
  e.bond = harmonic_bonds(s, pos, forces);
  e.angle = harmonic_angles(s, pos, forces);
  e.torsion = periodic_torsions(s, pos, forces);
  e.restraint = position_restraints(s, pos, box.data(), forces);
  if (s->has_nonbonded) {
    const Vec3 w = perpendicular_widths(box.data());
    if (s->cutoff > 0.5 * std::min({w[0], w[1], w[2]})) {
      out.status = MDB_ERR_CUTOFF_TOO_LARGE_FOR_BOX;
      return out;
    }
    const double alpha = splitting_parameter(s);
    PairAcc acc;
    direct_pairs(s, pos, box.data(), alpha, forces, acc, threads, naive);
    e.direct_coulomb = acc.coulomb;
    e.direct_lj = acc.lj;
    e.pairs_within_cutoff = acc.pairs;
    if (g_virial)
      for (int k = 0; k < 9; ++k) g_virial[k] += acc.vir[k];
    exception_terms(s, pos, box.data(), alpha, forces, e.exclusion_correction, e.exceptions);
    const double volume = box_volume(box.data());
    e.dispersion = s->use_dispersion_correction ? dispersion_correction(s, volume) : 0;
    e.direct_group = e.direct_coulomb + e.direct_lj + e.exclusion_correction + e.exceptions + e.dispersion;
    std::array<int, 3> g;
    if (grid_in && grid_in[0] > 0) g = {grid_in[0], grid_in[1], grid_in[2]};
    else if (s->grid[0] > 0) g = {s->grid[0], s->grid[1], s->grid[2]};
    else g = default_grid(s, box.data(), alpha);
    e.reciprocal_mesh = reciprocal_space(s, pos, box.data(), alpha, g.data(), forces, threads);
    e.self_energy = self_energy(s, alpha);
    e.net_charge = net_charge_correction(s, alpha, volume);
    e.reciprocal_group = e.reciprocal_mesh + e.self_energy + e.net_charge;
    if (g_virial)  // both scale as 1/V
      for (int a = 0; a < 3; ++a) g_virial[4 * a] += e.dispersion + e.net_charge;
  }
  e.potential = e.bond + e.angle + e.torsion + e.restraint + e.direct_group + e.reciprocal_group;
  return out;
}

// molecules.ts:71 -- connected components over constraints, bonds, angles,
// torsions and exceptions, numbered in order of first atom.
std::vector<std::vector<int>> find_molecules(const mdb_system_desc* s) {
  const int n = s->n_particles;
  std::vector<int> parent(n), size(n, 1);
  std::iota(parent.begin(), parent.end(), 0);
  auto find = [&](int x) {
    while (parent[x] != x) { parent[x] = parent[parent[x]]; x = parent[x]; }
    return x;
  };
  auto unite = [&](int a, int b) {
    int x = find(a), y = find(b);
    if (x == y) return;
    if (size[x] < size[y]) std::swap(x, y);
    parent[y] = x;
    size[x] += size[y];
  };
  for (int c = 0; c < s->n_constraints; ++c) unite(s->constraint_p1[c], s->constraint_p2[c]);
  for (int t = 0; t < s->n_bonds; ++t) unite(s->bond_p1[t], s->bond_p2[t]);
  for (int t = 0; t < s->n_angles; ++t) { unite(s->angle_p1[t], s->angle_p2[t]); unite(s->angle_p2[t], s->angle_p3[t]); }
  for (int t = 0; t < s->n_torsions; ++t) {
    unite(s->torsion_p1[t], s->torsion_p2[t]);
    unite(s->torsion_p2[t], s->torsion_p3[t]);
    unite(s->torsion_p3[t], s->torsion_p4[t]);
  }
  if (s->has_nonbonded)
    for (int e = 0; e < s->n_exceptions; ++e) unite(s->exception_p1[e], s->exception_p2[e]);
  std::vector<int> label(n, -1);
  std::vector<std::vector<int>> mols;
  for (int a = 0; a < n; ++a) {
    const int r = find(a);
    if (label[r] < 0) { label[r] = int(mols.size()); mols.push_back({}); }
    mols[label[r]].push_back(a);
  }
  return mols;
}

}  // namespace

// ====================================================================== ABI
extern "C" {

double orc_ewald_alpha(double cutoff, double tolerance) { return ewald_alpha(cutoff, tolerance); }
int32_t orc_pme_minimum_grid(double alpha, double length, double tolerance) {
  return pme_min_grid(alpha, length, tolerance);
}
int32_t orc_smooth_fft_size(int32_t minimum) { return smooth_size(minimum); }

double orc_erf(double x) { return erf_ref(x); }
double orc_erfc(double x) { return erfc_ref(x); }
double orc_erf_derivative(double x) { return erf_derivative(x); }

// fixed-point.ts:55 -- magnitude, round half even on the 2^32 fraction, negate.
int32_t orc_fixed_words(float value, uint32_t* lo, int32_t* hi) {
  const double v = value;
  if (!std::isfinite(v) || std::fabs(v) >= 2147483648.0) return MDB_ERR_RANGE;
  const double m = std::fabs(v), whole = std::floor(m), frac = m - whole;
  const double scaled = frac * 4294967296.0;
  double l = std::floor(scaled);
  const double rem = scaled - l;
  if (rem > 0.5 || (rem == 0.5 && std::fmod(l, 2.0) != 0.0)) l += 1;
  if (v >= 0) {
    *lo = uint32_t(l);
    *hi = int32_t(whole);
  } else if (l == 0) {
    *lo = 0;
    *hi = -int32_t(whole);
  } else {
    *lo = uint32_t(4294967296.0 - l);
    *hi = -int32_t(whole) - 1;
  }
  return MDB_OK;
}

// fixed-point.ts:104 -- the f32 reading, via the magnitude.
float orc_from_fixed_f32(int64_t fixed) {
  const bool neg = fixed < 0;
  const uint64_t m = neg ? uint64_t(-fixed) : uint64_t(fixed);
  const float hi = float(double(m >> 32));
  const float lo = float(float(double(m & 0xffffffffull)) * std::ldexp(1.0f, -32));
  const float v = hi + lo;
  return neg ? -v : v;
}
double orc_from_fixed(int64_t fixed) { return double(fixed) / 4294967296.0; }

void orc_threefry2x32(uint32_t c0, uint32_t c1, uint32_t k0, uint32_t k1, int32_t rounds,
                      uint32_t out[2]) {
  threefry(c0, c1, k0, k1, rounds, out);
}
double orc_open_unit_interval(uint32_t bits) { return open_unit(bits); }
double orc_thermostat_normal(uint32_t seed, uint32_t step, uint32_t particle, int32_t axis) {
  return thermostat_normal(seed, step, particle, axis);
}
double orc_domain_normal(uint32_t domain, uint32_t seed, uint32_t particle, int32_t axis) {
  double p[2];
  normal_pair(particle * 2u + uint32_t(axis >> 1), seed, seed, domain, p);
  return p[axis & 1];
}

int32_t orc_reduce_box(const double in[9], double out[9]) {
  const Box b = reduce_box(in);
  std::copy(b.begin(), b.end(), out);
  return MDB_OK;
}
void orc_perpendicular_widths(const double box[9], double out[3]) {
  const Vec3 w = perpendicular_widths(box);
  out[0] = w[0];
  out[1] = w[1];
  out[2] = w[2];
}
double orc_box_volume(const double box[9]) { return box_volume(box); }
void orc_minimum_image(const double box[9], const double d[3], double out[3]) {
  double x = d[0], y = d[1], z = d[2];
  nearest_image(box, x, y, z);
  out[0] = x;
  out[1] = y;
  out[2] = z;
}
// triclinic.ts:300 -- reduce, then search the 27 neighbouring images.
void orc_nearest_image_by_search(const double box[9], const double d[3], double out[3]) {
  double dx = d[0], dy = d[1], dz = d[2];
  nearest_image(box, dx, dy, dz);
  double best = 1e300;
  for (int i = -1; i <= 1; ++i)
    for (int j = -1; j <= 1; ++j)
      for (int k = -1; k <= 1; ++k) {
        const double x = dx + i * box[0] + j * box[3] + k * box[6];
        const double y = dy + j * box[4] + k * box[7];
        const double z = dz + k * box[8];
        const double q = x * x + y * y + z * z;
        if (q < best) {
          best = q;
          out[0] = x;
          out[1] = y;
          out[2] = z;
        }
      }
}

void orc_bspline(double w, double weights[5], double derivatives[5]) {
  bspline_with_derivatives(w, weights, derivatives);
}
void orc_bspline_moduli(int32_t n, double* out) {
  const auto m = bspline_moduli(n);
  std::copy(m.begin(), m.end(), out);
}

int32_t orc_potential(const mdb_system_desc* sys, const double* positions, const double box[9],
                      const int32_t* grid, int32_t threads, int32_t naive_direct, double* forces,
                      orc_energies* out) {
  Potential p = evaluate(sys, positions, box, grid, threads, naive_direct != 0, forces);
  if (out) *out = p.e;
  return p.status;
}

// The non-excluded pairs whose minimum-image distance lies within `eps` of
// the cutoff, with the force each would put on its first atom if it were
// inside.  The direct-space potential is discontinuous there (nonbonded.ts:330
// truncates erfc-Coulomb and LJ without a shift), so a pair this close to the
// cutoff may be counted by one precision and not by another; the parity tests
// use this list to allow either.  Single-threaded; writes at most `max_pairs`
// and returns how many there are.  No reference counterpart.
int32_t orc_cutoff_shell(const mdb_system_desc* sys, const double* positions, const double box[9],
                         double eps, int32_t max_pairs, int32_t* first, int32_t* second,
                         double* force_on_first, int32_t* inside) {
  const int n = sys->n_particles;
  const double cut = sys->cutoff, lo2 = (cut - eps) * (cut - eps), hi2 = (cut + eps) * (cut + eps);
  const double alpha = splitting_parameter(sys);
  const auto excluded = exclusion_set(sys);
  const Vec3 widths = perpendicular_widths(box);
  int counts[3];
  for (int a = 0; a < 3; ++a) counts[a] = std::max(1, int(std::floor(widths[a] / (cut + eps))));
  const bool naive = counts[0] < 3 || counts[1] < 3 || counts[2] < 3;
  int32_t found = 0;
  auto visit = [&](int i, int j) {
    const int lo = std::min(i, j), hi = std::max(i, j);
    if (excluded.count(uint64_t(lo) * 2097152ull + hi)) return;
    double dx = positions[3 * hi] - positions[3 * lo], dy = positions[3 * hi + 1] - positions[3 * lo + 1],
           dz = positions[3 * hi + 2] - positions[3 * lo + 2];
    nearest_image(box, dx, dy, dz);
    const double r2 = dx * dx + dy * dy + dz * dz;
    if (r2 < lo2 || r2 >= hi2) return;
    if (found < max_pairs) {
      double coulomb, lj;
      const double sc = pair_terms(sys, alpha, lo, hi, r2, coulomb, lj) / std::sqrt(r2);
      first[found] = lo;
      second[found] = hi;
      force_on_first[3 * found] = sc * dx;
      force_on_first[3 * found + 1] = sc * dy;
      force_on_first[3 * found + 2] = sc * dz;
      inside[found] = r2 < cut * cut ? 1 : 0;
    }
    ++found;
  };
  if (naive) {
    for (int i = 0; i < n; ++i)
      for (int j = i + 1; j < n; ++j) visit(i, j);
    return found;
  }
  const int ncell = counts[0] * counts[1] * counts[2];
  const auto inv = inverse_box(box);
  std::vector<int> cell_of(n), start(ncell + 1, 0), order(n);
  auto bucket = [](double f, int div) {
    const double w = f - std::floor(f);
    const int idx = int(std::floor(w * div));
    return idx == div ? div - 1 : idx;
  };
  for (int i = 0; i < n; ++i) {
    const Vec3 f = fractional_of(positions[3 * i], positions[3 * i + 1], positions[3 * i + 2], inv);
    cell_of[i] = (bucket(f[0], counts[0]) * counts[1] + bucket(f[1], counts[1])) * counts[2] + bucket(f[2], counts[2]);
    start[cell_of[i] + 1]++;
  }
  for (int c = 0; c < ncell; ++c) start[c + 1] += start[c];
  std::vector<int> cur(start.begin(), start.end() - 1);
  for (int i = 0; i < n; ++i) order[cur[cell_of[i]]++] = i;
  for (int cell = 0; cell < ncell; ++cell) {
    const int cz = cell % counts[2], cy = (cell / counts[2]) % counts[1], cx = cell / (counts[1] * counts[2]);
    for (int ddx = -1; ddx <= 1; ++ddx)
      for (int ddy = -1; ddy <= 1; ++ddy)
        for (int ddz = -1; ddz <= 1; ++ddz) {
          const int nb = (((cx + ddx + counts[0]) % counts[0]) * counts[1] + (cy + ddy + counts[1]) % counts[1]) *
                             counts[2] + (cz + ddz + counts[2]) % counts[2];
          if (nb < cell) continue;
          for (int a = start[cell]; a < start[cell + 1]; ++a)
            for (int b = nb == cell ? a + 1 : start[nb]; b < start[nb + 1]; ++b) visit(order[a], order[b]);
        }
  }
  return found;
}

int32_t orc_potential_virial(const mdb_system_desc* sys, const double* positions, const double box[9],
                             const int32_t* grid, int32_t threads, double* forces, orc_energies* out,
                             double virial[9]) {
  std::vector<double> scratch;
  if (!forces) {
    scratch.assign(3 * size_t(sys->n_particles), 0.0);
    forces = scratch.data();
  }
  std::fill(virial, virial + 9, 0.0);
  g_virial = virial;
  Potential p = evaluate(sys, positions, box, grid, threads, false, forces);
  g_virial = nullptr;
  if (out) *out = p.e;
  return p.status;
}

// The barostat screening network (no reference counterpart): inputs -> 64
// tanh -> 64 tanh -> 1, parameters W1[64][16], b1[64], W2[64][64], b2[64],
// w3[64], b3, in f64; the mean-squared-error loss over the first min(n, 128)
// samples and its gradient by reverse accumulation.
int32_t orc_mlp_gradient(const float* params, const float* x, const float* t, int32_t n, double* grad,
                         double* loss) {
  constexpr int I = 16, H = 64;
  constexpr int oB1 = H * I, oW2 = oB1 + H, oB2 = oW2 + H * H, oW3 = oB2 + H, oB3 = oW3 + H, P = oB3 + 1;
  if (!params || !x || !t || !grad || !loss || n <= 0) return MDB_ERR_INVALID_ARGUMENT;
  const int B = std::min(n, 128);
  std::vector<double> w(params, params + P);
  std::fill(grad, grad + P, 0.0);
  double l = 0;
  for (int b = 0; b < B; ++b) {
    const float* in = x + size_t(b) * I;
    double h1[H], h2[H];
    for (int j = 0; j < H; ++j) {
      double a = w[oB1 + j];
      for (int k = 0; k < I; ++k) a += w[j * I + k] * in[k];
      h1[j] = std::tanh(a);
    }
    for (int j = 0; j < H; ++j) {
      double a = w[oB2 + j];
      for (int k = 0; k < H; ++k) a += w[oW2 + j * H + k] * h1[k];
      h2[j] = std::tanh(a);
    }
    double y = w[oB3];
    for (int j = 0; j < H; ++j) y += w[oW3 + j] * h2[j];
    const double e = y - t[b];
    l += e * e;
    const double dy = 2 * e / B;
    double d2[H], d1[H];
    for (int j = 0; j < H; ++j) {
      grad[oW3 + j] += dy * h2[j];
      d2[j] = dy * w[oW3 + j] * (1 - h2[j] * h2[j]);
    }
    grad[oB3] += dy;
    for (int k = 0; k < H; ++k) {
      double a = 0;
      for (int j = 0; j < H; ++j) a += w[oW2 + j * H + k] * d2[j];
      d1[k] = a * (1 - h1[k] * h1[k]);
    }
    for (int j = 0; j < H; ++j) {
      for (int k = 0; k < H; ++k) grad[oW2 + j * H + k] += d2[j] * h1[k];
      grad[oB2 + j] += d2[j];
      for (int k = 0; k < I; ++k) grad[j * I + k] += d1[j] * in[k];
      grad[oB1 + j] += d1[j];
    }
  }
  *loss = l / B;
  return MDB_OK;
}

// ewald.ts:82 -- half the lattice, doubled; k-space only.
int32_t orc_ewald_reciprocal(const mdb_system_desc* s, const double* pos, const double box[9],
                             double alpha, int32_t kmax, double* forces, double* energy) {
  const auto inv = inverse_box(box);
  const double volume = box_volume(box);
  const double pref = (2 * kPi * kOne4PiEps0) / volume;
  const double q4 = 1 / (4 * alpha * alpha);
  const int n = s->n_particles;
  double e = 0;
  if (forces) std::fill(forces, forces + 3 * size_t(n), 0.0);
  for (int ma = 0; ma <= kmax; ++ma)
    for (int mb = ma == 0 ? 0 : -kmax; mb <= kmax; ++mb)
      for (int mc = (ma == 0 && mb == 0) ? 1 : -kmax; mc <= kmax; ++mc) {
        const Vec3 k = reciprocal_vector(ma, mb, mc, inv);
        const double k2 = k[0] * k[0] + k[1] * k[1] + k[2] * k[2];
        if (k2 == 0) continue;
        const double w = std::exp(-k2 * q4) / k2;
        if (w == 0) continue;
        double re = 0, im = 0;
        for (int i = 0; i < n; ++i) {
          const double ph = k[0] * pos[3 * i] + k[1] * pos[3 * i + 1] + k[2] * pos[3 * i + 2];
          re += s->charge[i] * std::cos(ph);
          im += s->charge[i] * std::sin(ph);
        }
        e += 2 * pref * w * (re * re + im * im);
        if (forces) {
          const double sc = 4 * pref * w;
          for (int i = 0; i < n; ++i) {
            const double ph = k[0] * pos[3 * i] + k[1] * pos[3 * i + 1] + k[2] * pos[3 * i + 2];
            const double t = sc * s->charge[i] * (std::sin(ph) * re - std::cos(ph) * im);
            forces[3 * i] += t * k[0];
            forces[3 * i + 1] += t * k[1];
            forces[3 * i + 2] += t * k[2];
          }
        }
      }
  *energy = e;
  return MDB_OK;
}

int32_t orc_split_counts(const mdb_system_desc* sys, int32_t* settle_clusters,
                         int32_t* iterative_clusters, int32_t* largest_atoms,
                         int32_t* largest_constraints) {
  const Split sp = split_constraints(sys);
  *settle_clusters = int32_t(sp.settle.size());
  *iterative_clusters = int32_t(sp.clusters.size());
  *largest_atoms = sp.largest_atoms;
  *largest_constraints = sp.largest_constraints;
  return sp.too_large ? MDB_ERR_CLUSTER_TOO_LARGE : MDB_OK;
}

// kinetic.ts:106
double orc_degrees_of_freedom(const mdb_system_desc* s) {
  int moving = 0;
  for (int i = 0; i < s->n_particles; ++i) moving += s->masses[i] > 0;
  return 3.0 * moving - s->n_constraints - (s->com_frequency > 0 ? 3 : 0);
}

// kinetic.ts:31
double orc_kinetic_energy(const mdb_system_desc* s, const double* v) {
  double t = 0;
  for (int i = 0; i < s->n_particles; ++i) {
    const double m = s->masses[i];
    if (m <= 0) continue;
    t += m * (v[3 * i] * v[3 * i] + v[3 * i + 1] * v[3 * i + 1] + v[3 * i + 2] * v[3 * i + 2]);
  }
  return 0.5 * t;
}

void orc_remove_com(const mdb_system_desc* sys, double* velocities) { remove_com(sys, velocities); }

int32_t orc_constrain_positions(const mdb_system_desc* sys, const double* reference, double* trial,
                                double tolerance) {
  const Split sp = split_constraints(sys);
  settle_positions(sys, sp.settle, reference, trial);
  return shake(sys, sp.iterative, reference, trial, tolerance) ? MDB_OK : MDB_ERR_NOT_CONVERGED;
}

int32_t orc_constrain_velocities(const mdb_system_desc* sys, const double* positions,
                                 double* velocities, double tolerance) {
  const Split sp = split_constraints(sys);
  settle_velocities(sys, sp.settle, positions, velocities);
  return rattle(sys, sp.iterative, positions, velocities, tolerance) ? MDB_OK : MDB_ERR_NOT_CONVERGED;
}

// The loop of src/gpu/loop.ts:715-751 in f64: COM on removesOnStep, forces,
// then one integrator step (src/reference/integrator.ts:68, :140).
int32_t orc_run(const mdb_system_desc* s, double* pos, double* vel, const double box[9],
                const orc_step_options* o, int64_t* step, int64_t steps) {
  const int n = s->n_particles;
  const Split sp = split_constraints(s);
  if (sp.too_large) return MDB_ERR_CLUSTER_TOO_LARGE;
  const auto inv = inverse_masses(s);
  std::vector<double> f(3 * size_t(n)), trial(3 * size_t(n)), old(3 * size_t(n));
  const double dt = o->time_step, half = 0.5 * dt;
  const double kT = kBoltzmann * o->temperature;
  const double vs = std::exp(-dt * o->friction), ns = std::sqrt(1 - vs * vs);
  int32_t status = MDB_OK;
  for (int64_t k = 0; k < steps; ++k) {
    const int64_t st = *step;
    if (s->com_frequency > 0 && st % s->com_frequency == 0) remove_com(s, vel);
    Potential p = evaluate(s, pos, box, o->grid, o->threads, false, f.data());
    if (p.status != MDB_OK) return p.status;
    if (o->integrator == MDB_INTEGRATOR_VERLET) {
      std::copy(pos, pos + 3 * n, old.begin());
      for (int i = 0; i < n; ++i)
        for (int ax = 0; ax < 3; ++ax) {
          const int a = 3 * i + ax;
          if (inv[i] == 0) { trial[a] = old[a]; continue; }
          vel[a] += inv[i] * f[a] * dt;
          trial[a] = old[a] + vel[a] * dt;
        }
      settle_positions(s, sp.settle, old.data(), trial.data());
      if (!shake(s, sp.iterative, old.data(), trial.data(), o->constraint_tolerance)) status = MDB_ERR_NOT_CONVERGED;
      for (int i = 0; i < n; ++i) {
        if (inv[i] == 0) continue;
        for (int ax = 0; ax < 3; ++ax) {
          const int a = 3 * i + ax;
          vel[a] = (trial[a] - old[a]) / dt;
          pos[a] = trial[a];
        }
      }
    } else {
      for (int i = 0; i < n; ++i) {
        if (inv[i] == 0) continue;
        for (int ax = 0; ax < 3; ++ax) vel[3 * i + ax] += dt * inv[i] * f[3 * i + ax];
      }
      settle_velocities(s, sp.settle, pos, vel);
      if (!rattle(s, sp.iterative, pos, vel, o->constraint_tolerance)) status = MDB_ERR_NOT_CONVERGED;
      std::copy(pos, pos + 3 * n, trial.begin());
      for (int i = 0; i < n; ++i) {
        if (inv[i] == 0) continue;
        const double noise = ns * std::sqrt(kT * inv[i]);
        for (int ax = 0; ax < 3; ++ax) {
          const int a = 3 * i + ax;
          trial[a] += vel[a] * half;
          vel[a] = vs * vel[a] +
                   (noise == 0 ? 0 : noise * thermostat_normal(o->seed, uint32_t(st), uint32_t(i), ax));
          trial[a] += vel[a] * half;
        }
      }
      std::copy(trial.begin(), trial.end(), old.begin());  // `unconstrained`
      settle_positions(s, sp.settle, pos, trial.data());
      if (!shake(s, sp.iterative, pos, trial.data(), o->constraint_tolerance)) status = MDB_ERR_NOT_CONVERGED;
      for (int i = 0; i < n; ++i) {
        if (inv[i] == 0) continue;
        for (int ax = 0; ax < 3; ++ax) {
          const int a = 3 * i + ax;
          vel[a] += (trial[a] - old[a]) / dt;
          pos[a] = trial[a];
        }
      }
    }
    *step = st + 1;
  }
  return status;
}

int32_t orc_molecule_count(const mdb_system_desc* sys) { return int32_t(find_molecules(sys).size()); }

// barostat.ts:148 -- unweighted centroid, translated rigidly.
void orc_scale_molecules(const mdb_system_desc* sys, double* pos, double scale) {
  for (const auto& m : find_molecules(sys)) {
    double c[3] = {0, 0, 0};
    for (int a : m)
      for (int ax = 0; ax < 3; ++ax) c[ax] += pos[3 * a + ax];
    double off[3];
    for (int ax = 0; ax < 3; ++ax) {
      const double mean = c[ax] / double(m.size());
      off[ax] = scale * mean - mean;
    }
    for (int a : m)
      for (int ax = 0; ax < 3; ++ax) pos[3 * a + ax] += off[ax];
  }
}

// velocities.ts:78 -- Maxwell-Boltzmann on VELOCITY_DOMAIN, then projected.
void orc_velocities_at_temperature(const mdb_system_desc* s, const double* positions,
                                   double temperature, uint32_t seed, double* out) {
  const double kT = kBoltzmann * temperature;
  for (int i = 0; i < s->n_particles; ++i) {
    const double m = s->masses[i];
    for (int ax = 0; ax < 3; ++ax) {
      out[3 * i + ax] = m == 0 ? 0 : std::sqrt(kT / m) * orc_domain_normal(kVelocityDomain, seed, i, ax);
    }
  }
  const Split sp = split_constraints(s);
  settle_velocities(s, sp.settle, positions, out);
  rattle(s, sp.iterative, positions, out, 1e-5);
}

}  // extern "C"
