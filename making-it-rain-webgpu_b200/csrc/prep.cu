// prep.cpp -- host-side preparation of one system (see prep.h).
#include "prep.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <numeric>
#include <sstream>

namespace mdb {
namespace {

constexpr double kPi = 3.14159265358979323846;

// src/engine/units.ts:53 -- alpha = sqrt(-ln(2 tol)) / rc
double ewald_alpha(double cutoff, double tol) { return std::sqrt(-std::log(2 * tol)) / cutoff; }

// units.ts:65 -- ceil(2 alpha L / (3 tol^0.2)), at least 6
int pme_minimum_grid(double alpha, double length, double tol) {
  return std::max(6, int(std::ceil(2 * alpha * length / (3 * std::pow(tol, 0.2)))));
}

// units.ts:78 -- the next 2/3/5/7-smooth size
int smooth_size(int minimum) {
  for (int n = std::max(1, minimum);; ++n) {
    int r = n;
    for (int p : {2, 3, 5, 7})
      while (r % p == 0) r /= p;
    if (r == 1) return n;
  }
}

template <typename T>
bool index_ok(const T* idx, int count, int n) {
  if (count == 0) return true;
  if (!idx) return false;
  for (int i = 0; i < count; ++i)
    if (idx[i] < 0 || idx[i] >= n) return false;
  return true;
}

int find_root(std::vector<int>& parent, int x) {
  while (parent[x] != x) {
    parent[x] = parent[parent[x]];
    x = parent[x];
  }
  return x;
}

}  // namespace

// src/reference/triclinic.ts:93 -- c against b, then c and b against a, ties to even.
bool reduce_box(const double* in, double* v) {
  std::memcpy(v, in, 9 * sizeof(double));
  auto by = [](double ratio) {
    const double nearest = std::round(ratio);
    if (std::fabs(ratio - std::trunc(ratio)) == 0.5 && std::fmod(std::fabs(nearest), 2.0) != 0.0)
      return nearest - (ratio > 0 ? 1.0 : -1.0);
    return nearest;
  };
  auto sub = [&](int t, int s, double k) {
    for (int i = 0; i < 3; ++i) v[t * 3 + i] -= k * v[s * 3 + i];
  };
  sub(2, 1, by(v[7] / v[4]));
  sub(2, 0, by(v[6] / v[0]));
  sub(1, 0, by(v[3] / v[0]));
  const double tol = 1e-9;
  return std::fabs(v[1]) <= tol && std::fabs(v[2]) <= tol && std::fabs(v[5]) <= tol && v[0] > 0 && v[4] > 0 &&
         v[8] > 0;
}

double box_volume(const double* b) {
  return std::fabs(b[0] * (b[4] * b[8] - b[5] * b[7]) - b[1] * (b[3] * b[8] - b[5] * b[6]) +
                   b[2] * (b[3] * b[7] - b[4] * b[6]));
}

// triclinic.ts:38 -- volume over face area
void perpendicular_widths(const double* b, double* out) {
  auto cross_norm = [](const double* u, const double* v) {
    const double x = u[1] * v[2] - u[2] * v[1], y = u[2] * v[0] - u[0] * v[2], z = u[0] * v[1] - u[1] * v[0];
    return std::sqrt(x * x + y * y + z * z);
  };
  const double vol = box_volume(b);
  out[0] = vol / cross_norm(b + 3, b + 6);
  out[1] = vol / cross_norm(b + 6, b);
  out[2] = vol / cross_norm(b, b + 3);
}

// triclinic.ts:394 -- lower-triangular inverse, f = r . M
void inverse_box(const double* b, double* m) {
  const double ax = b[0], bx = b[3], by = b[4], cx = b[6], cy = b[7], cz = b[8];
  const double v[9] = {1 / ax, 0, 0, -bx / (ax * by), 1 / by, 0, ((bx * cy) / (by * cz) - cx / cz) / ax,
                       -cy / (by * cz), 1 / cz};
  std::memcpy(m, v, sizeof(v));
}

// src/reference/forces/bspline.ts:102 -- |b(m)|^2 of the order-5 spline
std::vector<double> bspline_moduli(int n) {
  // order-5 cardinal B-spline at its integer knots: 1/24, 11/24, 11/24, 1/24
  const double knots[5] = {1.0 / 24, 11.0 / 24, 11.0 / 24, 1.0 / 24, 0.0};
  std::vector<double> mod(n);
  for (int m = 0; m < n; ++m) {
    double re = 0, im = 0;
    for (int k = 0; k < 5 && k < n; ++k) {
      const double a = 2 * kPi * double(m) * k / n;
      re += knots[k] * std::cos(a);
      im += knots[k] * std::sin(a);
    }
    mod[m] = re * re + im * im;
  }
  for (int m = 0; m < n; ++m)
    if (mod[m] < 1e-7) mod[m] = 0.5 * (mod[(m - 1 + n) % n] + mod[(m + 1) % n]);
  return mod;
}

// Stages for the shared-memory Stockham FFT: radix 4 where it divides, then
// 7, 5, 3, 2.  False for a length that is not 2/3/5/7-smooth.
bool plan_radices(int n, int* radices, int* count) {
  int c = 0, r = n;
  while (r % 4 == 0 && c < kMaxRadices) { radices[c++] = 4; r /= 4; }
  for (int p : {7, 5, 3, 2})
    while (r % p == 0 && c < kMaxRadices) { radices[c++] = p; r /= p; }
  *count = c;
  return r == 1;
}

// nonbonded.ts:107 (dispersion, grouped by class), :594 (net charge), :610 (self)
void update_box_constants(HostSystem& h) {
  const double vol = box_volume(h.box.data());
  if (h.dispersion && h.n > 0) {
    const double rc = h.cutoff, pairs = double(h.n) * (h.n + 1) / 2;
    h.dispersion_energy = (8 * kPi * double(h.n) * h.n / vol) *
                          ((h.dispersion_sums[0] / pairs) / (9 * std::pow(rc, 9)) -
                           (h.dispersion_sums[1] / pairs) / (3 * std::pow(rc, 3)));
  } else {
    h.dispersion_energy = 0;
  }
  h.net_charge_energy = h.has_nonbonded
                            ? (-kPi * h.charge_sum * h.charge_sum * kOne4PiEps0) / (2 * h.alpha * h.alpha * vol)
                            : 0;
}

int prepare_system(const mdb_system_desc& in, const mdb_state_desc& state, const mdb_run_options& opt,
                   HostSystem& h, std::string& error) {
  std::ostringstream msg;
  const int n = in.n_particles;
  if (n <= 0 || !in.masses || !state.positions) {
    error = "a system needs particles, masses and positions";
    return MDB_ERR_INVALID_ARGUMENT;
  }
  h.n = n;
  h.mass.assign(in.masses, in.masses + n);
  for (double m : h.mass)
    if (!(m >= 0) || !std::isfinite(m)) {
      error = "masses must be finite and non-negative";
      return MDB_ERR_INVALID_ARGUMENT;
    }
  for (int i = 0; i < 3 * n; ++i)
    if (!std::isfinite(state.positions[i]) || std::fabs(state.positions[i]) > 1.0e6) {
      error = "positions must be finite and inside the fixed-point range";
      return MDB_ERR_RANGE;
    }
  // The state's box wins over the system's default, as OpenMM's context does.
  const double* raw_box = state.box;
  bool zero = true;
  for (int i = 0; i < 9; ++i) zero &= raw_box[i] == 0;
  if (zero) raw_box = in.box;
  if (!reduce_box(raw_box, h.box.data())) {
    error = "the periodic box is degenerate (a, b, c must span a positive volume)";
    return MDB_ERR_INVALID_ARGUMENT;
  }

  // constraints
  if (!index_ok(in.constraint_p1, in.n_constraints, n) || !index_ok(in.constraint_p2, in.n_constraints, n) ||
      (in.n_constraints > 0 && !in.constraint_distance)) {
    error = "constraint indices out of range";
    return MDB_ERR_INVALID_ARGUMENT;
  }
  h.cp1.assign(in.constraint_p1, in.constraint_p1 + in.n_constraints);
  h.cp2.assign(in.constraint_p2, in.constraint_p2 + in.n_constraints);
  h.cdist.assign(in.constraint_distance, in.constraint_distance + in.n_constraints);

  if (!in.has_nonbonded) {
    error = "this engine runs PME systems; the System has no NonbondedForce";
    return MDB_ERR_UNSUPPORTED_FORCE;
  }
  h.has_nonbonded = true;
  if (!in.charge || !in.sigma || !in.epsilon || !(in.cutoff > 0) || !(in.ewald_tolerance > 0)) {
    error = "NonbondedForce needs per-particle parameters, a cutoff and an Ewald tolerance";
    return MDB_ERR_INVALID_ARGUMENT;
  }
  h.charge.assign(in.charge, in.charge + n);
  h.sigma.assign(in.sigma, in.sigma + n);
  h.epsilon.assign(in.epsilon, in.epsilon + n);
  h.cutoff = in.cutoff;
  h.tolerance = in.ewald_tolerance;
  h.dispersion = in.use_dispersion_correction != 0;
  double widths[3];
  perpendicular_widths(h.box.data(), widths);
  const double maxcut = 0.5 * std::min({widths[0], widths[1], widths[2]});
  if (h.cutoff > maxcut) {
    msg << "a " << h.cutoff << " nm cutoff does not fit this box: its narrowest perpendicular width is "
        << 2 * maxcut << " nm, so the minimum image is only exact below " << maxcut << " nm";
    error = msg.str();
    return MDB_ERR_CUTOFF_TOO_LARGE_FOR_BOX;
  }
  h.alpha = in.alpha != 0 ? in.alpha : ewald_alpha(h.cutoff, h.tolerance);
  // The pair kernel's screened-Coulomb polynomial is fitted for alpha r <= 3.6,
  // which covers Ewald tolerances down to about 1e-6.
  if (!(h.alpha > 0) || h.alpha * h.cutoff > 3.6) {
    msg << "alpha * cutoff = " << h.alpha * h.cutoff
        << " exceeds 3.6, the range the pair kernel's erfc is fitted on (Ewald tolerance below ~1e-6)";
    error = msg.str();
    return MDB_ERR_INVALID_ARGUMENT;
  }
  for (int k = 0; k < 3; ++k) {
    int g = opt.mesh[k] > 0 ? opt.mesh[k] : in.grid[k];
    // potential.ts:79 -- the mesh from the box *diagonal*
    if (g <= 0) g = smooth_size(pme_minimum_grid(h.alpha, h.box[k * 4], h.tolerance));
    int rad[kMaxRadices], nr = 0;
    if (!plan_radices(g, rad, &nr)) {
      msg << "mesh size " << g << " is not 2/3/5/7-smooth, so the transform cannot do it";
      error = msg.str();
      return MDB_ERR_NOT_SMOOTH;
    }
    if (g > 512) {
      msg << "mesh size " << g << " exceeds the 512 points per axis one CTA transforms";
      error = msg.str();
      return MDB_ERR_INVALID_ARGUMENT;
    }
    // The order-5 spline of an atom touches 5 consecutive mesh points, wrapped
    // once into the mesh; an axis shorter than that would wrap past its end.
    if (g < kPmeOrder) {
      msg << "mesh size " << g << " is below the " << kPmeOrder << " points the order-" << kPmeOrder
          << " B-spline spans";
      error = msg.str();
      return MDB_ERR_INVALID_ARGUMENT;
    }
    h.grid[k] = g;
  }

  // exceptions
  const int ne = in.n_exceptions;
  if (!index_ok(in.exception_p1, ne, n) || !index_ok(in.exception_p2, ne, n) ||
      (ne > 0 && (!in.exception_charge_prod || !in.exception_sigma || !in.exception_epsilon))) {
    error = "exception indices out of range";
    return MDB_ERR_INVALID_ARGUMENT;
  }
  h.ep1.assign(in.exception_p1, in.exception_p1 + ne);
  h.ep2.assign(in.exception_p2, in.exception_p2 + ne);
  h.eqq.assign(in.exception_charge_prod, in.exception_charge_prod + ne);
  h.esig.assign(in.exception_sigma, in.exception_sigma + ne);
  h.eeps.assign(in.exception_epsilon, in.exception_epsilon + ne);
  for (int e = 0; e < ne; ++e)
    if (h.ep1[e] == h.ep2[e]) {
      error = "an exception joins a particle to itself";
      return MDB_ERR_INVALID_ARGUMENT;
    }

  // bonded terms (local indices; the engine adds offsets)
  if (!index_ok(in.bond_p1, in.n_bonds, n) || !index_ok(in.bond_p2, in.n_bonds, n) ||
      !index_ok(in.angle_p1, in.n_angles, n) || !index_ok(in.angle_p2, in.n_angles, n) ||
      !index_ok(in.angle_p3, in.n_angles, n) || !index_ok(in.torsion_p1, in.n_torsions, n) ||
      !index_ok(in.torsion_p2, in.n_torsions, n) || !index_ok(in.torsion_p3, in.n_torsions, n) ||
      !index_ok(in.torsion_p4, in.n_torsions, n) || !index_ok(in.restraint_particle, in.n_restraints, n)) {
    error = "bonded-term indices out of range";
    return MDB_ERR_INVALID_ARGUMENT;
  }
  for (int t = 0; t < in.n_bonds; ++t) {
    const double r0sq = in.bond_length[t] * in.bond_length[t];
    const float r0sq_hi = float(r0sq);
    h.bonds.push_back({in.bond_p1[t], in.bond_p2[t], 0, float(in.bond_length[t]), float(in.bond_k[t]), r0sq_hi,
                       float(r0sq - double(r0sq_hi))});
  }
  for (int t = 0; t < in.n_angles; ++t)
    h.angles.push_back({in.angle_p1[t], in.angle_p2[t], in.angle_p3[t], 0, float(in.angle_theta[t]),
                        float(in.angle_k[t])});
  for (int t = 0; t < in.n_torsions; ++t)
    h.torsions.push_back({in.torsion_p1[t], in.torsion_p2[t], in.torsion_p3[t], in.torsion_p4[t], 0,
                          in.torsion_periodicity[t], float(in.torsion_phase[t]), float(in.torsion_k[t])});
  for (int t = 0; t < in.n_restraints; ++t) {
    h.rparticle.push_back(in.restraint_particle[t]);
    h.rk.push_back(in.restraint_k[t]);
    h.rx0.push_back(in.restraint_x0[t]);
    h.ry0.push_back(in.restraint_y0[t]);
    h.rz0.push_back(in.restraint_z0[t]);
  }
  h.com_frequency = in.com_frequency;
  h.barostat_frequency = in.barostat_frequency;
  h.barostat_pressure = in.barostat_pressure;
  h.barostat_temperature = in.barostat_temperature;

  // ---- constraint split: src/engine/constraint-clusters.ts:93 ----
  const int nc = in.n_constraints;
  std::vector<int> ccount(n, 0);
  std::vector<char> live(nc, 0);
  for (int c = 0; c < nc; ++c) {
    if (h.mass[h.cp1[c]] == 0 && h.mass[h.cp2[c]] == 0) continue;
    live[c] = 1;
    ccount[h.cp1[c]]++;
    ccount[h.cp2[c]]++;
  }
  // partners of atoms whose two ends both hold exactly two constraints,
  // distances compared after f32 rounding as OpenMM does (:88-92)
  std::vector<std::vector<std::pair<int, float>>> partner(n);
  auto link = [&](int a, int b, float dd) {
    for (auto& p : partner[a])
      if (p.first == b) { p.second = dd; return; }
    partner[a].push_back({b, dd});
  };
  for (int c = 0; c < nc; ++c) {
    if (!live[c]) continue;
    const int a = h.cp1[c], b = h.cp2[c];
    if (ccount[a] == 2 && ccount[b] == 2) {
      link(a, b, float(h.cdist[c]));
      link(b, a, float(h.cdist[c]));
    }
  }
  auto partner_distance = [&](int a, int b) -> float {
    for (auto& p : partner[a])
      if (p.first == b) return p.second;
    return -1.f;
  };
  std::vector<char> in_settle(n, 0);
  for (int a = 0; a < n; ++a) {
    if (partner[a].size() != 2) continue;
    const int p2 = partner[a][0].first, p3 = partner[a][1].first;
    if (partner[p2].size() != 2 || partner[p3].size() != 2 || partner_distance(p2, p3) < 0) continue;
    if (!(a < p2 && a < p3)) continue;
    const float d12 = partner_distance(a, p2), d13 = partner_distance(a, p3), d23 = partner_distance(p2, p3);
    SettleHost s{};
    if (d12 == d13) s = {a, p2, p3, d12, d23};
    else if (d12 == d23) s = {p2, a, p3, d12, d13};
    else if (d13 == d23) s = {p3, a, p2, d13, d12};
    else continue;
    h.settle.push_back(s);
    in_settle[a] = in_settle[p2] = in_settle[p3] = 1;
  }
  std::vector<int> iterative;
  for (int c = 0; c < nc; ++c)
    if (live[c] && !in_settle[h.cp1[c]]) iterative.push_back(c);
  std::vector<int> parent(n);
  std::iota(parent.begin(), parent.end(), 0);
  for (int c : iterative) {
    const int a = find_root(parent, h.cp1[c]), b = find_root(parent, h.cp2[c]);
    if (a != b) parent[a] = b;
  }
  std::map<int, int> cluster_of_root;
  for (int c : iterative) {
    const int r = find_root(parent, h.cp1[c]);
    auto it = cluster_of_root.find(r);
    int idx;
    if (it == cluster_of_root.end()) {
      idx = int(h.shake.size());
      cluster_of_root[r] = idx;
      h.shake.push_back({});
    } else {
      idx = it->second;
    }
    ShakeHost& cl = h.shake[idx];
    cl.constraints.push_back(c);
    for (int p : {h.cp1[c], h.cp2[c]})
      if (std::find(cl.atoms.begin(), cl.atoms.end(), p) == cl.atoms.end()) cl.atoms.push_back(p);
  }
  std::vector<char> in_unit(n, 0);
  for (const auto& s : h.settle) in_unit[s.central] = in_unit[s.first] = in_unit[s.second] = 1;
  for (auto& cl : h.shake) {
    std::sort(cl.atoms.begin(), cl.atoms.end());
    if (int(cl.atoms.size()) > kMaxClusterAtoms || int(cl.constraints.size()) > kMaxClusterConstraints) {
      msg << "a constraint cluster has " << cl.atoms.size() << " atoms and " << cl.constraints.size()
          << " constraints, beyond the " << kMaxClusterAtoms << " and " << kMaxClusterConstraints
          << " one GPU thread holds; rebuild with constraints=HBonds";
      error = msg.str();
      return MDB_ERR_CLUSTER_TOO_LARGE;
    }
    for (int a : cl.atoms) in_unit[a] = 1;
  }
  for (int a = 0; a < n; ++a)
    if (!in_unit[a]) h.free_atoms.push_back(a);

  // ---- molecules: src/engine/molecules.ts:71 ----
  std::iota(parent.begin(), parent.end(), 0);
  auto unite = [&](int a, int b) {
    a = find_root(parent, a);
    b = find_root(parent, b);
    if (a != b) parent[std::max(a, b)] = std::min(a, b);
  };
  for (int c = 0; c < nc; ++c) unite(h.cp1[c], h.cp2[c]);
  for (const auto& b : h.bonds) unite(b.a, b.b);
  for (const auto& a : h.angles) { unite(a.a, a.b); unite(a.b, a.c); }
  for (const auto& t : h.torsions) { unite(t.a, t.b); unite(t.b, t.c); unite(t.c, t.d); }
  for (int e = 0; e < ne; ++e) unite(h.ep1[e], h.ep2[e]);
  std::map<int, int> mol_of_root;
  for (int a = 0; a < n; ++a) {
    const int r = find_root(parent, a);
    auto it = mol_of_root.find(r);
    if (it == mol_of_root.end()) {
      mol_of_root[r] = int(h.molecules.size());
      h.molecules.push_back({a});
    } else {
      h.molecules[it->second].push_back(a);
    }
  }

  // ---- host constants ----
  int moving = 0;
  h.total_mass = 0;
  for (int a = 0; a < n; ++a) {
    moving += h.mass[a] > 0;
    h.total_mass += h.mass[a];
  }
  h.dof = 3.0 * moving - nc - (h.com_frequency > 0 ? 3 : 0);  // kinetic.ts:106
  double q2 = 0;
  h.charge_sum = 0;
  for (int a = 0; a < n; ++a) {
    q2 += h.charge[a] * h.charge[a];
    h.charge_sum += h.charge[a];
  }
  h.self_energy = -kOne4PiEps0 * h.alpha * q2 / std::sqrt(kPi);
  if (h.dispersion) {
    std::map<std::pair<double, double>, double> classes;
    for (int a = 0; a < n; ++a) classes[{h.sigma[a], h.epsilon[a]}] += 1;
    std::vector<std::pair<std::pair<double, double>, double>> cl(classes.begin(), classes.end());
    double s6 = 0, s12 = 0;
    for (size_t c = 0; c < cl.size(); ++c)
      for (size_t d = c; d < cl.size(); ++d) {
        const double sg = 0.5 * (cl[c].first.first + cl[d].first.first);
        const double ep = std::sqrt(cl[c].first.second * cl[d].first.second);
        const double sg6 = std::pow(sg, 6);
        const double mult = c == d ? cl[c].second * (cl[c].second + 1) / 2 : cl[c].second * cl[d].second;
        s6 += mult * ep * sg6;
        s12 += mult * ep * sg6 * sg6;
      }
    h.dispersion_sums = {s12, s6};
  }
  update_box_constants(h);
  return MDB_OK;
}

}  // namespace mdb
