// prep.h -- host-side preparation of one system: validation, the constraint
// split, integration units, exclusions, molecules, alpha and the mesh, and the
// box-dependent host constants.  Mirrors `StepLoop.fromParsed`
// (src/gpu/loop.ts:278-532) and the reference helpers it calls.
#pragma once
#include <array>
#include <string>
#include <vector>

#include "../../include/mdb.h"
#include "device_state.h"

namespace mdb {

struct SettleHost { int central, first, second; float d1, d2; };
struct ShakeHost { std::vector<int> atoms; std::vector<int> constraints; };

struct HostSystem {
  // inputs, copied
  int n = 0;
  std::vector<double> mass, charge, sigma, epsilon;
  std::array<double, 9> box{};
  std::vector<int> cp1, cp2;
  std::vector<double> cdist;
  bool has_nonbonded = false;
  double cutoff = 0, tolerance = 0, alpha = 0;
  bool dispersion = false;
  std::vector<int> ep1, ep2;
  std::vector<double> eqq, esig, eeps;
  std::vector<BondDev> bonds;
  std::vector<AngleDev> angles;
  std::vector<TorsionDev> torsions;
  std::vector<int> rparticle;
  std::vector<double> rk, rx0, ry0, rz0;
  int com_frequency = 0;
  int barostat_frequency = 0;
  double barostat_pressure = 0, barostat_temperature = 0;

  // derived
  std::array<int, 3> grid{0, 0, 0};
  std::vector<SettleHost> settle;
  std::vector<ShakeHost> shake;
  std::vector<int> free_atoms;
  std::vector<std::vector<int>> molecules;
  double dof = 0;
  double total_mass = 0;
  double self_energy = 0;
  double dispersion_energy = 0, net_charge_energy = 0;
  std::array<double, 2> dispersion_sums{0, 0};  // <eps s^12>, <eps s^6> numerators / pairs
  double charge_sum = 0;
};

// Runs every check the reference's constructors run, and fills `out`.
// Returns an mdb_status; `error` gets the message.
int prepare_system(const mdb_system_desc& in, const mdb_state_desc& state, const mdb_run_options& opt,
                   HostSystem& out, std::string& error);

// Box-dependent host constants (dispersion, net charge) for the current box.
void update_box_constants(HostSystem& h);

bool reduce_box(const double* in, double* out);
void perpendicular_widths(const double* box, double* out);
double box_volume(const double* box);
void inverse_box(const double* box, double* m);  // f = r . M, M[v*3+u]
std::vector<double> bspline_moduli(int n);
bool plan_radices(int n, int* radices, int* count);

}  // namespace mdb
