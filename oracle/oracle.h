/*
 * oracle.h -- TEST INFRASTRUCTURE, not part of the engine.
 *
 * A double-precision CPU restatement of the reference's own f64 oracle,
 * src/reference/ (all files) of making-it-rain-webgpu.  Only tests/, the smoke check and
 * bench.py's CPU-baseline leg may load it, and only as the checker.  The
 * engine (libmdb200) never links, loads or calls anything here.
 *
 * Parity of this restatement is pinned against the reference's committed
 * golden data, regenerated as JSON by tests/golden/make_golden.py:
 *   - test/fixtures/nonbonded-{system,state}.xml + nonbonded-facts.json
 *     (OpenMM 8.4 PME and Ewald group energies, forces, term decomposition);
 *   - the Random123 threefry2x32 known answers held in test/random.test.ts;
 *   - the mpmath erf/erfc values held in test/erf.test.ts;
 *   - the OpenMM triclinic minimum-image separations in
 *     test/fixtures/triclinic-openmm.json.
 */
#ifndef MDB_ORACLE_H
#define MDB_ORACLE_H

#include <stdint.h>
#include "../include/mdb.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_energies {
  double bond, angle, torsion, restraint;
  double direct_coulomb, direct_lj, exclusion_correction, exceptions, dispersion;
  double reciprocal_mesh, self_energy, net_charge;
  double direct_group, reciprocal_group, potential;
  int64_t pairs_within_cutoff;
} orc_energies;

typedef struct orc_step_options {
  double time_step, temperature, friction, constraint_tolerance;
  uint32_t seed;
  int32_t integrator;     /* MDB_INTEGRATOR_* */
  int32_t grid[3];        /* PME mesh; 0 = derive */
  int32_t threads;        /* OpenMP threads for the force evaluation; <=1 = serial */
} orc_step_options;

/* src/engine/units.ts:53,65,78 */
double orc_ewald_alpha(double cutoff, double tolerance);
int32_t orc_pme_minimum_grid(double alpha, double length, double tolerance);
int32_t orc_smooth_fft_size(int32_t minimum);

/* src/reference/erf.ts:68-100 */
double orc_erf(double x);
double orc_erfc(double x);
double orc_erf_derivative(double x);

/* src/reference/fixed-point.ts:55-114; status 0 ok, MDB_ERR_RANGE otherwise */
int32_t orc_fixed_words(float value, uint32_t* lo, int32_t* hi);
float orc_from_fixed_f32(int64_t fixed);
double orc_from_fixed(int64_t fixed);

/* src/reference/random.ts:63-196 */
void orc_threefry2x32(uint32_t c0, uint32_t c1, uint32_t k0, uint32_t k1,
                      int32_t rounds, uint32_t out[2]);
double orc_open_unit_interval(uint32_t bits);
double orc_thermostat_normal(uint32_t seed, uint32_t step, uint32_t particle, int32_t axis);
double orc_domain_normal(uint32_t domain, uint32_t seed, uint32_t particle, int32_t axis);

/* src/reference/triclinic.ts */
int32_t orc_reduce_box(const double in[9], double out[9]);
void orc_perpendicular_widths(const double box[9], double out[3]);
double orc_box_volume(const double box[9]);
void orc_minimum_image(const double box[9], const double d[3], double out[3]);
void orc_nearest_image_by_search(const double box[9], const double d[3], double out[3]);

/* src/reference/forces/bspline.ts:55,102 */
void orc_bspline(double w, double weights[5], double derivatives[5]);
void orc_bspline_moduli(int32_t n, double* out);

/*
 * Whole potential by group.  src/reference/potential.ts:94-171.
 * `forces` (3N) may be NULL.  `grid` NULL or zeros = the default mesh.
 * Returns a status.
 */
int32_t orc_potential(const mdb_system_desc* sys, const double* positions,
                      const double box[9], const int32_t* grid, int32_t threads,
                      int32_t naive_direct, double* forces, orc_energies* out);

/* The same evaluation plus the virial tensor W[3a+b] = sum r_a F_b
 * (= -dU/d eps_ab under the affine strain x -> (1 + eps) x of positions and
 * box), pairs, exceptions, bonded terms, the PME mesh sum and the 1/V
 * dispersion and net-charge corrections; restraints excluded.  No reference
 * counterpart.  Not thread-safe (a module-level accumulator). */
/* The barostat screening network's mean-squared-error gradient over the
 * first min(n, 128) samples, in f64 (the CUDA kernel's checker).  No reference
 * counterpart. */
int32_t orc_mlp_gradient(const float* params, const float* x, const float* t, int32_t n, double* grad,
                         double* loss);

/* The non-excluded pairs within `eps` of the cutoff (minimum image), the
 * force each would put on `first` if inside, and whether it is inside in f64.
 * Writes at most `max_pairs`; returns the total.  No reference counterpart:
 * the parity tests allow such pairs either way. */
int32_t orc_cutoff_shell(const mdb_system_desc* sys, const double* positions, const double box[9],
                         double eps, int32_t max_pairs, int32_t* first, int32_t* second,
                         double* force_on_first, int32_t* inside);

int32_t orc_potential_virial(const mdb_system_desc* sys, const double* positions, const double box[9],
                             const int32_t* grid, int32_t threads, double* forces, orc_energies* out,
                             double virial[9]);

/* Exact Ewald reciprocal sum (src/reference/forces/ewald.ts), k-space only. */
int32_t orc_ewald_reciprocal(const mdb_system_desc* sys, const double* positions,
                             const double box[9], double alpha, int32_t kmax,
                             double* forces, double* energy);

/* Constraint split (src/engine/constraint-clusters.ts:93). */
int32_t orc_split_counts(const mdb_system_desc* sys, int32_t* settle_clusters,
                         int32_t* iterative_clusters, int32_t* largest_atoms,
                         int32_t* largest_constraints);

/* Degrees of freedom (src/reference/kinetic.ts:106) and KE (kinetic.ts:31). */
double orc_degrees_of_freedom(const mdb_system_desc* sys);
double orc_kinetic_energy(const mdb_system_desc* sys, const double* velocities);

/* COM removal, src/reference/com-motion.ts:48.  In place. */
void orc_remove_com(const mdb_system_desc* sys, double* velocities);

/* Constraint projections (src/reference/constraints.ts:254,274). In place. */
int32_t orc_constrain_positions(const mdb_system_desc* sys, const double* reference,
                                double* trial, double tolerance);
int32_t orc_constrain_velocities(const mdb_system_desc* sys, const double* positions,
                                 double* velocities, double tolerance);

/*
 * `steps` steps of the step loop: COM removal on removesOnStep
 * (com-motion.ts:38), forces (potential.ts:94), then LFMiddle
 * (integrator.ts:140) or Verlet (integrator.ts:68), with thermostat noise from
 * thermostatNormal(seed, step, i, axis) (random.ts:178).  `positions` and
 * `velocities` are updated in place; `*step` advances.
 */
int32_t orc_run(const mdb_system_desc* sys, double* positions, double* velocities,
                const double box[9], const orc_step_options* options, int64_t* step,
                int64_t steps);

/* Molecule scaling for the barostat, src/reference/barostat.ts:148. */
int32_t orc_molecule_count(const mdb_system_desc* sys);
void orc_scale_molecules(const mdb_system_desc* sys, double* positions, double scale);

/* Maxwell-Boltzmann velocities on VELOCITY_DOMAIN (velocities.ts:78), projected. */
void orc_velocities_at_temperature(const mdb_system_desc* sys, const double* positions,
                                   double temperature, uint32_t seed, double* out);

#ifdef __cplusplus
}
#endif
#endif
