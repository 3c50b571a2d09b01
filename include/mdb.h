/*
 * mdb.h -- the C ABI of the B200 molecular-dynamics step engine.
 *
 * This is the drop-in boundary for the step loop of making-it-rain-webgpu:
 * every entry point below replaces one public member of `StepLoop`
 * (src/gpu/loop.ts) or of the single-configuration evaluators it is tested
 * through, and the comment on each names the reference interface it stands in
 * for (paths relative to the reference project root).
 *
 * Conventions, all of them fixed:
 *   - Plain C types only: pointers, sizes, doubles.  No torch, no CUDA types.
 *   - Units are OpenMM's: nm, ps, amu, kJ/mol, e, K, bar (src/engine/units.ts).
 *   - Positions, velocities and forces are xyz-interleaved double arrays of
 *     3*N entries, as `StepLoop.positions()` returns them (loop.ts:900).
 *   - Box vectors are row-major a, b, c (9 doubles) in OpenMM's reduced form.
 *   - Every function returns an `int` status (`mdb_status`); nothing is
 *     thrown across the ABI.  The message for the last failure on an engine
 *     is `mdb_last_error(engine)`.  The reference throws named Error subclasses
 *     instead (src/engine/system.ts:178, src/gpu/nonbonded.ts:54,
 *     src/engine/constraint-clusters.ts:71, src/reference/triclinic.ts:179);
 *     each has a status code here.
 *   - Calls on one engine are not thread-safe: one host thread per engine, as
 *     the reference's single JS thread (src/gpu/loop.ts:208).
 *   - Input arrays are copied; nothing is aliased after a call returns
 *     (src/gpu/allocator.ts:69 ownership rule).
 */
#ifndef MDB_H
#define MDB_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MDB_ABI_VERSION 3

typedef enum mdb_status {
  MDB_OK = 0,
  MDB_ERR_INVALID_ARGUMENT = 1,
  /* UnsupportedForce, src/engine/system.ts:178 */
  MDB_ERR_UNSUPPORTED_FORCE = 2,
  /* CutoffTooLargeForBox, src/reference/triclinic.ts:179 */
  MDB_ERR_CUTOFF_TOO_LARGE_FOR_BOX = 3,
  /* ClusterTooLarge, src/engine/constraint-clusters.ts:71 */
  MDB_ERR_CLUSTER_TOO_LARGE = 4,
  /* SHAKE/RATTLE gave up after the iteration cap, src/reference/constraints.ts:34 */
  MDB_ERR_NOT_CONVERGED = 5,
  /* a device-side table (tile list, cell list) ran out of room */
  MDB_ERR_CAPACITY = 6,
  /* fixed-point range exceeded: a diverged run, src/reference/fixed-point.ts:56 */
  MDB_ERR_RANGE = 7,
  MDB_ERR_DEVICE = 8,
  /* a bounded device-side wait gave up */
  MDB_ERR_TIMEOUT = 9,
  MDB_ERR_NO_DEVICE = 10,
  /* NotSmooth, src/reference/fft.ts:24 */
  MDB_ERR_NOT_SMOOTH = 11,
  MDB_ERR_DEVICE_LOST = 12
} mdb_status;

enum { MDB_INTEGRATOR_LFMIDDLE = 0, MDB_INTEGRATOR_VERLET = 1 };

/* Run-option flags. */
enum {
  /* Launch every kernel directly instead of replaying captured CUDA graphs. */
  MDB_FLAG_NO_GRAPH = 1,
  /* Rebuild the tile list every step, whatever the displacement. */
  MDB_FLAG_ALWAYS_REBUILD = 2,
  /* Run the list build's phases as separate kernel launches instead of one
     cooperative launch (each phase then shows up on its own in a profiler). */
  MDB_FLAG_PHASE_LAUNCHES = 4
};

/*
 * An OpenMM System, as flat arrays.  Mirrors `OpenMMSystem` and the force
 * interfaces of src/engine/system.ts:41-173.  A force that is absent has its
 * count set to zero (or `has_nonbonded` = 0).  Bonded forces never use
 * periodic boundary conditions (src/reference/forces/bonded.ts:14-18).
 */
typedef struct mdb_system_desc {
  int32_t n_particles;
  const double* masses; /* amu; 0 = frozen particle */
  double box[9];        /* default periodic box vectors */

  int32_t n_constraints;
  const int32_t* constraint_p1;
  const int32_t* constraint_p2;
  const double* constraint_distance; /* nm */

  /* NonbondedForce with method PME (system.ts:88-121) */
  int32_t has_nonbonded;
  double cutoff;          /* nm */
  double ewald_tolerance;
  double alpha;           /* nm^-1; 0 = derive from cutoff and tolerance */
  int32_t grid[3];        /* 0 = derive from box and tolerance */
  int32_t use_dispersion_correction;
  const double* charge;   /* e */
  const double* sigma;    /* nm */
  const double* epsilon;  /* kJ/mol */
  int32_t n_exceptions;
  const int32_t* exception_p1;
  const int32_t* exception_p2;
  const double* exception_charge_prod; /* e^2 */
  const double* exception_sigma;
  const double* exception_epsilon;

  /* HarmonicBondForce: E = k/2 (r - length)^2 */
  int32_t n_bonds;
  const int32_t* bond_p1;
  const int32_t* bond_p2;
  const double* bond_length;
  const double* bond_k;

  /* HarmonicAngleForce: E = k/2 (theta - angle)^2 */
  int32_t n_angles;
  const int32_t* angle_p1;
  const int32_t* angle_p2;
  const int32_t* angle_p3;
  const double* angle_theta;
  const double* angle_k;

  /* PeriodicTorsionForce: E = k (1 + cos(n phi - phase)) */
  int32_t n_torsions;
  const int32_t* torsion_p1;
  const int32_t* torsion_p2;
  const int32_t* torsion_p3;
  const int32_t* torsion_p4;
  const int32_t* torsion_periodicity;
  const double* torsion_phase;
  const double* torsion_k;

  /* CMMotionRemover; 0 = absent (com-motion.ts:38) */
  int32_t com_frequency;

  /* MonteCarloBarostat; frequency 0 = absent (system.ts:128) */
  int32_t barostat_frequency;
  double barostat_pressure;    /* bar */
  double barostat_temperature; /* K */

  /* PositionRestraint, k*periodicdistance(x,y,z,x0,y0,z0)^2 (system.ts:139) */
  int32_t n_restraints;
  const int32_t* restraint_particle;
  const double* restraint_k;
  const double* restraint_x0;
  const double* restraint_y0;
  const double* restraint_z0;
} mdb_system_desc;

/* An OpenMM State: mirrors `OpenMMState`, src/engine/state.ts:18-39. */
typedef struct mdb_state_desc {
  const double* positions;  /* 3N, nm */
  const double* velocities; /* 3N, nm/ps; NULL = all zero */
  double box[9];
  int64_t step;
} mdb_state_desc;

/* Mirrors `RunOptions`, src/gpu/loop.ts:117-168. */
/*
 * Per-system tuning of the neighbour machinery (no reference counterpart):
 * chosen per size bucket by mdb_autotune, passed one per system through
 * mdb_run_options.tuning.  Zero or negative fields keep the defaults.
 */
typedef struct mdb_tuning {
  double verlet_skin;  /* nm; list radius = cutoff + skin; default 0.15 (nonbonded.ts:227) */
  double sort_cell;    /* nm; width of the fractional cells of the spatial sort; default 0.25 */
  int32_t tile_atoms;  /* atoms per cluster of the pair tiles, 8 or 32; default 8.  One shape per
                          engine: a batch takes the first system's that sets one */
  int32_t prune_tiles; /* 1: each rebuild drops the tiles with no pair inside cutoff + skin;
                          2: keeps them; 0: default (1).  Per engine, like tile_atoms */
  double inner_skin;   /* nm; > 0: the pair kernel reads an inner list of the tiles with a pair
                          inside cutoff + inner_skin, pruned again from the outer list whenever an
                          atom has moved inner_skin / 2 (results are bit-identical to the outer
                          list's); negative: off; 0: the default */
} mdb_tuning;

typedef struct mdb_run_options {
  double time_step;            /* ps */
  double temperature;          /* K */
  double friction;             /* ps^-1; 0 = deterministic without a seed */
  double constraint_tolerance; /* relative */
  uint32_t seed;
  int32_t integrator;          /* MDB_INTEGRATOR_* */
  double verlet_skin;          /* nm; negative = the default 0.15 (nonbonded.ts:227) */
  int32_t max_batch;           /* steps per captured graph; 0 = 100 (loop.ts:171) */
  int32_t mesh[3];             /* PME mesh override; 0 = from the box */
  int32_t device;              /* CUDA device ordinal */
  int32_t flags;               /* MDB_FLAG_* */
  const mdb_tuning* tuning;    /* NULL, or one entry per system of the engine (no reference counterpart) */
  int32_t surrogate_attempts;  /* > 0: the engine's barostats learn one screening network from that many
                                  exact attempts (pooled over the engine's systems), then screen proposals
                                  by delayed acceptance; 0 = plain barostat (no reference counterpart) */
  int32_t tile_row_capacity;   /* starting capacity of the tile list, tiles per cluster; 0 = the
                                  default.  A list that needs more is grown and rebuilt before any step
                                  uses it (no reference counterpart: the reference's list has a fixed
                                  capacity and an overflow pass, src/gpu/loop.ts:380-392) */
} mdb_run_options;

/*
 * Energies by OpenMM force group, kJ/mol.  `direct_group` and
 * `reciprocal_group` are what OpenMM reports for "NonbondedForce[direct]" and
 * "NonbondedForce[reciprocal]" (src/reference/potential.ts:122-141); the parts
 * they sum are given separately (src/reference/forces/nonbonded.ts:79-96).
 */
typedef struct mdb_energies {
  double bond;
  double angle;
  double torsion;
  double restraint;
  double direct_coulomb;       /* erfc Coulomb over non-excluded pairs */
  double direct_lj;            /* LJ over non-excluded pairs */
  double exclusion_correction; /* minus the reciprocal part of excluded pairs */
  double exceptions;           /* the exceptions' own Coulomb + LJ */
  double dispersion;           /* analytic long-range correction */
  double reciprocal_mesh;      /* the mesh sum alone */
  double self_energy;
  double net_charge;
  double direct_group;
  double reciprocal_group;
  double potential;
  double kinetic;              /* from the velocities as they are (kinetic.ts:31) */
  double temperature;          /* K, from `kinetic` and the constrained DoF */
  double degrees_of_freedom;
  double virial[9];            /* W[3a+b] = sum r_a F_b = -dU/d eps_ab under the strain x -> (1+eps) x
                                  of positions and box: pairs, exceptions, bonded terms, PME mesh,
                                  dispersion and net-charge corrections (not restraints); kJ/mol.
                                  No reference counterpart. */
  double pairs_within_cutoff;  /* non-excluded pairs inside the cutoff (count) */
  double molecular_virial[9];  /* -dU/d eps under scaling of molecule centres (the plain mean of a
                                  molecule's positions, as the barostat moves them): the virial
                                  minus sum_i (r_i - R_mol(i)) (x) F_i.  No reference counterpart. */
} mdb_energies;

/* Mirrors `StepLoop.barostatStatistics`, src/gpu/loop.ts:572. */
typedef struct mdb_barostat_stats {
  int64_t attempts;
  int64_t accepted;
  double volume_scale;     /* nm^3 */
  /* delayed-acceptance screening (no reference counterpart) */
  int64_t screened;          /* proposals rejected by the network stage alone */
  int64_t exact_evaluations; /* exact potential evaluations the attempts made */
  int64_t training_samples;  /* exact attempts the network learned from (all systems of the engine) */
  int32_t surrogate_active;  /* 1 while proposals are screened */
  int32_t surrogate_disabled;/* 1 when the exact stage found the network too inaccurate */
  double surrogate_rms;      /* running RMS of (predicted - exact) potential change, kJ/mol */
  double training_loss;      /* final mean squared training loss (standardised units) */
  double training_ms;        /* device time of the network's fits so far */
} mdb_barostat_stats;

/*
 * Device time per stage of one step, each stage launched alone on the
 * engine's stream and timed with CUDA events over `repeats` launches.
 * Mirrors `StepLoop.profileStep()`, src/gpu/loop.ts:705, and like it
 * advances the system (the integrator stage runs `repeats` times).
 */
typedef struct mdb_profile {
  int32_t launches_per_step;   /* kernels one graph-replayed step launches */
  int32_t repeats;
  double ms_step;              /* one whole step, as replayed from a graph */
  double ms_list_check;        /* list kernels when no rebuild is due */
  double ms_list_rebuild;      /* a full sort + tile-list rebuild */
  double ms_nonbonded;
  double ms_listed;
  double ms_pme;               /* spread + 5 FFT passes + gather */
  double ms_pme_spread;
  double ms_pme_fft;
  double ms_pme_gather;
  double ms_integrate;
  int64_t pairs_within_cutoff; /* at the configuration profiled, summed over the engine's systems */
  int64_t tiles;
  int64_t atoms;
  int64_t mesh_points;
  int64_t inner_tiles;         /* tiles the pair kernel reads (the inner list, or the whole list) */
  double ms_inner_prune;       /* an inner-list prune with no rebuild (0 without an inner list) */
  int64_t tile_atoms;          /* atoms per cluster: a tile holds tile_atoms^2 pair slots */
} mdb_profile;

/* Mirrors `StepLoop.verletFlags`, src/gpu/loop.ts:941. */
typedef struct mdb_neighbour_stats {
  int64_t rebuilds;
  int64_t tiles;          /* cluster-pair tiles in the current list */
  int64_t tile_capacity;  /* tiles the list can hold at its current size */
  int64_t blocks;         /* clusters of tile_atoms atoms (rows of the tile list) */
  int32_t overflowed;     /* 1 if the list has outgrown its capacity since creation (it was then grown
                             and rebuilt before any step used it) */
  double skin;            /* nm */
  int64_t inner_tiles;    /* tiles of the inner list the pair kernel reads (= tiles without one) */
  int64_t prunes;         /* inner-list prunes between rebuilds since creation */
  double inner_skin;      /* nm; 0 without an inner list */
  int32_t tile_atoms;     /* atoms per cluster: 8 (8x8 tiles) or 32 (32x32 tiles) */
  int64_t list_grown;     /* times the list was grown after an overflow */
} mdb_neighbour_stats;

typedef struct mdb_engine mdb_engine;

/* ---- lifetime --------------------------------------------------------- */

int mdb_abi_version(void);
const char* mdb_status_string(int status);

/* Number of CUDA devices visible; 0 with MDB_ERR_NO_DEVICE when there are none. */
int mdb_device_count(int32_t* out);

/*
 * One system.  Replaces `StepLoop.fromParsed(device, system, state, options)`,
 * src/gpu/loop.ts:278.  Validates, splits the constraints
 * (constraint-clusters.ts:93), derives alpha and the mesh (loop.ts:298-306),
 * uploads, and builds the first neighbour list.
 */
int mdb_create(const mdb_system_desc* system, const mdb_state_desc* state,
               const mdb_run_options* options, mdb_engine** out);

/*
 * Many independent systems advanced together, one launch per stage for all of
 * them.  No reference counterpart: the reference runs one system per device.
 * `systems` and `states` are arrays of `n` descriptors.
 */
int mdb_batch_create(int32_t n, const mdb_system_desc* systems,
                     const mdb_state_desc* states, const mdb_run_options* options,
                     mdb_engine** out);

/* Replaces `StepLoop.destroy()`, loop.ts:1113.  `leaked_bytes` may be NULL. */
int mdb_destroy(mdb_engine* engine, int64_t* leaked_bytes);

const char* mdb_last_error(const mdb_engine* engine);
int mdb_system_count(const mdb_engine* engine, int32_t* out);

/* ---- stepping ----------------------------------------------------------- */

/*
 * Advance every system by `steps` steps.  Replaces `StepLoop.run(n)`,
 * loop.ts:651, including the barostat attempts it makes between batches
 * (loop.ts:662-685).  Systems whose barostats are due at the same step attempt
 * together: one evaluation of the engine for their current energies and one
 * for their proposals; each draws from its own counter, so its moves are the
 * ones it makes alone.
 */
int mdb_run(mdb_engine* engine, int64_t steps);

/*
 * `mdb_run` timed on the device with CUDA events recorded on the engine's own
 * stream; `*device_ms` is the elapsed device time.  No reference counterpart
 * (the reference times passes with timestamp queries, src/gpu/profile.ts:68).
 */
int mdb_run_timed(mdb_engine* engine, int64_t steps, double* device_ms);

/* Replaces `StepLoop.advanceStepCount`, loop.ts:564. */
int mdb_set_step(mdb_engine* engine, int64_t step);
int mdb_get_step(const mdb_engine* engine, int64_t* step);

/* ---- state in and out --------------------------------------------------- */

/* Replace `StepLoop.positions()` / `velocities()`, loop.ts:900/909. */
int mdb_get_positions(mdb_engine* engine, int32_t system, double* out);
int mdb_get_velocities(mdb_engine* engine, int32_t system, double* out);

/* Replace `StepLoop.setPositions` / `setVelocities`, loop.ts:819/842.
 * setPositions clears the integrator's residual, as the reference does. */
int mdb_set_positions(mdb_engine* engine, int32_t system, const double* positions);
int mdb_set_velocities(mdb_engine* engine, int32_t system, const double* velocities);

/* Replaces `StepLoop.setBox(vectors)`, loop.ts:1031; the mesh is kept. */
int mdb_set_box(mdb_engine* engine, int32_t system, const double box[9]);
int mdb_get_box(const mdb_engine* engine, int32_t system, double box[9]);
int mdb_get_mesh(const mdb_engine* engine, int32_t system, int32_t mesh[3]);

/* ---- evaluation ---------------------------------------------------------- */

/*
 * Forces and energies by group at the current configuration.  Replaces
 * `StepLoop.evaluateForces()` + `report()` (loop.ts:924, 761) and the
 * per-group evaluators `evaluateDirectSpace` (nonbonded.ts:1000),
 * `evaluateReciprocalSpace` (pme.ts:454) and `evaluateBondedForce`
 * (forces.ts:189).  `forces` (3N, kJ/mol/nm) and `energies` may be NULL.
 */
int mdb_evaluate(mdb_engine* engine, int32_t system, double* forces,
                 mdb_energies* energies);

/*
 * Energy and forces at the given positions, leaving the engine's own state
 * unchanged.  Replaces `StepLoop.potential(positions)`, loop.ts:870.
 */
int mdb_potential(mdb_engine* engine, int32_t system, const double* positions,
                  double* forces, mdb_energies* energies);

/* ---- statistics ------------------------------------------------------------ */

/*
 * The cell grid the list was built on: divisions per axis of the spatial
 * sort's fractional cells and each cell's extent along the box's diagonal, nm.
 * Replaces `StepLoop.cellGeometry()`, src/gpu/loop.ts:894 (whose cells are the
 * neighbour search's; here they are the finer cells of the sort that orders
 * the clusters).
 */
int mdb_get_cell_geometry(const mdb_engine* engine, int32_t system, int32_t divisions[3], double extent[3]);

/* Kernel launches one step makes.  Replaces `StepLoop.passesPerStep`, loop.ts:1105. */
int mdb_get_passes_per_step(const mdb_engine* engine, int32_t* out);

int mdb_get_barostat_stats(const mdb_engine* engine, int32_t system,
                           mdb_barostat_stats* out);
int mdb_get_neighbour_stats(mdb_engine* engine, int32_t system,
                            mdb_neighbour_stats* out);

/*
 * Reciprocal-space PME (mesh energy and forces) that allocates nothing.  No
 * counterpart in the reference.  For callers that cannot allocate device
 * memory -- code running inside another framework's memory pool, a host that
 * only receives device buffers from its own allocator, or a loop that must
 * not allocate once started: the caller passes its own device buffers, and
 * every intermediate lives in one fixed-size device array inside the library,
 * so no cudaMalloc/cudaFree or allocating library call is made.
 *
 *   positions  device, 3n doubles, nm            charges  device, n doubles, e
 *   forces     device, 3n doubles, overwritten with the reciprocal forces
 *   energy     device, 1 double, the mesh sum (no self or net-charge term)
 *   box        host, 9 doubles; mesh host, 3 ints; alpha in nm^-1
 *   stream     a cudaStream_t, or NULL for the default stream
 *
 * Limits: at most 262,144 mesh points (64^3) and 128 points per axis, at
 * least 5 points per axis (the order-5 spline's span), each axis
 * 2/3/5/7-smooth; larger meshes return MDB_ERR_CAPACITY, shorter axes
 * MDB_ERR_INVALID_ARGUMENT and non-smooth ones MDB_ERR_NOT_SMOOTH, before any
 * device work.  The array (about 5.3 MB) stays resident on every device that
 * loads the library until the process exits.  A call on a stream that is not
 * capturing looks up the array's device address (so after cudaDeviceReset the
 * next such call finds the reloaded array); a call inside a stream capture
 * reuses the address the last call outside one found, so make the first call
 * on a device, and the first after a device reset, before any stream capture.
 * Every call shares the array and leaves its contents behind (the charge grid
 * is cleared at the start of each call); calls whose device work overlaps
 * race on it.  A CUDA error pending from the caller's earlier work is
 * reported as MDB_ERR_DEVICE and left pending; this call then does nothing.
 */
int mdb_reciprocal_noalloc(int32_t n, const double* positions, const double* charges,
                           const double box[9], double alpha, const int32_t mesh[3],
                           double* forces, double* energy, void* stream);

/*
 * Autotuner (no reference counterpart).  Times every candidate of a fixed grid
 * of (tile_atoms, prune_tiles, verlet_skin, sort_cell, inner_skin) on the device -- a temporary engine per
 * candidate, `steps` graph-replayed steps after a warm-up of the same length,
 * CUDA-event timed -- and returns the fastest in `best` and its ms per step.
 * `tried` (may be NULL) receives the number of candidates.  The state the
 * candidates start from is `state`; nothing else is changed.
 */
int mdb_autotune(const mdb_system_desc* system, const mdb_state_desc* state, const mdb_run_options* options,
                 int32_t steps, mdb_tuning* best, double* best_ms_per_step, int32_t* tried);

/*
 * The same search on a batch: every candidate is applied to all `n` systems
 * of one batched engine (as mdb_batch_create), and the time is that engine's
 * step.  A batch keeps the device busy where one small system leaves it
 * waiting on launches, so the candidate that wins for a batch of a size
 * bucket's systems can differ from the one that wins for any one of them.
 * With n > 1 the grid is 8-atom tiles only, over ten (skin, inner skin)
 * pairs from (0.15 nm, none) to (0.5, 0.1) and two sort cells: 20 candidates.
 */
int mdb_autotune_batch(int32_t n, const mdb_system_desc* systems, const mdb_state_desc* states,
                       const mdb_run_options* options, int32_t steps, mdb_tuning* best, double* best_ms_per_step,
                       int32_t* tried);

/*
 * The barostat screening network's kernels on their own (no reference
 * counterpart), for checking them against a CPU restatement.  Layout of
 * `params` (kMlpParams = 5313 floats): W1[64][16], b1[64], W2[64][64], b2[64],
 * w3[64], b3.  Inputs x[n][16], targets t[n], host arrays; these entry points
 * allocate device memory.
 *   mdb_mlp_gradient: the weights are rounded to BF16 as the kernels use them;
 *     writes the mean-squared-error gradient of the first min(n, 128) samples
 *     (FP32, accumulated in FP32) and that loss.
 *   mdb_mlp_fit: seeded Glorot start, `epochs` epochs of Adam (lr 2e-3,
 *     minibatch 128); writes the final FP32 master weights and, per epoch, the
 *     mean minibatch loss.
 */
int mdb_mlp_gradient(const float* params, const float* x, const float* t, int32_t n, float* grad, float* loss);
int mdb_mlp_fit(const float* x, const float* t, int32_t n, int32_t epochs, uint32_t seed, float* params,
                float* epoch_loss);
int mdb_mlp_predict(const float* params, const float* x, int32_t n, float* y);

/* Per-stage device timing (see mdb_profile).  Replaces `StepLoop.profileStep`, loop.ts:705. */
int mdb_profile_step(mdb_engine* engine, int32_t repeats, mdb_profile* out);

/*
 * Device memory the engine holds, by owner label, as "label=bytes;" pairs in
 * `buffer` (NUL-terminated, truncated to `capacity`).  Replaces
 * `BufferPool.report()`, src/gpu/allocator.ts:69.
 */
int mdb_memory_report(const mdb_engine* engine, char* buffer, int64_t capacity,
                      int64_t* total_bytes);

#ifdef __cplusplus
}
#endif

#endif /* MDB_H */
