// addon.cc -- Node-API binding of libmdb200 for the TypeScript StepLoop shim
// (../ts/step-loop.ts).  Written against Node-API's documented C interface
// (node_api.h, NAPI_VERSION 8).  Neither Node nor its headers exist on the
// build or GPU machines of this project, so this file is not compiled there;
// a maintainer builds it with node-gyp next to libmdb200.so.
//
// Every method is synchronous: the engine returns when the device work it
// queued has finished (loop.ts awaits `onSubmittedWorkDone` the same way).
// Errors become JS exceptions whose `name` is the reference's error class
// (UnsupportedForce, CutoffTooLargeForBox, ClusterTooLarge, NotSmooth, ...).
#include <node_api.h>

#include <cstring>
#include <string>
#include <vector>

#include "../../include/mdb.h"

namespace {

const char* error_name(int status) {
  switch (status) {
    case MDB_ERR_UNSUPPORTED_FORCE: return "UnsupportedForce";
    case MDB_ERR_CUTOFF_TOO_LARGE_FOR_BOX: return "CutoffTooLargeForBox";
    case MDB_ERR_CLUSTER_TOO_LARGE: return "ClusterTooLarge";
    case MDB_ERR_NOT_SMOOTH: return "NotSmooth";
    case MDB_ERR_RANGE: return "RangeError";
    default: return "Error";
  }
}

napi_value throw_status(napi_env env, int status, mdb_engine* e) {
  std::string msg = e ? mdb_last_error(e) : mdb_status_string(status);
  napi_value message, error, name;
  napi_create_string_utf8(env, msg.c_str(), NAPI_AUTO_LENGTH, &message);
  napi_create_error(env, nullptr, message, &error);
  napi_create_string_utf8(env, error_name(status), NAPI_AUTO_LENGTH, &name);
  napi_set_named_property(env, error, "name", name);
  napi_throw(env, error);
  return nullptr;
}

napi_value throw_message(napi_env env, const std::string& msg) {
  napi_value message, error;
  napi_create_string_utf8(env, msg.c_str(), NAPI_AUTO_LENGTH, &message);
  napi_create_error(env, nullptr, message, &error);
  napi_throw(env, error);
  return nullptr;
}

mdb_engine* engine_of(napi_env env, napi_value v) {
  void* p = nullptr;
  napi_get_value_external(env, v, &p);
  return static_cast<mdb_engine*>(p);
}

template <typename T>
T* typed_array(napi_env env, napi_value v, size_t* length) {
  napi_typedarray_type type;
  void* data = nullptr;
  napi_value buffer;
  size_t offset = 0;
  napi_get_typedarray_info(env, v, &type, length, &data, &buffer, &offset);
  return static_cast<T*>(data);
}

double number(napi_env env, napi_value obj, const char* key, double fallback) {
  bool has = false;
  napi_has_named_property(env, obj, key, &has);
  if (!has) return fallback;
  napi_value v;
  napi_get_named_property(env, obj, key, &v);
  double out = fallback;
  napi_get_value_double(env, v, &out);
  return out;
}

// A boolean member (or a number, non-zero = true); `fallback` when absent.
bool flag(napi_env env, napi_value obj, const char* key, bool fallback) {
  bool has = false;
  napi_has_named_property(env, obj, key, &has);
  if (!has) return fallback;
  napi_value v;
  napi_get_named_property(env, obj, key, &v);
  napi_valuetype t;
  napi_typeof(env, v, &t);
  if (t == napi_boolean) {
    bool out = fallback;
    napi_get_value_bool(env, v, &out);
    return out;
  }
  if (t == napi_number) {
    double out = fallback ? 1.0 : 0.0;
    napi_get_value_double(env, v, &out);
    return out != 0.0;
  }
  return fallback;
}

napi_value property(napi_env env, napi_value obj, const char* key) {
  napi_value v = nullptr;
  napi_get_named_property(env, obj, key, &v);
  return v;
}

// `boxVectors` ([a, b, c] rows, nm) of a System or a State into `out`; false
// when the object has none.
bool read_box(napi_env env, napi_value obj, double* out) {
  bool has = false;
  napi_has_named_property(env, obj, "boxVectors", &has);
  if (!has) return false;
  napi_value bv = property(env, obj, "boxVectors");
  uint32_t rows = 0;
  if (napi_get_array_length(env, bv, &rows) != napi_ok || rows != 3) return false;
  for (uint32_t r = 0; r < 3; ++r) {
    napi_value row;
    napi_get_element(env, bv, r, &row);
    for (uint32_t c = 0; c < 3; ++c) {
      napi_value x;
      napi_get_element(env, row, c, &x);
      napi_get_value_double(env, x, &out[r * 3 + c]);
    }
  }
  return true;
}

// OpenMMSystem (src/engine/system.ts:161) -> mdb_system_desc.  The typed
// arrays are borrowed for the duration of the create call only.  A force type
// the engine does not implement is refused by name (`unsupported` holds it),
// as the reference's parser refuses it, rather than dropped.
bool fill_system(napi_env env, napi_value sys, mdb_system_desc* d, std::vector<double>& box,
                 std::string& unsupported) {
  std::memset(d, 0, sizeof(*d));
  size_t n = 0;
  d->masses = typed_array<double>(env, property(env, sys, "masses"), &n);
  d->n_particles = int32_t(n);
  read_box(env, sys, d->box);
  size_t nc = 0;
  d->constraint_p1 = typed_array<int32_t>(env, property(env, sys, "constraintP1"), &nc);
  d->constraint_p2 = typed_array<int32_t>(env, property(env, sys, "constraintP2"), &nc);
  d->constraint_distance = typed_array<double>(env, property(env, sys, "constraintDistance"), &nc);
  d->n_constraints = int32_t(nc);
  napi_value forces = property(env, sys, "forces");
  uint32_t count = 0;
  napi_get_array_length(env, forces, &count);
  for (uint32_t k = 0; k < count; ++k) {
    napi_value f;
    napi_get_element(env, forces, k, &f);
    char type[64] = {0};
    size_t len = 0;
    napi_get_value_string_utf8(env, property(env, f, "type"), type, sizeof(type), &len);
    size_t m = 0;
    if (!std::strcmp(type, "NonbondedForce")) {
      d->has_nonbonded = 1;
      d->cutoff = number(env, f, "cutoff", 1.0);
      d->ewald_tolerance = number(env, f, "ewaldTolerance", 5e-4);
      d->alpha = number(env, f, "alpha", 0);
      d->use_dispersion_correction = flag(env, f, "useDispersionCorrection", true) ? 1 : 0;
      d->charge = typed_array<double>(env, property(env, f, "charge"), &m);
      d->sigma = typed_array<double>(env, property(env, f, "sigma"), &m);
      d->epsilon = typed_array<double>(env, property(env, f, "epsilon"), &m);
      d->exception_p1 = typed_array<int32_t>(env, property(env, f, "exceptionP1"), &m);
      d->n_exceptions = int32_t(m);
      d->exception_p2 = typed_array<int32_t>(env, property(env, f, "exceptionP2"), &m);
      d->exception_charge_prod = typed_array<double>(env, property(env, f, "exceptionChargeProd"), &m);
      d->exception_sigma = typed_array<double>(env, property(env, f, "exceptionSigma"), &m);
      d->exception_epsilon = typed_array<double>(env, property(env, f, "exceptionEpsilon"), &m);
    } else if (!std::strcmp(type, "HarmonicBondForce")) {
      d->bond_p1 = typed_array<int32_t>(env, property(env, f, "p1"), &m);
      d->n_bonds = int32_t(m);
      d->bond_p2 = typed_array<int32_t>(env, property(env, f, "p2"), &m);
      d->bond_length = typed_array<double>(env, property(env, f, "length"), &m);
      d->bond_k = typed_array<double>(env, property(env, f, "k"), &m);
    } else if (!std::strcmp(type, "HarmonicAngleForce")) {
      d->angle_p1 = typed_array<int32_t>(env, property(env, f, "p1"), &m);
      d->n_angles = int32_t(m);
      d->angle_p2 = typed_array<int32_t>(env, property(env, f, "p2"), &m);
      d->angle_p3 = typed_array<int32_t>(env, property(env, f, "p3"), &m);
      d->angle_theta = typed_array<double>(env, property(env, f, "angle"), &m);
      d->angle_k = typed_array<double>(env, property(env, f, "k"), &m);
    } else if (!std::strcmp(type, "PeriodicTorsionForce")) {
      d->torsion_p1 = typed_array<int32_t>(env, property(env, f, "p1"), &m);
      d->n_torsions = int32_t(m);
      d->torsion_p2 = typed_array<int32_t>(env, property(env, f, "p2"), &m);
      d->torsion_p3 = typed_array<int32_t>(env, property(env, f, "p3"), &m);
      d->torsion_p4 = typed_array<int32_t>(env, property(env, f, "p4"), &m);
      d->torsion_periodicity = typed_array<int32_t>(env, property(env, f, "periodicity"), &m);
      d->torsion_phase = typed_array<double>(env, property(env, f, "phase"), &m);
      d->torsion_k = typed_array<double>(env, property(env, f, "k"), &m);
    } else if (!std::strcmp(type, "CMMotionRemover")) {
      d->com_frequency = int32_t(number(env, f, "frequency", 1));
    } else if (!std::strcmp(type, "MonteCarloBarostat")) {
      d->barostat_frequency = int32_t(number(env, f, "frequency", 25));
      d->barostat_pressure = number(env, f, "defaultPressure", 1);
      d->barostat_temperature = number(env, f, "defaultTemperature", 300);
    } else if (!std::strcmp(type, "PositionRestraint")) {
      // k*periodicdistance(x,y,z,x0,y0,z0)^2 per particle (system.ts:139-150)
      d->restraint_particle = typed_array<int32_t>(env, property(env, f, "particle"), &m);
      d->n_restraints = int32_t(m);
      d->restraint_k = typed_array<double>(env, property(env, f, "k"), &m);
      d->restraint_x0 = typed_array<double>(env, property(env, f, "x0"), &m);
      d->restraint_y0 = typed_array<double>(env, property(env, f, "y0"), &m);
      d->restraint_z0 = typed_array<double>(env, property(env, f, "z0"), &m);
    } else {
      unsupported = type;
      return false;
    }
  }
  (void)box;
  return d->n_particles > 0;
}

napi_value Create(napi_env env, napi_callback_info info) {
  size_t argc = 3;
  napi_value argv[3];
  napi_get_cb_info(env, info, &argc, argv, nullptr, nullptr);
  mdb_system_desc sys;
  std::vector<double> box;
  std::string unsupported;
  if (!fill_system(env, argv[0], &sys, box, unsupported)) {
    if (unsupported.empty()) return throw_status(env, MDB_ERR_INVALID_ARGUMENT, nullptr);
    napi_value message, error, name;
    const std::string text = unsupported + " is not implemented by this engine";
    napi_create_string_utf8(env, text.c_str(), NAPI_AUTO_LENGTH, &message);
    napi_create_error(env, nullptr, message, &error);
    napi_create_string_utf8(env, "UnsupportedForce", NAPI_AUTO_LENGTH, &name);
    napi_set_named_property(env, error, "name", name);
    napi_throw(env, error);
    return nullptr;
  }
  mdb_state_desc st;
  std::memset(&st, 0, sizeof(st));
  size_t n = 0;
  st.positions = typed_array<double>(env, property(env, argv[1], "positions"), &n);
  bool has_v = false;
  napi_has_named_property(env, argv[1], "velocities", &has_v);
  if (has_v) st.velocities = typed_array<double>(env, property(env, argv[1], "velocities"), &n);
  // the run's box is the State's (loop.ts:295), the System's default otherwise
  if (!read_box(env, argv[1], st.box)) std::memcpy(st.box, sys.box, sizeof(st.box));
  mdb_run_options o;
  std::memset(&o, 0, sizeof(o));
  o.time_step = number(env, argv[2], "timeStep", 0.002);
  o.temperature = number(env, argv[2], "temperature", 300);
  o.friction = number(env, argv[2], "friction", 1);
  o.constraint_tolerance = number(env, argv[2], "constraintTolerance", 1e-6);
  o.seed = uint32_t(number(env, argv[2], "seed", 0));
  o.verlet_skin = number(env, argv[2], "verletSkin", -1);
  o.max_batch = int32_t(number(env, argv[2], "maxBatch", 100));
  // the CUDA device: an extra member of the options object (the reference's
  // GPUDevice argument has no counterpart here); 0 when absent
  o.device = int32_t(number(env, argv[2], "device", 0));
  // RunOptions.integrator, "lfmiddle" or "verlet" (loop.ts:127)
  o.integrator = MDB_INTEGRATOR_LFMIDDLE;
  bool has_integrator = false;
  napi_has_named_property(env, argv[2], "integrator", &has_integrator);
  if (has_integrator) {
    char name[32] = {0};
    size_t len = 0;
    napi_get_value_string_utf8(env, property(env, argv[2], "integrator"), name, sizeof(name), &len);
    if (std::strcmp(name, "verlet") == 0) o.integrator = MDB_INTEGRATOR_VERLET;
    else if (std::strcmp(name, "lfmiddle") != 0)
      return throw_message(env, std::string("unknown integrator '") + name + "': expected lfmiddle or verlet");
  }
  // RunOptions.mesh, a pinned [x, y, z] PME mesh (loop.ts:167); absent = by rule
  bool has_mesh = false;
  napi_has_named_property(env, argv[2], "mesh", &has_mesh);
  if (has_mesh) {
    napi_value m = property(env, argv[2], "mesh");
    uint32_t len = 0;
    if (napi_get_array_length(env, m, &len) == napi_ok)
      for (uint32_t k = 0; k < 3 && k < len; ++k) {
        napi_value x;
        double v = 0;
        napi_get_element(env, m, k, &x);
        napi_get_value_double(env, x, &v);
        o.mesh[k] = int32_t(v);
      }
  }
  mdb_engine* e = nullptr;
  const int status = mdb_create(&sys, &st, &o, &e);
  if (status != MDB_OK) {
    napi_value r = throw_status(env, status, e);
    if (e) mdb_destroy(e, nullptr);
    return r;
  }
  napi_value handle;
  napi_create_external(env, e, nullptr, nullptr, &handle);
  return handle;
}

napi_value Run(napi_env env, napi_callback_info info) {
  size_t argc = 2;
  napi_value argv[2];
  napi_get_cb_info(env, info, &argc, argv, nullptr, nullptr);
  mdb_engine* e = engine_of(env, argv[0]);
  int64_t steps = 0;
  napi_get_value_int64(env, argv[1], &steps);
  const int status = mdb_run(e, steps);
  if (status != MDB_OK) return throw_status(env, status, e);
  return nullptr;
}

napi_value energies_object(napi_env env, const mdb_energies& en);

napi_value CopyOut(napi_env env, napi_callback_info info, int (*fn)(mdb_engine*, int32_t, double*)) {
  size_t argc = 2;
  napi_value argv[2];
  napi_get_cb_info(env, info, &argc, argv, nullptr, nullptr);
  mdb_engine* e = engine_of(env, argv[0]);
  size_t n = 0;
  double* out = typed_array<double>(env, argv[1], &n);
  const int status = fn(e, 0, out);
  if (status != MDB_OK) return throw_status(env, status, e);
  return nullptr;
}

napi_value Positions(napi_env env, napi_callback_info info) { return CopyOut(env, info, mdb_get_positions); }
napi_value Velocities(napi_env env, napi_callback_info info) { return CopyOut(env, info, mdb_get_velocities); }

napi_value Evaluate(napi_env env, napi_callback_info info) {
  size_t argc = 2;
  napi_value argv[2];
  napi_get_cb_info(env, info, &argc, argv, nullptr, nullptr);
  mdb_engine* e = engine_of(env, argv[0]);
  napi_valuetype t;
  napi_typeof(env, argv[1], &t);
  size_t n = 0;
  double* forces = t == napi_null ? nullptr : typed_array<double>(env, argv[1], &n);
  mdb_energies en;
  const int status = mdb_evaluate(e, 0, forces, &en);
  if (status != MDB_OK) return throw_status(env, status, e);
  return energies_object(env, en);
}

napi_value energies_object(napi_env env, const mdb_energies& en) {
  napi_value obj;
  napi_create_object(env, &obj);
  auto put = [&](const char* k, double v) {
    napi_value x;
    napi_create_double(env, v, &x);
    napi_set_named_property(env, obj, k, x);
  };
  put("potential", en.potential);
  put("kinetic", en.kinetic);
  put("temperature", en.temperature);
  put("directGroup", en.direct_group);
  put("reciprocalGroup", en.reciprocal_group);
  put("HarmonicBondForce", en.bond);
  put("HarmonicAngleForce", en.angle);
  put("PeriodicTorsionForce", en.torsion);
  return obj;
}

// potential(handle, positions, forces): the energies at `positions`, forces
// written into `forces`; the engine's own state is left as it was.
napi_value Potential(napi_env env, napi_callback_info info) {
  size_t argc = 3;
  napi_value argv[3];
  napi_get_cb_info(env, info, &argc, argv, nullptr, nullptr);
  mdb_engine* e = engine_of(env, argv[0]);
  size_t n = 0, m = 0;
  const double* positions = typed_array<double>(env, argv[1], &n);
  double* forces = typed_array<double>(env, argv[2], &m);
  mdb_energies en;
  const int status = mdb_potential(e, 0, positions, forces, &en);
  if (status != MDB_OK) return throw_status(env, status, e);
  return energies_object(env, en);
}

napi_value CopyIn(napi_env env, napi_callback_info info, int (*fn)(mdb_engine*, int32_t, const double*)) {
  size_t argc = 2;
  napi_value argv[2];
  napi_get_cb_info(env, info, &argc, argv, nullptr, nullptr);
  mdb_engine* e = engine_of(env, argv[0]);
  size_t n = 0;
  const double* in = typed_array<double>(env, argv[1], &n);
  const int status = fn(e, 0, in);
  if (status != MDB_OK) return throw_status(env, status, e);
  return nullptr;
}

napi_value SetPositions(napi_env env, napi_callback_info info) { return CopyIn(env, info, mdb_set_positions); }
napi_value SetVelocities(napi_env env, napi_callback_info info) { return CopyIn(env, info, mdb_set_velocities); }
napi_value SetBox(napi_env env, napi_callback_info info) { return CopyIn(env, info, mdb_set_box); }

// box(handle): the nine box vector components, rows a, b, c.
napi_value Box(napi_env env, napi_callback_info info) {
  size_t argc = 1;
  napi_value argv[1];
  napi_get_cb_info(env, info, &argc, argv, nullptr, nullptr);
  mdb_engine* e = engine_of(env, argv[0]);
  void* data = nullptr;
  napi_value buffer, array;
  napi_create_arraybuffer(env, 9 * sizeof(double), &data, &buffer);
  const int status = mdb_get_box(e, 0, static_cast<double*>(data));
  if (status != MDB_OK) return throw_status(env, status, e);
  napi_create_typedarray(env, napi_float64_array, 9, buffer, 0, &array);
  return array;
}

// mesh(handle): the PME mesh, three sizes.
napi_value Mesh(napi_env env, napi_callback_info info) {
  size_t argc = 1;
  napi_value argv[1];
  napi_get_cb_info(env, info, &argc, argv, nullptr, nullptr);
  mdb_engine* e = engine_of(env, argv[0]);
  void* data = nullptr;
  napi_value buffer, array;
  napi_create_arraybuffer(env, 3 * sizeof(int32_t), &data, &buffer);
  const int status = mdb_get_mesh(e, 0, static_cast<int32_t*>(data));
  if (status != MDB_OK) return throw_status(env, status, e);
  napi_create_typedarray(env, napi_int32_array, 3, buffer, 0, &array);
  return array;
}

napi_value SetStep(napi_env env, napi_callback_info info) {
  size_t argc = 2;
  napi_value argv[2];
  napi_get_cb_info(env, info, &argc, argv, nullptr, nullptr);
  mdb_engine* e = engine_of(env, argv[0]);
  int64_t step = 0;
  napi_get_value_int64(env, argv[1], &step);
  const int status = mdb_set_step(e, step);
  if (status != MDB_OK) return throw_status(env, status, e);
  return nullptr;
}

napi_value Step(napi_env env, napi_callback_info info) {
  size_t argc = 1;
  napi_value argv[1];
  napi_get_cb_info(env, info, &argc, argv, nullptr, nullptr);
  mdb_engine* e = engine_of(env, argv[0]);
  int64_t step = 0;
  const int status = mdb_get_step(e, &step);
  if (status != MDB_OK) return throw_status(env, status, e);
  napi_value v;
  napi_create_int64(env, step, &v);
  return v;
}

// barostat(handle): {attempts, accepted, volumeScale}, barostatStatistics' fields.
napi_value Barostat(napi_env env, napi_callback_info info) {
  size_t argc = 1;
  napi_value argv[1];
  napi_get_cb_info(env, info, &argc, argv, nullptr, nullptr);
  mdb_engine* e = engine_of(env, argv[0]);
  mdb_barostat_stats b;
  const int status = mdb_get_barostat_stats(e, 0, &b);
  if (status != MDB_OK) return throw_status(env, status, e);
  napi_value obj, v;
  napi_create_object(env, &obj);
  napi_create_int64(env, b.attempts, &v);
  napi_set_named_property(env, obj, "attempts", v);
  napi_create_int64(env, b.accepted, &v);
  napi_set_named_property(env, obj, "accepted", v);
  napi_create_double(env, b.volume_scale, &v);
  napi_set_named_property(env, obj, "volumeScale", v);
  return obj;
}

// neighbours(handle): verletFlags' fields (loop.ts:941) -- rebuilds,
// overflowed, capacity (tiles), skin (nm), byteLength (of the tile list) --
// plus the tile counts of the outer and inner lists and the prune count.
napi_value Neighbours(napi_env env, napi_callback_info info) {
  size_t argc = 1;
  napi_value argv[1];
  napi_get_cb_info(env, info, &argc, argv, nullptr, nullptr);
  mdb_engine* e = engine_of(env, argv[0]);
  mdb_neighbour_stats ns;
  const int status = mdb_get_neighbour_stats(e, 0, &ns);
  if (status != MDB_OK) return throw_status(env, status, e);
  napi_value obj, v;
  napi_create_object(env, &obj);
  napi_create_int64(env, ns.rebuilds, &v);
  napi_set_named_property(env, obj, "rebuilds", v);
  napi_create_int64(env, ns.tiles, &v);
  napi_set_named_property(env, obj, "tiles", v);
  napi_get_boolean(env, ns.overflowed != 0, &v);
  napi_set_named_property(env, obj, "overflowed", v);
  napi_create_int64(env, ns.tile_capacity, &v);
  napi_set_named_property(env, obj, "capacity", v);
  napi_create_double(env, ns.skin, &v);
  napi_set_named_property(env, obj, "skin", v);
  // a tile is its cluster pair (8 B), image shift (16 B) and interaction mask
  napi_create_int64(env, ns.tile_capacity * (24 + int64_t(ns.tile_atoms) * ns.tile_atoms / 8), &v);
  napi_set_named_property(env, obj, "byteLength", v);
  napi_create_int64(env, ns.inner_tiles, &v);
  napi_set_named_property(env, obj, "innerTiles", v);
  napi_create_int64(env, ns.prunes, &v);
  napi_set_named_property(env, obj, "prunes", v);
  return obj;
}

// cellGeometry(handle): {divisions, extent}, `StepLoop.cellGeometry()` (loop.ts:894).
napi_value CellGeometry(napi_env env, napi_callback_info info) {
  size_t argc = 1;
  napi_value argv[1];
  napi_get_cb_info(env, info, &argc, argv, nullptr, nullptr);
  mdb_engine* e = engine_of(env, argv[0]);
  int32_t div[3] = {0, 0, 0};
  double ext[3] = {0, 0, 0};
  const int status = mdb_get_cell_geometry(e, 0, div, ext);
  if (status != MDB_OK) return throw_status(env, status, e);
  napi_value obj, divisions, extent, v;
  napi_create_object(env, &obj);
  napi_create_array_with_length(env, 3, &divisions);
  napi_create_array_with_length(env, 3, &extent);
  for (uint32_t k = 0; k < 3; ++k) {
    napi_create_int32(env, div[k], &v);
    napi_set_element(env, divisions, k, v);
    napi_create_double(env, ext[k], &v);
    napi_set_element(env, extent, k, v);
  }
  napi_set_named_property(env, obj, "divisions", divisions);
  napi_set_named_property(env, obj, "extent", extent);
  return obj;
}

// passesPerStep(handle): kernel launches one step makes (loop.ts:1105).
napi_value PassesPerStep(napi_env env, napi_callback_info info) {
  size_t argc = 1;
  napi_value argv[1];
  napi_get_cb_info(env, info, &argc, argv, nullptr, nullptr);
  mdb_engine* e = engine_of(env, argv[0]);
  int32_t n = 0;
  const int status = mdb_get_passes_per_step(e, &n);
  if (status != MDB_OK) return throw_status(env, status, e);
  napi_value v;
  napi_create_int32(env, n, &v);
  return v;
}

// memory(handle): {count, totalBytes}, the engine's device allocations for
// `report_pool()` (every allocation is a named one; there is no scratch pool).
napi_value Memory(napi_env env, napi_callback_info info) {
  size_t argc = 1;
  napi_value argv[1];
  napi_get_cb_info(env, info, &argc, argv, nullptr, nullptr);
  mdb_engine* e = engine_of(env, argv[0]);
  int64_t total = 0;
  const int status = mdb_memory_report(e, nullptr, 0, &total);
  if (status != MDB_OK) return throw_status(env, status, e);
  std::vector<char> text(1 << 16);
  mdb_memory_report(e, text.data(), int64_t(text.size()), nullptr);
  int64_t count = 0;
  for (const char* c = text.data(); *c; ++c) count += *c == ';';
  napi_value obj, v;
  napi_create_object(env, &obj);
  napi_create_int64(env, count, &v);
  napi_set_named_property(env, obj, "count", v);
  napi_create_int64(env, total, &v);
  napi_set_named_property(env, obj, "totalBytes", v);
  return obj;
}

napi_value Destroy(napi_env env, napi_callback_info info) {
  size_t argc = 1;
  napi_value argv[1];
  napi_get_cb_info(env, info, &argc, argv, nullptr, nullptr);
  int64_t leaked = 0;
  mdb_destroy(engine_of(env, argv[0]), &leaked);
  napi_value obj, v;
  napi_create_object(env, &obj);
  napi_create_int64(env, leaked, &v);
  napi_set_named_property(env, obj, "leaked", v);
  return obj;
}

napi_value Init(napi_env env, napi_value exports) {
  const napi_property_descriptor props[] = {
      {"create", nullptr, Create, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"run", nullptr, Run, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"positions", nullptr, Positions, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"velocities", nullptr, Velocities, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"evaluate", nullptr, Evaluate, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"potential", nullptr, Potential, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"setPositions", nullptr, SetPositions, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"setVelocities", nullptr, SetVelocities, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"setBox", nullptr, SetBox, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"box", nullptr, Box, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"mesh", nullptr, Mesh, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"setStep", nullptr, SetStep, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"step", nullptr, Step, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"barostat", nullptr, Barostat, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"neighbours", nullptr, Neighbours, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"cellGeometry", nullptr, CellGeometry, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"passesPerStep", nullptr, PassesPerStep, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"memory", nullptr, Memory, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"destroy", nullptr, Destroy, nullptr, nullptr, nullptr, napi_default, nullptr},
  };
  napi_define_properties(env, exports, sizeof(props) / sizeof(props[0]), props);
  return exports;
}

}  // namespace

NAPI_MODULE(NODE_GYP_MODULE_NAME, Init)
