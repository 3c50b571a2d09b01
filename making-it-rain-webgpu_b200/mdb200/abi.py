"""ctypes mirror of include/mdb.h, and the loader for the engine library.

The engine is `lib/libmdb200.so`, built in-tree from `csrc/` for sm_100a.
Loading fails loudly when it is missing: there is no CPU fallback anywhere in
this package, by design.
"""

from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

PACKAGE_ROOT = Path(__file__).resolve().parent.parent
LIBRARY_PATH = PACKAGE_ROOT / "lib" / "libmdb200.so"

ABI_VERSION = 3

# mdb_status
OK = 0
ERR_INVALID_ARGUMENT = 1
ERR_UNSUPPORTED_FORCE = 2
ERR_CUTOFF_TOO_LARGE_FOR_BOX = 3
ERR_CLUSTER_TOO_LARGE = 4
ERR_NOT_CONVERGED = 5
ERR_CAPACITY = 6
ERR_RANGE = 7
ERR_DEVICE = 8
ERR_TIMEOUT = 9
ERR_NO_DEVICE = 10
ERR_NOT_SMOOTH = 11
ERR_DEVICE_LOST = 12

INTEGRATOR_LFMIDDLE = 0
INTEGRATOR_VERLET = 1

FLAG_NO_GRAPH = 1
FLAG_ALWAYS_REBUILD = 2
FLAG_PHASE_LAUNCHES = 4

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


class SystemDesc(C.Structure):
    """`mdb_system_desc`."""

    _fields_ = [
        ("n_particles", C.c_int32),
        ("masses", _dp),
        ("box", C.c_double * 9),
        ("n_constraints", C.c_int32),
        ("constraint_p1", _ip),
        ("constraint_p2", _ip),
        ("constraint_distance", _dp),
        ("has_nonbonded", C.c_int32),
        ("cutoff", C.c_double),
        ("ewald_tolerance", C.c_double),
        ("alpha", C.c_double),
        ("grid", C.c_int32 * 3),
        ("use_dispersion_correction", C.c_int32),
        ("charge", _dp),
        ("sigma", _dp),
        ("epsilon", _dp),
        ("n_exceptions", C.c_int32),
        ("exception_p1", _ip),
        ("exception_p2", _ip),
        ("exception_charge_prod", _dp),
        ("exception_sigma", _dp),
        ("exception_epsilon", _dp),
        ("n_bonds", C.c_int32),
        ("bond_p1", _ip),
        ("bond_p2", _ip),
        ("bond_length", _dp),
        ("bond_k", _dp),
        ("n_angles", C.c_int32),
        ("angle_p1", _ip),
        ("angle_p2", _ip),
        ("angle_p3", _ip),
        ("angle_theta", _dp),
        ("angle_k", _dp),
        ("n_torsions", C.c_int32),
        ("torsion_p1", _ip),
        ("torsion_p2", _ip),
        ("torsion_p3", _ip),
        ("torsion_p4", _ip),
        ("torsion_periodicity", _ip),
        ("torsion_phase", _dp),
        ("torsion_k", _dp),
        ("com_frequency", C.c_int32),
        ("barostat_frequency", C.c_int32),
        ("barostat_pressure", C.c_double),
        ("barostat_temperature", C.c_double),
        ("n_restraints", C.c_int32),
        ("restraint_particle", _ip),
        ("restraint_k", _dp),
        ("restraint_x0", _dp),
        ("restraint_y0", _dp),
        ("restraint_z0", _dp),
    ]


class StateDesc(C.Structure):
    """`mdb_state_desc`."""

    _fields_ = [
        ("positions", _dp),
        ("velocities", _dp),
        ("box", C.c_double * 9),
        ("step", C.c_int64),
    ]


class Tuning(C.Structure):
    """`mdb_tuning` (no reference counterpart)."""

    _fields_ = [("verlet_skin", C.c_double), ("sort_cell", C.c_double), ("tile_atoms", C.c_int32),
                ("prune_tiles", C.c_int32), ("inner_skin", C.c_double)]


class RunOptions(C.Structure):
    """`mdb_run_options`."""

    _fields_ = [
        ("time_step", C.c_double),
        ("temperature", C.c_double),
        ("friction", C.c_double),
        ("constraint_tolerance", C.c_double),
        ("seed", C.c_uint32),
        ("integrator", C.c_int32),
        ("verlet_skin", C.c_double),
        ("max_batch", C.c_int32),
        ("mesh", C.c_int32 * 3),
        ("device", C.c_int32),
        ("flags", C.c_int32),
        ("tuning", C.POINTER(Tuning)),
        ("surrogate_attempts", C.c_int32),
        ("tile_row_capacity", C.c_int32),
    ]


class Energies(C.Structure):
    """`mdb_energies`."""

    _fields_ = [
        ("bond", C.c_double),
        ("angle", C.c_double),
        ("torsion", C.c_double),
        ("restraint", C.c_double),
        ("direct_coulomb", C.c_double),
        ("direct_lj", C.c_double),
        ("exclusion_correction", C.c_double),
        ("exceptions", C.c_double),
        ("dispersion", C.c_double),
        ("reciprocal_mesh", C.c_double),
        ("self_energy", C.c_double),
        ("net_charge", C.c_double),
        ("direct_group", C.c_double),
        ("reciprocal_group", C.c_double),
        ("potential", C.c_double),
        ("kinetic", C.c_double),
        ("temperature", C.c_double),
        ("degrees_of_freedom", C.c_double),
        ("virial", C.c_double * 9),
        ("pairs_within_cutoff", C.c_double),
        ("molecular_virial", C.c_double * 9),
    ]

    def as_dict(self) -> dict:
        out = {name: getattr(self, name) for name, _ in self._fields_ if name not in ("virial", "molecular_virial")}
        out["virial"] = list(self.virial)
        out["molecular_virial"] = list(self.molecular_virial)
        return out


class BarostatStats(C.Structure):
    _fields_ = [
        ("attempts", C.c_int64),
        ("accepted", C.c_int64),
        ("volume_scale", C.c_double),
        ("screened", C.c_int64),
        ("exact_evaluations", C.c_int64),
        ("training_samples", C.c_int64),
        ("surrogate_active", C.c_int32),
        ("surrogate_disabled", C.c_int32),
        ("surrogate_rms", C.c_double),
        ("training_loss", C.c_double),
        ("training_ms", C.c_double),
    ]


class Profile(C.Structure):
    """`mdb_profile`."""

    _fields_ = [
        ("launches_per_step", C.c_int32),
        ("repeats", C.c_int32),
        ("ms_step", C.c_double),
        ("ms_list_check", C.c_double),
        ("ms_list_rebuild", C.c_double),
        ("ms_nonbonded", C.c_double),
        ("ms_listed", C.c_double),
        ("ms_pme", C.c_double),
        ("ms_pme_spread", C.c_double),
        ("ms_pme_fft", C.c_double),
        ("ms_pme_gather", C.c_double),
        ("ms_integrate", C.c_double),
        ("pairs_within_cutoff", C.c_int64),
        ("tiles", C.c_int64),
        ("atoms", C.c_int64),
        ("mesh_points", C.c_int64),
        ("inner_tiles", C.c_int64),
        ("ms_inner_prune", C.c_double),
        ("tile_atoms", C.c_int64),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class NeighbourStats(C.Structure):
    _fields_ = [
        ("rebuilds", C.c_int64),
        ("tiles", C.c_int64),
        ("tile_capacity", C.c_int64),
        ("blocks", C.c_int64),
        ("overflowed", C.c_int32),
        ("skin", C.c_double),
        ("inner_tiles", C.c_int64),
        ("prunes", C.c_int64),
        ("inner_skin", C.c_double),
        ("tile_atoms", C.c_int32),
        ("list_grown", C.c_int64),
    ]


# Every entry point include/mdb.h declares, with its ctypes signature.
_E = C.c_void_p
EXPORTS = {
    "mdb_abi_version": (C.c_int, []),
    "mdb_status_string": (C.c_char_p, [C.c_int]),
    "mdb_device_count": (C.c_int, [_ip]),
    "mdb_create": (C.c_int, [C.POINTER(SystemDesc), C.POINTER(StateDesc), C.POINTER(RunOptions), C.POINTER(_E)]),
    "mdb_batch_create": (
        C.c_int,
        [C.c_int32, C.POINTER(SystemDesc), C.POINTER(StateDesc), C.POINTER(RunOptions), C.POINTER(_E)],
    ),
    "mdb_destroy": (C.c_int, [_E, C.POINTER(C.c_int64)]),
    "mdb_last_error": (C.c_char_p, [_E]),
    "mdb_system_count": (C.c_int, [_E, _ip]),
    "mdb_run": (C.c_int, [_E, C.c_int64]),
    "mdb_run_timed": (C.c_int, [_E, C.c_int64, _dp]),
    "mdb_set_step": (C.c_int, [_E, C.c_int64]),
    "mdb_get_step": (C.c_int, [_E, C.POINTER(C.c_int64)]),
    "mdb_get_positions": (C.c_int, [_E, C.c_int32, _dp]),
    "mdb_get_velocities": (C.c_int, [_E, C.c_int32, _dp]),
    "mdb_set_positions": (C.c_int, [_E, C.c_int32, _dp]),
    "mdb_set_velocities": (C.c_int, [_E, C.c_int32, _dp]),
    "mdb_set_box": (C.c_int, [_E, C.c_int32, _dp]),
    "mdb_get_box": (C.c_int, [_E, C.c_int32, _dp]),
    "mdb_get_mesh": (C.c_int, [_E, C.c_int32, _ip]),
    "mdb_evaluate": (C.c_int, [_E, C.c_int32, _dp, C.POINTER(Energies)]),
    "mdb_potential": (C.c_int, [_E, C.c_int32, _dp, _dp, C.POINTER(Energies)]),
    "mdb_get_barostat_stats": (C.c_int, [_E, C.c_int32, C.POINTER(BarostatStats)]),
    "mdb_get_neighbour_stats": (C.c_int, [_E, C.c_int32, C.POINTER(NeighbourStats)]),
    "mdb_get_cell_geometry": (C.c_int, [_E, C.c_int32, _ip, C.POINTER(C.c_double)]),
    "mdb_get_passes_per_step": (C.c_int, [_E, _ip]),
    "mdb_memory_report": (C.c_int, [_E, C.c_char_p, C.c_int64, C.POINTER(C.c_int64)]),
    "mdb_profile_step": (C.c_int, [_E, C.c_int32, C.POINTER(Profile)]),
    "mdb_mlp_gradient": (C.c_int, [C.POINTER(C.c_float)] * 3 + [C.c_int32, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "mdb_mlp_fit": (C.c_int, [C.POINTER(C.c_float)] * 2 + [C.c_int32, C.c_int32, C.c_uint32, C.POINTER(C.c_float),
                                                        C.POINTER(C.c_float)]),
    "mdb_mlp_predict": (C.c_int, [C.POINTER(C.c_float)] * 2 + [C.c_int32, C.POINTER(C.c_float)]),
    "mdb_autotune": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(RunOptions), C.c_int32, C.POINTER(Tuning),
                               C.POINTER(C.c_double), C.POINTER(C.c_int32)]),
    "mdb_autotune_batch": (C.c_int, [C.c_int32, C.c_void_p, C.c_void_p, C.POINTER(RunOptions), C.c_int32,
                                     C.POINTER(Tuning), C.POINTER(C.c_double), C.POINTER(C.c_int32)]),
    "mdb_reciprocal_noalloc": (
        C.c_int,
        [C.c_int32, C.c_void_p, C.c_void_p, _dp, C.c_double, _ip, C.c_void_p, C.c_void_p, C.c_void_p],
    ),
}

_library = None


class EngineLibraryMissing(RuntimeError):
    """The CUDA engine library has not been built, or cannot be loaded."""


def load(path: os.PathLike | str | None = None) -> C.CDLL:
    """Load libmdb200 and declare every exported signature.

    Raises `EngineLibraryMissing` rather than returning anything that could be
    mistaken for a working engine.
    """
    global _library
    if _library is not None and path is None:
        return _library
    target = Path(path) if path is not None else LIBRARY_PATH
    if not target.exists():
        raise EngineLibraryMissing(
            f"{target} is not built. Run `python making-it-rain-webgpu_b200/build.py` "
            "(nvcc for sm_100a); this package has no "
            "CPU fallback."
        )
    try:
        lib = C.CDLL(str(target))
    except OSError as error:  # pragma: no cover - depends on the box
        raise EngineLibraryMissing(f"{target} failed to load: {error}") from error
    for name, (restype, argtypes) in EXPORTS.items():
        fn = getattr(lib, name)
        fn.restype = restype
        fn.argtypes = argtypes
    if lib.mdb_abi_version() != ABI_VERSION:
        raise EngineLibraryMissing(
            f"{target} reports ABI {lib.mdb_abi_version()}, expected {ABI_VERSION}"
        )
    if path is None:
        _library = lib
    return lib
