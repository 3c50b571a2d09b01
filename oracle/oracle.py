"""TEST INFRASTRUCTURE: ctypes wrapper of the CPU f64 oracle (oracle.cpp).

The oracle restates the reference's own f64 path (src/reference/ of
making-it-rain-webgpu) in C++.  Only tests/, the smoke check and bench.py's
CPU-baseline leg import this module, and only as the checker or the timed CPU
baseline; the engine never does.  Parity is pinned by tests/test_oracle.py
against the reference's golden vectors in tests/golden/.
"""

from __future__ import annotations

import ctypes as C
import subprocess
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIBRARY = HERE / "_build" / "liboracle.so"
sys.path.insert(0, str(HERE.parent / "making-it-rain-webgpu_b200"))

from mdb200 import abi  # noqa: E402  (struct layouts shared with the engine ABI)
from mdb200.system import State, System  # noqa: E402


class Energies(C.Structure):
    _fields_ = [(name, C.c_double) for name in (
        "bond", "angle", "torsion", "restraint", "direct_coulomb", "direct_lj",
        "exclusion_correction", "exceptions", "dispersion", "reciprocal_mesh",
        "self_energy", "net_charge", "direct_group", "reciprocal_group", "potential")] + [
        ("pairs_within_cutoff", C.c_int64)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class StepOptions(C.Structure):
    _fields_ = [("time_step", C.c_double), ("temperature", C.c_double), ("friction", C.c_double),
                ("constraint_tolerance", C.c_double), ("seed", C.c_uint32), ("integrator", C.c_int32),
                ("grid", C.c_int32 * 3), ("threads", C.c_int32)]


_lib = None
_dp = C.POINTER(C.c_double)
_SD = C.POINTER(abi.SystemDesc)


def build() -> Path:
    """Compile the oracle with its Makefile (g++, OpenMP)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIBRARY


def lib() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not LIBRARY.exists():
        build()
    L = C.CDLL(str(LIBRARY))
    sig = {
        "orc_ewald_alpha": (C.c_double, [C.c_double, C.c_double]),
        "orc_pme_minimum_grid": (C.c_int32, [C.c_double, C.c_double, C.c_double]),
        "orc_smooth_fft_size": (C.c_int32, [C.c_int32]),
        "orc_erf": (C.c_double, [C.c_double]),
        "orc_erfc": (C.c_double, [C.c_double]),
        "orc_erf_derivative": (C.c_double, [C.c_double]),
        "orc_fixed_words": (C.c_int32, [C.c_float, C.POINTER(C.c_uint32), C.POINTER(C.c_int32)]),
        "orc_from_fixed_f32": (C.c_float, [C.c_int64]),
        "orc_from_fixed": (C.c_double, [C.c_int64]),
        "orc_threefry2x32": (None, [C.c_uint32] * 4 + [C.c_int32, C.POINTER(C.c_uint32)]),
        "orc_open_unit_interval": (C.c_double, [C.c_uint32]),
        "orc_thermostat_normal": (C.c_double, [C.c_uint32, C.c_uint32, C.c_uint32, C.c_int32]),
        "orc_domain_normal": (C.c_double, [C.c_uint32, C.c_uint32, C.c_uint32, C.c_int32]),
        "orc_reduce_box": (C.c_int32, [_dp, _dp]),
        "orc_perpendicular_widths": (None, [_dp, _dp]),
        "orc_box_volume": (C.c_double, [_dp]),
        "orc_minimum_image": (None, [_dp, _dp, _dp]),
        "orc_nearest_image_by_search": (None, [_dp, _dp, _dp]),
        "orc_bspline": (None, [C.c_double, _dp, _dp]),
        "orc_bspline_moduli": (None, [C.c_int32, _dp]),
        "orc_potential": (C.c_int32, [_SD, _dp, _dp, C.POINTER(C.c_int32), C.c_int32, C.c_int32, _dp,
                                      C.POINTER(Energies)]),
        "orc_mlp_gradient": (C.c_int32, [C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float),
                                         C.c_int32, _dp, _dp]),
        "orc_potential_virial": (C.c_int32, [_SD, _dp, _dp, C.POINTER(C.c_int32), C.c_int32, _dp,
                                             C.POINTER(Energies), _dp]),
        "orc_cutoff_shell": (C.c_int32, [_SD, _dp, _dp, C.c_double, C.c_int32, C.POINTER(C.c_int32),
                                         C.POINTER(C.c_int32), _dp, C.POINTER(C.c_int32)]),
        "orc_ewald_reciprocal": (C.c_int32, [_SD, _dp, _dp, C.c_double, C.c_int32, _dp, _dp]),
        "orc_split_counts": (C.c_int32, [_SD] + [C.POINTER(C.c_int32)] * 4),
        "orc_degrees_of_freedom": (C.c_double, [_SD]),
        "orc_kinetic_energy": (C.c_double, [_SD, _dp]),
        "orc_remove_com": (None, [_SD, _dp]),
        "orc_constrain_positions": (C.c_int32, [_SD, _dp, _dp, C.c_double]),
        "orc_constrain_velocities": (C.c_int32, [_SD, _dp, _dp, C.c_double]),
        "orc_run": (C.c_int32, [_SD, _dp, _dp, _dp, C.POINTER(StepOptions), C.POINTER(C.c_int64), C.c_int64]),
        "orc_molecule_count": (C.c_int32, [_SD]),
        "orc_scale_molecules": (None, [_SD, _dp, C.c_double]),
        "orc_velocities_at_temperature": (None, [_SD, _dp, C.c_double, C.c_uint32, _dp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def _p(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def _box(box) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(box, dtype=np.float64).reshape(9))


def potential(system: System, positions, box=None, grid=None, threads: int = 1, naive: bool = False,
              forces: bool = True):
    """Energies by group and forces (N, 3), in f64 (potential.ts:94)."""
    handle = system.desc()
    pos = np.ascontiguousarray(np.asarray(positions, dtype=np.float64).reshape(-1))
    b = _box(system.box if box is None else box)
    f = np.zeros_like(pos) if forces else None
    e = Energies()
    g = (C.c_int32 * 3)(*(grid if grid is not None else (0, 0, 0)))
    status = lib().orc_potential(handle.pointer(), _p(pos), _p(b), g, threads, int(naive),
                                 _p(f) if f is not None else _dp(), C.byref(e))
    if status != 0:
        raise RuntimeError(f"oracle potential failed with status {status}")
    return e.as_dict(), (f.reshape(-1, 3) if f is not None else None)


def potential_virial(system: System, positions, box=None, grid=None, threads: int = 1):
    """Energies, forces (N, 3) and the 3x3 virial W_ab = sum r_a F_b = -dU/d eps_ab."""
    handle = system.desc()
    pos = np.ascontiguousarray(np.asarray(positions, dtype=np.float64).reshape(-1))
    b = _box(system.box if box is None else box)
    f = np.zeros_like(pos)
    w = np.zeros(9)
    e = Energies()
    g = (C.c_int32 * 3)(*(grid if grid is not None else (0, 0, 0)))
    status = lib().orc_potential_virial(handle.pointer(), _p(pos), _p(b), g, threads, _p(f), C.byref(e), _p(w))
    if status != 0:
        raise RuntimeError(f"oracle potential failed with status {status}")
    return e.as_dict(), f.reshape(-1, 3), w.reshape(3, 3)


def cutoff_shell(system: System, positions, box=None, eps: float = 2e-7):
    """Pairs within `eps` nm of the cutoff: (first, second, force on first if
    inside (k, 3), inside in f64 (k,) bool)."""
    pos = np.ascontiguousarray(np.asarray(positions, dtype=np.float64).reshape(-1))
    b = _box(system.box if box is None else box)
    cap = 64
    while True:
        i = np.zeros(cap, np.int32)
        j = np.zeros(cap, np.int32)
        f = np.zeros(3 * cap)
        inside = np.zeros(cap, np.int32)
        ip = C.POINTER(C.c_int32)
        k = lib().orc_cutoff_shell(system.desc().pointer(), _p(pos), _p(b), eps, cap, i.ctypes.data_as(ip),
                                   j.ctypes.data_as(ip), _p(f), inside.ctypes.data_as(ip))
        if k <= cap:
            return i[:k], j[:k], f.reshape(-1, 3)[:k], inside[:k].astype(bool)
        cap = k


def mlp_gradient(params, x, t):
    """f64 loss and gradient of the screening network (first min(n, 128) samples)."""
    p = np.ascontiguousarray(params, dtype=np.float32)
    xx = np.ascontiguousarray(x, dtype=np.float32)
    tt = np.ascontiguousarray(t, dtype=np.float32)
    g = np.zeros(p.size)
    loss = C.c_double()
    fp = C.POINTER(C.c_float)
    status = lib().orc_mlp_gradient(p.ctypes.data_as(fp), xx.ctypes.data_as(fp), tt.ctypes.data_as(fp),
                                    int(tt.size), _p(g), C.byref(loss))
    if status != 0:
        raise RuntimeError(f"oracle mlp gradient failed with status {status}")
    return loss.value, g


def ewald_reciprocal(system: System, positions, alpha: float, kmax: int, box=None):
    handle = system.desc()
    pos = np.ascontiguousarray(np.asarray(positions, dtype=np.float64).reshape(-1))
    f = np.zeros_like(pos)
    e = C.c_double()
    lib().orc_ewald_reciprocal(handle.pointer(), _p(pos), _p(_box(system.box if box is None else box)),
                               alpha, kmax, _p(f), C.byref(e))
    return e.value, f.reshape(-1, 3)


def run(system: System, state: State, steps: int, *, time_step=0.002, temperature=300.0, friction=1.0,
        constraint_tolerance=1e-6, seed=0, integrator=0, grid=None, threads=1):
    """`steps` oracle steps from `state`; returns (positions, velocities, step)."""
    handle = system.desc()
    pos = np.ascontiguousarray(np.asarray(state.positions, dtype=np.float64).reshape(-1)).copy()
    vel = (np.zeros_like(pos) if state.velocities is None
           else np.ascontiguousarray(np.asarray(state.velocities, dtype=np.float64).reshape(-1)).copy())
    o = StepOptions(time_step, temperature, friction, constraint_tolerance, seed, integrator,
                    (C.c_int32 * 3)(*(grid if grid is not None else (0, 0, 0))), threads)
    step = C.c_int64(int(state.step))
    status = lib().orc_run(handle.pointer(), _p(pos), _p(vel), _p(_box(state.box)), C.byref(o),
                           C.byref(step), steps)
    if status not in (0, 5):
        raise RuntimeError(f"oracle run failed with status {status}")
    return pos.reshape(-1, 3), vel.reshape(-1, 3), step.value


def velocities_at_temperature(system: System, positions, temperature: float, seed: int) -> np.ndarray:
    handle = system.desc()
    pos = np.ascontiguousarray(np.asarray(positions, dtype=np.float64).reshape(-1))
    out = np.zeros_like(pos)
    lib().orc_velocities_at_temperature(handle.pointer(), _p(pos), temperature, seed, _p(out))
    return out.reshape(-1, 3)


def kinetic_energy(system: System, velocities) -> float:
    v = np.ascontiguousarray(np.asarray(velocities, dtype=np.float64).reshape(-1))
    return lib().orc_kinetic_energy(system.desc().pointer(), _p(v))


def degrees_of_freedom(system: System) -> float:
    return lib().orc_degrees_of_freedom(system.desc().pointer())


def split_counts(system: System):
    vals = [C.c_int32() for _ in range(4)]
    status = lib().orc_split_counts(system.desc().pointer(), *[C.byref(v) for v in vals])
    return status, [v.value for v in vals]


def scale_molecules(system: System, positions, scale: float) -> np.ndarray:
    pos = np.ascontiguousarray(np.asarray(positions, dtype=np.float64).reshape(-1)).copy()
    lib().orc_scale_molecules(system.desc().pointer(), _p(pos), scale)
    return pos.reshape(-1, 3)
