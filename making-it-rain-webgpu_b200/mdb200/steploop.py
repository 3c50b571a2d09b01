"""`StepLoop` over the C ABI: the reference's engine surface, in Python.

Mirrors the public members of `StepLoop` (src/gpu/loop.ts:208-1116, paths
relative to the reference project root) and its `Report` (loop.ts:173-199):
`create` / `from_parsed`, `run`, `report`, `potential`, `positions`,
`velocities`, `set_positions`, `set_velocities`, `set_box`,
`advance_step_count`, `steps`, `barostat_statistics`, `mesh`,
`box_vectors`, `verlet_flags`, `cell_geometry`, `passes_per_step`,
`profile_step`, `destroy`.  The per-group evaluators
`evaluateDirectSpace` / `evaluateReciprocalSpace` / `evaluateBondedForce`
become `evaluate()`.  Failures raise the reference's named errors.

Every call goes to libmdb200 (CUDA, sm_100a).  There is no CPU path.
"""

from __future__ import annotations

import ctypes as C
import dataclasses
import json
import math
import os
from pathlib import Path
from typing import Optional, Sequence

import numpy as np

from . import abi
from .system import State, System, UnsupportedForce, parse_state, parse_system

BOLTZMANN = 0.008314462618153242


class EngineError(RuntimeError):
    """A failure reported by the engine, with its status code."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{message} (status {status})")
        self.status = status


class CutoffTooLargeForBox(EngineError):
    """src/reference/triclinic.ts:179."""


class ClusterTooLarge(EngineError):
    """src/engine/constraint-clusters.ts:71."""


class NotSmooth(EngineError):
    """src/reference/fft.ts:24."""


class NoDevice(EngineError):
    """No CUDA device is visible."""


_ERRORS = {
    abi.ERR_CUTOFF_TOO_LARGE_FOR_BOX: CutoffTooLargeForBox,
    abi.ERR_CLUSTER_TOO_LARGE: ClusterTooLarge,
    abi.ERR_NOT_SMOOTH: NotSmooth,
    abi.ERR_NO_DEVICE: NoDevice,
}


@dataclasses.dataclass
class RunOptions:
    """`RunOptions`, src/gpu/loop.ts:117-168."""

    time_step: float = 0.002
    temperature: float = 300.0
    friction: float = 1.0
    constraint_tolerance: float = 1e-6
    seed: int = 0
    integrator: str = "lfmiddle"
    verlet_skin: Optional[float] = None
    max_batch: int = 100
    mesh: Optional[Sequence[int]] = None
    device: int = 0
    graphs: bool = True
    always_rebuild: bool = False
    phase_launches: bool = False  # list build as separate launches (profiling)
    # per-system (verlet_skin, sort_cell[, tile_atoms[, prune_tiles]]) from `autotune`; None = defaults
    tuning: Optional[Sequence[tuple]] = None
    # > 0: each barostat learns a screening network from that many exact
    # attempts, then screens proposals by delayed acceptance
    surrogate_attempts: int = 0
    # starting capacity of the tile list, tiles per cluster; 0 = default
    # (a list that needs more is grown and rebuilt before a step uses it)
    tile_row_capacity: int = 0

    def to_c(self) -> abi.RunOptions:
        o = abi.RunOptions()
        o.time_step = self.time_step
        o.temperature = self.temperature
        o.friction = self.friction
        o.constraint_tolerance = self.constraint_tolerance
        o.seed = int(self.seed) & 0xFFFFFFFF
        o.integrator = abi.INTEGRATOR_VERLET if self.integrator == "verlet" else abi.INTEGRATOR_LFMIDDLE
        o.verlet_skin = -1.0 if self.verlet_skin is None else float(self.verlet_skin)
        o.max_batch = int(self.max_batch)
        o.mesh[:] = list(self.mesh) if self.mesh is not None else [0, 0, 0]
        o.device = int(self.device)
        o.flags = ((0 if self.graphs else abi.FLAG_NO_GRAPH) | (abi.FLAG_ALWAYS_REBUILD if self.always_rebuild else 0)
                   | (abi.FLAG_PHASE_LAUNCHES if self.phase_launches else 0))
        o.surrogate_attempts = int(self.surrogate_attempts)
        o.tile_row_capacity = int(self.tile_row_capacity)
        if self.tuning is not None:
            arr = (abi.Tuning * len(self.tuning))(*[abi.Tuning(float(t[0]), float(t[1]),
                                                               int(t[2]) if len(t) > 2 else 0,
                                                               int(t[3]) if len(t) > 3 else 0,
                                                               float(t[4]) if len(t) > 4 else 0.0)
                                                    for t in self.tuning])
            o.tuning = C.cast(arr, C.POINTER(abi.Tuning))
            o._keep = arr  # the array must outlive the create call
        return o


@dataclasses.dataclass
class Report:
    """`Report`, src/gpu/loop.ts:173-199."""

    step: int
    time: float
    potential_energy: float
    kinetic_energy: float
    temperature: float
    energies: dict


class StepLoop:
    """One engine: a single system, or a batch of independent ones."""

    def __init__(self, handle: C.c_void_p, lib: C.CDLL, systems: list, states: list, options: RunOptions):
        self._handle = handle
        self._lib = lib
        self._systems = systems
        self._options = options
        self._start_step = int(states[0].step)
        self._destroyed = False

    # ---- construction ----------------------------------------------------
    @classmethod
    def create(cls, system_xml: str, state_xml: str, options: RunOptions | None = None) -> "StepLoop":
        """`StepLoop.create`, loop.ts:268 -- from OpenMM XML text."""
        return cls.from_parsed(parse_system(system_xml), parse_state(state_xml), options)

    @classmethod
    def from_parsed(cls, system: System, state: State, options: RunOptions | None = None) -> "StepLoop":
        """`StepLoop.fromParsed`, loop.ts:278."""
        return cls.batch([system], [state], options)

    @classmethod
    def batch(cls, systems: Sequence[System], states: Sequence[State],
              options: RunOptions | None = None) -> "StepLoop":
        """Many independent systems in one engine (no reference counterpart)."""
        options = options or RunOptions()
        lib = abi.load()
        if len(systems) != len(states) or not systems:
            raise ValueError("one state per system, and at least one system")
        sys_handles = [s.desc() for s in systems]
        st_handles = [s.desc() for s in states]
        sys_array = (abi.SystemDesc * len(systems))(*[h.desc for h in sys_handles])
        st_array = (abi.StateDesc * len(states))(*[h.desc for h in st_handles])
        opts = options.to_c()
        handle = C.c_void_p()
        status = lib.mdb_batch_create(len(systems), sys_array, st_array, C.byref(opts), C.byref(handle))
        if status != abi.OK:
            message = lib.mdb_last_error(handle).decode() if handle.value else abi.load().mdb_status_string(status).decode()
            if handle.value:
                lib.mdb_destroy(handle, None)
            raise _ERRORS.get(status, EngineError)(status, message)
        return cls(handle, lib, list(systems), list(states), options)

    @property
    def system_count(self) -> int:
        """Systems in the engine."""
        return len(self._systems)

    # ---- internals -------------------------------------------------------
    def _check(self, status: int) -> None:
        if status != abi.OK:
            message = self._lib.mdb_last_error(self._handle).decode()
            raise _ERRORS.get(status, EngineError)(status, message or self._lib.mdb_status_string(status).decode())

    def _n(self, system: int) -> int:
        return self._systems[system].particle_count

    @staticmethod
    def _dp(a: np.ndarray):
        return a.ctypes.data_as(C.POINTER(C.c_double))

    # ---- stepping ----------------------------------------------------------
    def run(self, steps: int) -> None:
        """`StepLoop.run(n)`, loop.ts:651."""
        self._check(self._lib.mdb_run(self._handle, int(steps)))

    def run_timed(self, steps: int) -> float:
        """Run and return the device time in ms (CUDA events on the engine stream)."""
        ms = C.c_double()
        self._check(self._lib.mdb_run_timed(self._handle, int(steps), C.byref(ms)))
        return ms.value

    @property
    def steps(self) -> int:
        v = C.c_int64()
        self._check(self._lib.mdb_get_step(self._handle, C.byref(v)))
        return v.value

    def advance_step_count(self, step: int) -> None:
        """`StepLoop.advanceStepCount`, loop.ts:564."""
        if int(step) != step or step < 0:
            raise ValueError(f"a step count must be a non-negative integer, got {step}")
        self._check(self._lib.mdb_set_step(self._handle, int(step)))

    # ---- state -------------------------------------------------------------
    def positions(self, system: int = 0) -> np.ndarray:
        out = np.zeros(self._n(system) * 3)
        self._check(self._lib.mdb_get_positions(self._handle, system, self._dp(out)))
        return out.reshape(-1, 3)

    def velocities(self, system: int = 0) -> np.ndarray:
        out = np.zeros(self._n(system) * 3)
        self._check(self._lib.mdb_get_velocities(self._handle, system, self._dp(out)))
        return out.reshape(-1, 3)

    def set_positions(self, positions, system: int = 0) -> None:
        p = np.ascontiguousarray(np.asarray(positions, dtype=np.float64).reshape(-1))
        if p.size != self._n(system) * 3:
            raise ValueError(f"expected {self._n(system) * 3} coordinates, got {p.size}")
        self._check(self._lib.mdb_set_positions(self._handle, system, self._dp(p)))

    def set_velocities(self, velocities, system: int = 0) -> None:
        v = np.ascontiguousarray(np.asarray(velocities, dtype=np.float64).reshape(-1))
        if v.size != self._n(system) * 3:
            raise ValueError(f"expected {self._n(system) * 3} velocities, got {v.size}")
        self._check(self._lib.mdb_set_velocities(self._handle, system, self._dp(v)))

    def set_box(self, vectors, system: int = 0) -> None:
        b = np.ascontiguousarray(np.asarray(vectors, dtype=np.float64).reshape(9))
        self._check(self._lib.mdb_set_box(self._handle, system, self._dp(b)))

    def box_vectors(self, system: int = 0) -> np.ndarray:
        b = np.zeros(9)
        self._check(self._lib.mdb_get_box(self._handle, system, self._dp(b)))
        return b.reshape(3, 3)

    def mesh(self, system: int = 0) -> tuple:
        m = (C.c_int32 * 3)()
        self._check(self._lib.mdb_get_mesh(self._handle, system, m))
        return tuple(m)

    # ---- evaluation ----------------------------------------------------------
    def evaluate(self, system: int = 0):
        """Energies by group and forces (N, 3) at the current configuration."""
        f = np.zeros(self._n(system) * 3)
        e = abi.Energies()
        self._check(self._lib.mdb_evaluate(self._handle, system, self._dp(f), C.byref(e)))
        return e.as_dict(), f.reshape(-1, 3)

    def potential(self, positions, system: int = 0):
        """`StepLoop.potential(positions)`, loop.ts:870: (energy, forces), state unchanged."""
        p = np.ascontiguousarray(np.asarray(positions, dtype=np.float64).reshape(-1))
        f = np.zeros_like(p)
        e = abi.Energies()
        self._check(self._lib.mdb_potential(self._handle, system, self._dp(p), self._dp(f), C.byref(e)))
        return e.potential, f.reshape(-1, 3)

    @property
    def options(self) -> RunOptions:
        return self._options

    def set_velocities_to_temperature(self, temperature: float, seed: int, system: int = 0) -> np.ndarray:
        """`Context.setVelocitiesToTemperature` as src/reference/velocities.ts:78
        restates it: a Maxwell-Boltzmann draw from the velocity domain of the
        counter-based generator, shifted by -(dt/2) F/m (the velocity time
        offset of both integrators) with the forces from the device, projected
        onto the constraints at 1e-5.  Sets and returns the velocities."""
        from .velocities import velocities_at_temperature

        _, forces = self.evaluate(system)
        v = velocities_at_temperature(self._systems[system], self.positions(system), temperature, seed,
                                      0.5 * self._options.time_step, forces)
        self.set_velocities(v, system)
        return v

    def minimise(self, tolerance: float = 10.0, max_iterations: int = 0, system: int = 0):
        """`minimiseOnDevice`, src/gpu/minimise.ts:33: OpenMM's minimisation of
        this system's current configuration with the device's forces (one
        `potential` call per evaluation); the result is left in place and the
        `MinimiseResult` returned."""
        from .minimise import minimise

        result = minimise(self._systems[system], self.positions(system), lambda p: self.potential(p, system),
                          tolerance=tolerance, max_iterations=max_iterations,
                          constraint_tolerance=self._options.constraint_tolerance)
        # the last evaluation was the line search's last trial, not necessarily the result
        self.set_positions(result.positions, system)
        return result

    def report(self, system: int = 0) -> Report:
        """`StepLoop.report()`, loop.ts:761."""
        energies, _ = self.evaluate(system)
        step = self.steps
        return Report(step=step, time=step * self._options.time_step,
                      potential_energy=energies["potential"], kinetic_energy=energies["kinetic"],
                      temperature=energies["temperature"], energies=energies)

    def shifted_kinetic_energy(self, system: int = 0) -> float:
        """The shifted kinetic energy `StepLoop.report()` carries (loop.ts:788-803):
        the velocities advanced half a step with the forces at the current
        coordinates and re-constrained, kJ/mol; potential plus this is the
        total a leapfrog integrator conserves."""
        from . import velocities as vel

        _, forces = self.evaluate(system)
        return vel.shifted_kinetic_energy(self._systems[system], self.positions(system), self.velocities(system),
                                          forces, 0.5 * self._options.time_step)

    def box_lengths(self, system: int = 0) -> np.ndarray:
        """`StepLoop.boxLengths`, loop.ts:995: the box's diagonal, nm."""
        return np.diag(self.box_vectors(system)).copy()

    # ---- statistics -----------------------------------------------------------
    def barostat_statistics(self, system: int = 0) -> dict:
        s = abi.BarostatStats()
        self._check(self._lib.mdb_get_barostat_stats(self._handle, system, C.byref(s)))
        return {"attempts": s.attempts, "accepted": s.accepted, "volumeScale": s.volume_scale,
                "screened": s.screened, "exactEvaluations": s.exact_evaluations,
                "trainingSamples": s.training_samples, "surrogateActive": bool(s.surrogate_active),
                "surrogateDisabled": bool(s.surrogate_disabled), "surrogateRms": s.surrogate_rms,
                "trainingLoss": s.training_loss, "trainingMs": s.training_ms}

    def verlet_flags(self, system: int = 0) -> dict:
        """`StepLoop.verletFlags`, loop.ts:941."""
        s = abi.NeighbourStats()
        self._check(self._lib.mdb_get_neighbour_stats(self._handle, system, C.byref(s)))
        return {"rebuilds": s.rebuilds, "tiles": s.tiles, "tileCapacity": s.tile_capacity,
                "blocks": s.blocks, "overflowed": bool(s.overflowed), "skin": s.skin,
                "innerTiles": s.inner_tiles, "prunes": s.prunes, "innerSkin": s.inner_skin,
                "tileAtoms": s.tile_atoms, "listGrown": s.list_grown}

    def cell_geometry(self, system: int = 0) -> dict:
        """`StepLoop.cellGeometry()`, loop.ts:894: the divisions of the cell
        grid the list was built on and each cell's extent along the box's
        diagonal (nm)."""
        div = (C.c_int32 * 3)()
        ext = (C.c_double * 3)()
        self._check(self._lib.mdb_get_cell_geometry(self._handle, system, div, ext))
        return {"divisions": tuple(div), "extent": tuple(ext)}

    @property
    def passes_per_step(self) -> int:
        """`StepLoop.passesPerStep`, loop.ts:1105: kernel launches one step makes."""
        n = C.c_int32()
        self._check(self._lib.mdb_get_passes_per_step(self._handle, C.byref(n)))
        return n.value

    def profile_step(self, repeats: int = 20) -> dict:
        """`StepLoop.profileStep`, loop.ts:705: device ms per stage.  Advances the system."""
        p = abi.Profile()
        self._check(self._lib.mdb_profile_step(self._handle, int(repeats), C.byref(p)))
        return p.as_dict()

    def memory_report(self) -> dict:
        buf = C.create_string_buffer(1 << 16)
        total = C.c_int64()
        self._check(self._lib.mdb_memory_report(self._handle, buf, len(buf), C.byref(total)))
        out = {}
        for item in buf.value.decode().split(";"):
            if "=" in item:
                k, v = item.split("=")
                out[k] = int(v)
        return out

    def destroy(self) -> dict:
        """`StepLoop.destroy()`, loop.ts:1113: {leaked: bytes}."""
        if self._destroyed:
            return {"leaked": 0}
        leaked = C.c_int64()
        self._lib.mdb_destroy(self._handle, C.byref(leaked))
        self._destroyed = True
        return {"leaked": leaked.value}

    def __del__(self):  # pragma: no cover - interpreter shutdown order varies
        try:
            if not self._destroyed:
                self.destroy()
        except Exception:
            pass


__all__ = ["StepLoop", "RunOptions", "Report", "EngineError", "CutoffTooLargeForBox", "ClusterTooLarge",
           "NotSmooth", "NoDevice", "UnsupportedForce"]


# ---- autotuner (no reference counterpart) -------------------------------------
def autotune(system: System, state: State, options: RunOptions | None = None, steps: int = 200) -> dict:
    """Time the library's candidate grid of list settings for one system on
    the device (`mdb_autotune`) and return the fastest."""
    return autotune_batch([system], [state], options, steps)


def autotune_batch(systems: Sequence[System], states: Sequence[State], options: RunOptions | None = None,
                   steps: int = 200) -> dict:
    """The same search with every candidate applied to all the systems of one
    batched engine (`mdb_autotune_batch`): the fastest for the batch's step."""
    options = options or RunOptions()
    lib = abi.load()
    if len(systems) != len(states) or not systems:
        raise ValueError("one state per system, and at least one system")
    sys_handles = [s.desc() for s in systems]
    st_handles = [s.desc() for s in states]
    sys_array = (abi.SystemDesc * len(systems))(*[h.desc for h in sys_handles])
    st_array = (abi.StateDesc * len(states))(*[h.desc for h in st_handles])
    opts = dataclasses.replace(options, tuning=None).to_c()
    best = abi.Tuning()
    ms = C.c_double()
    tried = C.c_int32()
    status = lib.mdb_autotune_batch(len(systems), sys_array, st_array, C.byref(opts), int(steps), C.byref(best),
                                    C.byref(ms), C.byref(tried))
    if status != abi.OK:
        raise _ERRORS.get(status, EngineError)(status, lib.mdb_status_string(status).decode())
    return {"verlet_skin": best.verlet_skin, "sort_cell": best.sort_cell, "tile_atoms": best.tile_atoms,
            "prune_tiles": best.prune_tiles, "inner_skin": best.inner_skin, "ms_per_step": ms.value,
            "candidates": tried.value, "systems": len(systems)}


def size_bucket(atoms: int) -> int:
    """Size buckets of the autotuner: powers of two of the atom count."""
    return int(math.floor(math.log2(max(1, atoms))))


def tune_by_bucket(systems: Sequence[System], states: Sequence[State], options: RunOptions | None = None,
                   steps: int = 200, cache: dict | None = None, batched: bool = False,
                   cache_file: os.PathLike | str | None = None, gpu: str | None = None) -> tuple[list, dict]:
    """One search per size bucket; every system of the bucket takes its
    result.  Without `batched`, `autotune` on the bucket's median-sized
    system; with it, `autotune_batch` on the bucket's own systems together
    (from the smallest up, at most 2^18 atoms in all), which is how a batched
    engine runs them.  Returns the per-system tuning list for
    `RunOptions.tuning` and the per-bucket results.  `cache` (bucket ->
    result) skips buckets already tuned.

    `cache_file` keeps the results between runs: a JSON file of tuned buckets
    under a key made of the GPU model (`gpu`, else NVML's name for
    `options.device`), the library's ABI version and the search (batched or
    not, steps per candidate).  Buckets found there are not searched again;
    the file is rewritten with every bucket known afterwards.  One file suits
    one kind of workload: the buckets are by atom count alone."""
    cache = {} if cache is None else cache
    key = None
    if cache_file is not None:
        model = gpu if gpu is not None else gpu_model((options or RunOptions()).device)
        key = tuning_cache_key(model, batched, steps)
        for b, result in load_tuning_cache(cache_file, key).items():
            cache.setdefault(b, result)
    buckets: dict[int, list[int]] = {}
    for k, s in enumerate(systems):
        buckets.setdefault(size_bucket(s.particle_count), []).append(k)
    for b, members in sorted(buckets.items()):
        if b in cache:
            continue
        members = sorted(members, key=lambda k: systems[k].particle_count)
        if batched:
            take, atoms = [], 0
            for k in members:
                if take and atoms + systems[k].particle_count > (1 << 18):
                    break
                take.append(k)
                atoms += systems[k].particle_count
            cache[b] = autotune_batch([systems[k] for k in take], [states[k] for k in take], options, steps)
        else:
            rep = members[len(members) // 2]
            cache[b] = autotune(systems[rep], states[rep], options, steps)
    if cache_file is not None:
        save_tuning_cache(cache_file, key, cache)
    tuning = [tuple(cache[size_bucket(s.particle_count)][k]
                    for k in ("verlet_skin", "sort_cell", "tile_atoms", "prune_tiles", "inner_skin"))
              for s in systems]
    return tuning, cache


def gpu_model(device: int = 0) -> str:
    """The model name NVML gives for device index `device` ("unknown" when
    NVML is not there): list settings tuned on one model hold for every GPU
    of that model.  NVML counts devices as the driver does, which is CUDA's
    order unless CUDA_VISIBLE_DEVICES reorders them."""
    try:
        import pynvml

        pynvml.nvmlInit()
        try:
            name = pynvml.nvmlDeviceGetName(pynvml.nvmlDeviceGetHandleByIndex(int(device)))
        finally:
            pynvml.nvmlShutdown()
    except Exception:  # no driver, no NVML, no such device
        return "unknown"
    return name.decode() if isinstance(name, bytes) else str(name)


def tuning_cache_key(model: str, batched: bool, steps: int) -> str:
    """The key of a tuning-cache entry: GPU model, library ABI, search."""
    return f"{model} | abi {abi.ABI_VERSION} | {'batched' if batched else 'median system'} | {int(steps)} steps"


def load_tuning_cache(path: os.PathLike | str, key: str) -> dict:
    """The buckets saved under `key` in the JSON file at `path` ({} when the
    file or the key is absent)."""
    target = Path(path)
    if not target.exists():
        return {}
    data = json.loads(target.read_text())
    return {int(b): dict(r) for b, r in data.get(key, {}).items()}


def save_tuning_cache(path: os.PathLike | str, key: str, cache: dict) -> None:
    """Write `cache` (bucket -> result) under `key`, keeping the file's other
    keys; the file is replaced in one rename, so a reader never sees half of
    it."""
    target = Path(path)
    data = json.loads(target.read_text()) if target.exists() else {}
    data[key] = {str(b): cache[b] for b in sorted(cache)}
    partial = target.with_name(target.name + ".partial")
    partial.write_text(json.dumps(data, indent=1, sort_keys=True))
    os.replace(partial, target)


# ---- the barostat screening network's kernels on their own ---------------------
MLP_IN, MLP_HIDDEN = 16, 64
MLP_PARAMS = MLP_HIDDEN * MLP_IN + MLP_HIDDEN + MLP_HIDDEN * MLP_HIDDEN + MLP_HIDDEN + MLP_HIDDEN + 1


def _fptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def mlp_gradient(params, x, t) -> tuple[float, np.ndarray]:
    """Loss and gradient of the first min(n, 128) samples, by the CUDA kernel."""
    p = np.ascontiguousarray(params, dtype=np.float32)
    xx = np.ascontiguousarray(x, dtype=np.float32)
    tt = np.ascontiguousarray(t, dtype=np.float32)
    g = np.zeros(MLP_PARAMS, dtype=np.float32)
    loss = np.zeros(1, dtype=np.float32)
    status = abi.load().mdb_mlp_gradient(_fptr(p), _fptr(xx), _fptr(tt), int(tt.size), _fptr(g), _fptr(loss))
    if status != abi.OK:
        raise EngineError(status, abi.load().mdb_status_string(status).decode())
    return float(loss[0]), g


def mlp_fit(x, t, epochs: int, seed: int = 0) -> tuple[np.ndarray, np.ndarray]:
    """Train the network on the device; (FP32 master weights, per-epoch loss)."""
    xx = np.ascontiguousarray(x, dtype=np.float32)
    tt = np.ascontiguousarray(t, dtype=np.float32)
    params = np.zeros(MLP_PARAMS, dtype=np.float32)
    losses = np.zeros(epochs, dtype=np.float32)
    status = abi.load().mdb_mlp_fit(_fptr(xx), _fptr(tt), int(tt.size), int(epochs), int(seed) & 0xFFFFFFFF,
                                    _fptr(params), _fptr(losses))
    if status != abi.OK:
        raise EngineError(status, abi.load().mdb_status_string(status).decode())
    return params, losses


def mlp_predict(params, x) -> np.ndarray:
    p = np.ascontiguousarray(params, dtype=np.float32)
    xx = np.ascontiguousarray(x, dtype=np.float32)
    y = np.zeros(xx.shape[0], dtype=np.float32)
    status = abi.load().mdb_mlp_predict(_fptr(p), _fptr(xx), int(xx.shape[0]), _fptr(y))
    if status != abi.OK:
        raise EngineError(status, abi.load().mdb_status_string(status).decode())
    return y

