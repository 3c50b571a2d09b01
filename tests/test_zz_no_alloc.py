"""The allocation-free reciprocal-space entry point, `mdb_reciprocal_noalloc`.

It exists for callers that cannot allocate device memory (a host that only
receives device buffers from its own allocator, or a loop that must not
allocate once it runs): they pass their own device buffers and the library's
fixed-size device array holds every intermediate.  This test calls it through
the C ABI on caller-owned buffers, twice in a row, and checks each result
against the engine's own reciprocal-space output for the same charges (a
system whose charges are all farther apart than the cutoff, so the engine's
forces are the reciprocal forces alone and `reciprocal_mesh` is the mesh sum):
the same per-point arithmetic, so the force bits are equal and the energy
agrees to 1e-12.  It also checks each
result against the f64 oracle at the PME force and reciprocal-energy
tolerances.

This file is collected last on purpose: it must pass on its own in a fresh
process and after every other test.
"""

from __future__ import annotations

import ctypes as C
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# Against the f64 oracle: these forces are the reciprocal forces alone, which
# the f32 mesh arithmetic carries to a few 1e-6; the bound is the one the
# oracle's own PME forces are pinned to against OpenMM (1e-5 relative RMS).
# The engine's 1.1e-6 bound is on whole forces, where direct space dominates.
RECIPROCAL_FORCE_REL_RMS = 1e-5
ENERGY_REL = 1e-5
MESH = (32, 32, 32)


def separated_charges():
    from mdb200.system import Nonbonded, State, System

    rng = np.random.default_rng(17)
    width, cutoff = 3.0, 0.5
    g = (np.arange(4) + 0.5) * (width / 4)
    sites = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    pos = sites + rng.uniform(-0.05, 0.05, size=sites.shape)
    n = len(pos)
    q = np.where(np.arange(n) % 2 == 0, 1.0, -1.0) * rng.uniform(0.5, 1.0, size=n)
    q -= q.mean()
    box = np.eye(3) * width
    system = System(masses=np.full(n, 10.0), box=box,
                    nonbonded=Nonbonded(cutoff=cutoff, ewald_tolerance=5e-4, charge=q, sigma=np.full(n, 0.3),
                                        epsilon=np.zeros(n), exception_p1=np.zeros(0, dtype=np.int32),
                                        exception_p2=np.zeros(0, dtype=np.int32),
                                        exception_charge_prod=np.zeros(0), exception_sigma=np.zeros(0),
                                        exception_epsilon=np.zeros(0), use_dispersion_correction=False))
    alpha = math.sqrt(-math.log(2 * 5e-4)) / cutoff
    return system, State(positions=pos, box=box), alpha


def test_noalloc_reciprocal_matches_the_engine_twice(oracle):
    import torch

    from mdb200 import abi, steploop

    system, state, alpha = separated_charges()
    want, oracle_forces = oracle.potential(system, state.positions, grid=MESH)
    loop = steploop.StepLoop.from_parsed(system, state, steploop.RunOptions(mesh=MESH, friction=0.0))
    energies, want_forces = loop.evaluate()
    loop.destroy()
    assert energies["pairs_within_cutoff"] == 0 and energies["direct_coulomb"] == 0.0
    want_energy = energies["reciprocal_mesh"]

    lib = abi.load()
    n = system.particle_count
    dev = torch.device("cuda:0")
    positions = torch.tensor(state.positions.reshape(-1), dtype=torch.float64, device=dev)
    charges = torch.tensor(system.nonbonded.charge, dtype=torch.float64, device=dev)
    forces = torch.full((3 * n,), float("nan"), dtype=torch.float64, device=dev)
    energy = torch.full((1,), float("nan"), dtype=torch.float64, device=dev)
    box = np.ascontiguousarray(state.box.reshape(9), dtype=np.float64)
    mesh = (C.c_int32 * 3)(*MESH)
    torch.cuda.synchronize()
    for call in range(2):
        status = lib.mdb_reciprocal_noalloc(n, positions.data_ptr(), charges.data_ptr(),
                                            box.ctypes.data_as(C.POINTER(C.c_double)), alpha, mesh,
                                            forces.data_ptr(), energy.data_ptr(), None)
        assert status == abi.OK, lib.mdb_status_string(status)
        torch.cuda.synchronize()
        got_f = forces.cpu().numpy().reshape(-1, 3)
        got_e = float(energy.cpu().item())
        err = float(np.sqrt(((got_f - oracle_forces) ** 2).sum() / (oracle_forces**2).sum()))
        print(f"call {call}: force rel RMS {err:.2e} against the oracle, energy {got_e:.6f} "
              f"(engine {want_energy:.6f}, oracle {want['reciprocal_mesh']:.6f})")
        # the engine's reciprocal space runs the same per-point arithmetic: the
        # same force bits; the FP64 energy partials are summed over a different
        # split of the spectrum, so the energy may differ in its last bits
        assert np.array_equal(got_f, want_forces), (call, np.abs(got_f - want_forces).max())
        assert abs(got_e - want_energy) <= 1e-12 * abs(want_energy), (call, got_e, want_energy)
        # and against the f64 oracle, at the PME force bound and the reciprocal-group tolerance
        assert err <= RECIPROCAL_FORCE_REL_RMS, (call, err)
        assert abs(got_e - want["reciprocal_mesh"]) <= ENERGY_REL * abs(want["reciprocal_mesh"]), (call, got_e)


def test_noalloc_refuses_meshes_beyond_its_array():
    from mdb200 import abi

    lib = abi.load()
    box = np.ascontiguousarray((np.eye(3) * 3.0).reshape(9))
    dummy = C.c_void_p(1)  # never dereferenced: the size check comes first
    too_many = (C.c_int32 * 3)(128, 128, 32)     # 524,288 points > 262,144
    too_long = (C.c_int32 * 3)(256, 8, 8)        # an axis beyond 128
    not_smooth = (C.c_int32 * 3)(22, 22, 22)
    for mesh, want in ((too_many, abi.ERR_CAPACITY), (too_long, abi.ERR_CAPACITY), (not_smooth, abi.ERR_NOT_SMOOTH)):
        status = lib.mdb_reciprocal_noalloc(1, dummy, dummy, box.ctypes.data_as(C.POINTER(C.c_double)), 3.0, mesh,
                                            dummy, dummy, None)
        assert status == want
