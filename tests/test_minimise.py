"""The minimiser (src/reference/minimise.ts, src/reference/lbfgs.ts,
src/gpu/minimise.ts): L-BFGS against closed-form minima and OpenMM's spring
schedule on the CPU (test/lbfgs.test.ts is the model); on the GPU, the
device-force minimisation against the same search over the oracle's f64
forces at matched iteration counts, and a long run's descent and
constraints (the reference's validate-minimise.ts thresholds)."""

from __future__ import annotations

import numpy as np
import pytest

from mdb200.minimise import constrain_positions, lbfgs, max_constraint_error, minimise


def quadratic(centre, scales):
    centre, scales = np.asarray(centre, float), np.asarray(scales, float)

    def f(x, g):
        d = x - centre
        g[:] = 2 * scales * d
        return float(np.sum(scales * d * d))
    return f


def rosenbrock(x, g):
    a, b = x[0::2], x[1::2]
    t1, t2 = 1 - a, 10 * (b - a * a)
    g[0::2] = -2 * t1 - 400 * a * (b - a * a)
    g[1::2] = 200 * (b - a * a)
    return float(np.sum(t1 * t1 + t2 * t2))


def test_lbfgs_finds_a_quadratic_minimum():
    x = np.array([5.0, -3.0, 11.0])
    r = lbfgs(x, quadratic([1, 2, 3], [1, 1, 1]), epsilon=1e-10)
    assert r.status == "converged"
    np.testing.assert_allclose(x, [1, 2, 3], atol=1e-8)


def test_lbfgs_handles_a_badly_conditioned_quadratic():
    x = np.array([3.0, 3.0, 3.0, 3.0])
    r = lbfgs(x, quadratic([0, 0, 0, 0], [1, 1e2, 1e4, 1e6]), epsilon=1e-9)
    assert r.status == "converged" and r.iterations < 200
    np.testing.assert_allclose(x, 0, atol=1e-6)


def test_lbfgs_solves_extended_rosenbrock():
    x = np.tile([-1.2, 1.0], 10)
    r = lbfgs(x, rosenbrock, epsilon=1e-8)
    assert r.status == "converged"
    np.testing.assert_allclose(x, 1.0, atol=1e-5)


def test_lbfgs_reports_max_iterations_and_keeps_its_last_point():
    x = np.tile([-1.2, 1.0], 4)
    r = lbfgs(x, rosenbrock, epsilon=1e-12, max_iterations=3)
    assert r.status == "max-iterations" and r.iterations == 3
    g = np.zeros_like(x)
    assert abs(rosenbrock(x, g) - r.value) < 1e-12


def dimers(n=6, seed=0):
    """n constrained dimers (0.1 nm) pulled apart by springs to fixed anchors:
    a potential whose minimum stretches the constraints."""
    from mdb200.system import System

    rng = np.random.default_rng(seed)
    pos = np.zeros((2 * n, 3))
    pos[0::2] = rng.uniform(0, 3, (n, 3))
    pos[1::2] = pos[0::2] + 0.1 / np.sqrt(3)
    system = System(masses=np.ones(2 * n) * 12.0, box=np.eye(3) * 5.0,
                    constraint_p1=np.arange(0, 2 * n, 2, dtype=np.int32),
                    constraint_p2=np.arange(1, 2 * n, 2, dtype=np.int32),
                    constraint_distance=np.full(n, 0.1))
    anchors = pos + rng.normal(0, 0.05, pos.shape)

    def potential(p):
        d = p - anchors
        return float(500.0 * np.sum(d * d)), -1000.0 * d
    return system, pos, potential


def test_constraint_projection_meets_its_tolerance():
    system, pos, _ = dimers()
    noisy = pos + np.random.default_rng(3).normal(0, 0.01, pos.shape)
    assert max_constraint_error(system, noisy) > 1e-2
    out = constrain_positions(system, noisy, 1e-8)
    assert max_constraint_error(system, out) <= 1e-8


def test_minimise_with_springs_meets_the_tolerances():
    system, pos, potential = dimers()
    r = minimise(system, pos, potential, tolerance=1.0, constraint_tolerance=1e-6)
    assert not r.gave_up
    assert r.status in ("converged", "line-search-failed", "step-too-small")
    assert r.initial_restraint_strength == 100 / 1e-4
    assert r.restraint_strength >= r.initial_restraint_strength
    assert max_constraint_error(system, r.positions) <= 1e-6
    e0, _ = potential(pos)
    e1, _ = potential(r.positions)
    assert e1 < e0


def test_minimise_stiffens_the_springs_until_the_constraints_hold():
    """OpenMM's schedule: a force pulling each dimer apart (U = -A r, A = 1e4
    kJ/mol/nm) stretches it by A / k against the springs, so k is raised ten
    times per round from 1e6 until A / (k d) falls below the working 1e-4 --
    five rounds -- and the final projection meets the caller's 1e-6."""
    system, pos, _ = dimers(n=3)
    A = 1e4

    def pulling(p):
        d = p[1::2] - p[0::2]
        r = np.linalg.norm(d, axis=1)
        f = np.zeros_like(p)
        f[1::2] = A * d / r[:, None]
        f[0::2] = -A * d / r[:, None]
        return float(-A * np.sum(r)), f
    r = minimise(system, pos, pulling, tolerance=1e-3, constraint_tolerance=1e-6)
    print(r.rounds, r.restraint_strength, r.max_constraint_error, r.status)
    assert not r.gave_up
    assert r.rounds >= 4
    assert np.isclose(r.restraint_strength, 1e6 * 10 ** (r.rounds - 1))
    assert r.max_constraint_error <= 1e-4
    assert max_constraint_error(system, r.positions) <= 1e-6


@pytest.mark.gpu
def test_device_minimisation_matches_the_oracle_search_and_descends(oracle):
    from mdb200 import steploop, synth

    system, state = synth.config_water_2652(seed=2)
    mesh = (30, 30, 30)
    frames = {}
    for iters in (1, 2, 5):
        loop = steploop.StepLoop.from_parsed(system, state, steploop.RunOptions(mesh=mesh))
        dev = loop.minimise(tolerance=10.0, max_iterations=iters)
        loop.destroy()

        def f64(p):
            e, f = oracle.potential(system, p, grid=mesh, threads=8)
            return e["potential"], f
        ref = minimise(system, state.positions, f64, tolerance=10.0, max_iterations=iters)
        rel = abs(dev.energy - ref.energy) / abs(ref.energy)
        frames[iters] = (dev.energy, ref.energy, rel)
        print("iterations", iters, "device", dev.energy, "oracle", ref.energy, "rel", rel)
        assert rel <= 1e-3, (iters, rel)
    loop = steploop.StepLoop.from_parsed(system, state, steploop.RunOptions(mesh=mesh))
    e0 = loop.report().potential_energy
    long = loop.minimise(tolerance=10.0, max_iterations=200)
    e1 = loop.report().potential_energy
    print("long run", e0, "->", e1, long.status, long.iterations, long.potential_force_rms)
    assert (e0 - e1) / system.particle_count >= 0.5
    assert max_constraint_error(system, loop.positions()) <= 2e-6
    loop.destroy()
