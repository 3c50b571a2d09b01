"""Dynamics checks on the GPU that need many steps.

* Energy conservation (src/gpu/validate-loop.ts:24-93): velocity Verlet with
  no thermostat, reports every tenth of the run, total energy = potential +
  the shifted kinetic energy (velocities advanced half a step with the
  current forces and re-constrained, src/reference/kinetic.ts:59 -- OpenMM's
  computeShiftedVelocities), least-squares slope per atom per ns below the
  reference's calibrated gate of 1.5 kJ/mol/ns/atom.
* Position restraints (restraint.wgsl:81; oracle forces/restraint.ts:38)
  against the oracle.
"""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DRIFT_GATE = 1.5  # kJ/mol/ns/atom, validate-loop.ts:93
TIME_STEP = 0.002


def shifted_kinetic(oracle, system, positions, velocities, forces, shift):
    m = np.asarray(system.masses)
    v = np.array(velocities, dtype=np.float64)
    moving = m > 0
    v[moving] += forces[moving] * (shift / m[moving])[:, None]
    flat = np.ascontiguousarray(v.reshape(-1))
    pos = np.ascontiguousarray(np.asarray(positions, dtype=np.float64).reshape(-1))
    status = oracle.lib().orc_constrain_velocities(system.desc().pointer(), oracle._p(pos), oracle._p(flat), 1e-10)
    assert status == 0
    v = flat.reshape(-1, 3)
    return 0.5 * float((m[:, None] * v * v).sum())


def test_verlet_conserves_energy_within_the_reference_gate(oracle):
    from mdb200 import steploop, synth
    from mdb200.system import State

    system, state = synth.config_water_2652()
    # equilibrate the lattice start with the thermostat first
    nvt = steploop.StepLoop.from_parsed(system, state, steploop.RunOptions(seed=3))
    nvt.run(3000)
    start = State(positions=nvt.positions(), velocities=nvt.velocities(), box=state.box.copy())
    nvt.destroy()
    nve = steploop.StepLoop.from_parsed(system, start, steploop.RunOptions(integrator="verlet", friction=0.0))
    steps, reports = 5000, 10
    times, totals = [], []
    for k in range(reports + 1):
        if k:
            nve.run(steps // reports)
        e, f = nve.evaluate()
        ke = shifted_kinetic(oracle, system, nve.positions(), nve.velocities(), f, 0.5 * TIME_STEP)
        times.append(k * steps // reports * TIME_STEP / 1000.0)  # ns
        totals.append(e["potential"] + ke)
    nve.destroy()
    slope = np.polyfit(times, totals, 1)[0]
    drift = abs(slope) / system.particle_count
    print("total energy", [round(t, 2) for t in totals], "drift kJ/mol/ns/atom", drift)
    assert drift < DRIFT_GATE, drift


def test_position_restraints_match_oracle(oracle):
    from mdb200 import steploop, synth

    system, state = synth.config_water_2652()
    rng = np.random.default_rng(6)
    chosen = np.sort(rng.choice(system.particle_count, size=200, replace=False)).astype(np.int32)
    anchors = state.positions[chosen] + rng.normal(0, 0.05, size=(200, 3))
    k = rng.uniform(100.0, 1000.0, size=200)
    system.restraints = (chosen, k, anchors[:, 0].copy(), anchors[:, 1].copy(), anchors[:, 2].copy())
    loop = steploop.StepLoop.from_parsed(system, state, steploop.RunOptions())
    e, f = loop.evaluate()
    loop.destroy()
    want, wf = oracle.potential(system, state.positions, grid=(30, 30, 30), threads=8)
    print("restraint energy", e["restraint"], want["restraint"])
    assert abs(e["restraint"] - want["restraint"]) <= 1e-5 * abs(want["restraint"])
    err = float(np.sqrt(((f - wf) ** 2).sum() / (wf ** 2).sum()))
    assert err <= 1.1e-6, err
