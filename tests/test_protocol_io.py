"""Velocity initialisation and what a run writes: the
counter-based draw against the Random123 known answers and the oracle, the
constraint projection, the -(dt/2) F/m shift; DCD frames in OpenMM's layout
(src/analysis/dcd.ts), the StateDataReporter log (src/analysis/log.ts) and
the .rst checkpoint round trip (src/engine/state.ts)."""

from __future__ import annotations

import io

import numpy as np
import pytest

from conftest import golden
from mdb200 import reporters, velocities
from mdb200.system import parse_state


def test_threefry_matches_the_known_answers():
    for case in golden("random_kat")["cases"]:
        c0, c1, k0, k1 = case["input"]
        x0, x1 = velocities.threefry2x32([c0], [c1], k0, k1, case["rounds"])
        assert [int(x0[0]), int(x1[0])] == case["output"], case


def test_domain_normals_match_the_oracle(oracle):
    out = velocities.domain_normals(velocities.VELOCITY_DOMAIN, 12345, 50)
    for i in range(50):
        for axis in range(3):
            want = oracle.lib().orc_domain_normal(velocities.VELOCITY_DOMAIN, 12345, i, axis)
            assert abs(out[i, axis] - want) <= 1e-12 * max(1.0, abs(want))


def test_velocities_match_the_oracle_and_hold_the_constraints(oracle):
    from mdb200 import synth

    system, state = synth.water_box(n_waters=300, width=2.1, seed=5)
    v = velocities.velocities_at_temperature(system, state.positions, 300.0, 7, time_offset=0.0)
    want = oracle.velocities_at_temperature(system, state.positions, 300.0, 7)
    assert np.abs(v - want).max() < 2e-4, np.abs(v - want).max()
    p = state.positions
    r = p[system.constraint_p2] - p[system.constraint_p1]
    rv = np.einsum("ij,ij->i", r, v[system.constraint_p2] - v[system.constraint_p1])
    assert np.max(np.abs(rv) / np.einsum("ij,ij->i", r, r)) <= 1e-5


def test_the_draw_is_maxwell_boltzmann_and_shifted_by_half_a_step():
    from mdb200.system import System

    n = 20000
    rng = np.random.default_rng(1)
    masses = rng.uniform(1.0, 40.0, n)
    system = System(masses=masses, box=np.eye(3) * 10.0)
    pos = rng.uniform(0, 10, (n, 3))
    v0 = velocities.velocities_at_temperature(system, pos, 300.0, 3, time_offset=0.0)
    ratio = np.mean(masses[:, None] * v0**2) / (velocities.BOLTZMANN_KJ_PER_MOL_K * 300.0)
    assert abs(ratio - 1.0) < 0.02, ratio
    forces = rng.normal(0, 500.0, (n, 3))
    v1 = velocities.velocities_at_temperature(system, pos, 300.0, 3, time_offset=0.001, forces=forces)
    np.testing.assert_allclose(v1 - v0, -(0.001 / masses)[:, None] * forces, rtol=1e-12, atol=1e-15)
    with pytest.raises(ValueError):
        velocities.velocities_at_temperature(system, pos, 300.0, 3, time_offset=0.001)


def test_shifted_kinetic_energy_matches_the_oracle_projection(oracle):
    """The report's shifted kinetic energy (kinetic.ts:87): velocities
    advanced by dt/2 with the forces, re-constrained, then (1/2) sum m v^2 --
    against the same shift projected by the oracle's constraint solve."""
    from mdb200 import synth

    system, state = synth.water_box(n_waters=300, width=2.1, seed=5)
    rng = np.random.default_rng(3)
    v = velocities.velocities_at_temperature(system, state.positions, 300.0, 7, time_offset=0.0)
    forces = rng.normal(0.0, 800.0, v.shape)
    m = np.asarray(system.masses)
    shifted = v + (0.001 / m)[:, None] * forces
    flat = np.ascontiguousarray(shifted.reshape(-1))
    pos = np.ascontiguousarray(np.asarray(state.positions, dtype=np.float64).reshape(-1))
    assert oracle.lib().orc_constrain_velocities(system.desc().pointer(), oracle._p(pos), oracle._p(flat),
                                                 1e-10) == 0
    want = oracle.kinetic_energy(system, flat)
    got = velocities.shifted_kinetic_energy(system, state.positions, v, forces, 0.001, tolerance=1e-10)
    assert abs(got - want) <= 1e-8 * want, (got, want)
    loose = velocities.shifted_kinetic_energy(system, state.positions, v, forces, 0.001)
    assert abs(loose - want) <= 1e-4 * want, (loose, want)
    # the shift moves energy: the unshifted and shifted values differ, and a zero shift is the plain sum
    assert abs(velocities.kinetic_energy(system, v) - want) > 1e-3 * want
    assert velocities.shifted_kinetic_energy(system, state.positions, v, forces, 0.0) == \
        velocities.kinetic_energy(system, v)
    assert abs(velocities.kinetic_energy(system, v) - oracle.kinetic_energy(system, v)) <= 1e-12 * want


def test_dcd_layout_and_round_trip():
    buf = io.BytesIO()
    w = reporters.DcdWriter(buf, 37, time_step=0.002, first_step=100, interval=50)
    rng = np.random.default_rng(2)
    frames = [rng.uniform(0, 3, (37, 3)) for _ in range(5)]
    box = np.eye(3) * 3.1
    for f in frames:
        w.write_frame(f, box)
    data = buf.getvalue()
    # 276 header bytes + 5 x 524 for 37 atoms, the sizes OpenMM's writer produces
    assert reporters.DCD_HEADER_BYTES == 276 and w.frame_bytes == 524 and len(data) == 2896
    back = reporters.read_dcd(data)
    assert back["frames"] == 5 and back["first_step"] == 100 and back["interval"] == 50
    assert back["last_step"] == 100 + 4 * 50 and back["atoms"] == 37 and back["periodic"]
    assert abs(back["time_step"] - 0.002) < 1e-9
    for a, b in zip(frames, back["positions"]):
        np.testing.assert_allclose(b, a, rtol=0, atol=3e-6)  # f32 angstrom
    assert back["cells"][0] == (31.0, 0.0, 31.0, 0.0, 0.0, 31.0)
    with pytest.raises(ValueError):
        w.write_frame(np.full((37, 3), np.nan), box)


def test_dcd_cell_of_a_rhombic_dodecahedron():
    w = 4.0
    box = np.array([[w, 0, 0], [0, w, 0], [w / 2, w / 2, w * np.sqrt(2) / 2]])
    (la, lb, lc), (ca, cb, cg) = reporters.unit_cell(box)
    np.testing.assert_allclose([la, lb, lc], [w, w, w])
    np.testing.assert_allclose([ca, cb, cg], [0.5, 0.5, 0.0], atol=1e-15)


def test_log_header_and_rows():
    assert reporters.log_header() == ('#"Step","Potential Energy (kJ/mole)","Kinetic Energy (kJ/mole)",'
                                      '"Total Energy (kJ/mole)","Temperature (K)","Box Volume (nm^3)",'
                                      '"Speed (ns/day)"\n')
    assert reporters.log_row(0, -10.0, 4.0, 300.0, 27.0, None) == "0,-10.0,4.0,-6.0,300.0,27.0,--\n"
    assert reporters.log_row(500, -10.5, 4.0, 301.0, 27.1, 123.0).endswith(",123.0\n")


def test_checkpoint_round_trips_exactly():
    from mdb200.system import State, serialise_state

    rng = np.random.default_rng(4)
    st = State(positions=rng.normal(size=(7, 3)), box=np.eye(3) * 3.080639849905961,
               velocities=rng.normal(size=(7, 3)), step=12500, time=25.000000000000004)
    back = parse_state(serialise_state(st))
    assert np.array_equal(back.positions, st.positions) and np.array_equal(back.velocities, st.velocities)
    assert back.step == st.step and back.time == st.time and np.array_equal(back.box, st.box)


@pytest.mark.gpu
def test_engine_draw_checkpoint_and_trajectory(tmp_path):
    """On the device: velocities to temperature with the device forces, a short
    run written as DCD frames and a log, and a checkpoint that resumes with the
    same state exactly (positions are 2^-32 fixed point, velocities f32, both
    exact in the decimal round trip) and the same energies.  The resumed run is
    close, not bit-identical: a new engine starts a new pair list, whose tiles
    group the f32 pair sums differently, and the drift residuals start at zero."""
    from mdb200 import steploop, synth

    system, state = synth.config_peptide_12k()
    loop = steploop.StepLoop.from_parsed(system, state, steploop.RunOptions(seed=11))
    v = loop.set_velocities_to_temperature(300.0, seed=5)
    t0 = loop.report().temperature
    print("temperature after the draw", t0)
    assert 270.0 < t0 < 340.0
    p = loop.positions()
    r = p[system.constraint_p2] - p[system.constraint_p1]
    rv = np.einsum("ij,ij->i", r, v[system.constraint_p2] - v[system.constraint_p1])
    assert np.max(np.abs(rv) / np.einsum("ij,ij->i", r, r)) <= 1e-5
    path = tmp_path / "run.dcd"
    log = [reporters.log_header()]
    with open(path, "w+b") as f:
        w = reporters.DcdWriter(f, system.particle_count, 0.002, first_step=loop.steps, interval=100)
        for k in range(3):
            loop.run(100)
            rep = loop.report()
            w.write_frame(loop.positions(), loop.box_vectors())
            log.append(reporters.log_row(rep.step, rep.potential_energy, rep.kinetic_energy, rep.temperature,
                                         abs(np.linalg.det(loop.box_vectors())), None if k == 0 else 1.0))
    back = reporters.read_dcd(path.read_bytes())
    assert back["frames"] == 3
    np.testing.assert_allclose(back["positions"][-1], loop.positions(), atol=5e-5)
    rst = reporters.checkpoint(loop)
    resumed = steploop.StepLoop.from_parsed(system, parse_state(rst), steploop.RunOptions(seed=11))
    assert resumed.steps == loop.steps
    assert np.array_equal(resumed.positions(), loop.positions())
    assert np.array_equal(resumed.velocities(), loop.velocities())
    a, b = loop.report(), resumed.report()
    assert abs(a.potential_energy - b.potential_energy) <= 1e-6 * abs(a.potential_energy)
    assert a.kinetic_energy == b.kinetic_energy
    loop.run(50)
    resumed.run(50)
    assert np.abs(loop.positions() - resumed.positions()).max() < 1e-3
    loop.destroy()
    resumed.destroy()
