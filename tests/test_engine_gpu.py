"""Parity of the CUDA engine against the f64 oracle, through the C ABI.

Tolerances are the reference's own (src/gpu/validate.ts:80-117,
src/gpu/validate-loop.ts:90-100) and the engine's force bound:
  forces                     relative RMS <= 1.1e-6 against the f64 oracle
  direct-space group energy  1e-4 relative
  reciprocal group energy    1e-5 relative
  bonded energies            1e-5 relative
  one LFMiddle step          positions 4e-7 nm, velocities 4e-4 nm/ps
  repeat runs                bit-identical
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import force_error_allowing_cutoff_shell, golden_nonbonded_system, rel_rms

pytestmark = pytest.mark.gpu

FORCE_REL_RMS = 1.1e-6


@pytest.fixture(scope="module")
def mdb():
    from mdb200 import steploop

    return steploop


@pytest.fixture(scope="module")
def water():
    from mdb200 import synth

    return synth.config_water_2652()


def make_loop(mdb, system, state, **kw):
    opts = mdb.RunOptions(**kw)
    return mdb.StepLoop.from_parsed(system, state, opts)


def test_fixture_groups_and_forces(mdb, oracle):
    """The reference's 10-particle OpenMM fixture (nonbonded-reference.test.ts)."""
    system, state, g = golden_nonbonded_system()
    mesh = (24, 24, 24)
    loop = make_loop(mdb, system, state, mesh=mesh, friction=0.0)
    e, f = loop.evaluate()
    want, wf = oracle.potential(system, state.positions, grid=mesh)
    for key in ("direct_coulomb", "direct_lj", "exclusion_correction", "exceptions"):
        assert abs(e[key] - want[key]) <= 1e-4 * max(1.0, abs(want[key])), (key, e[key], want[key])
    assert abs(e["reciprocal_group"] - want["reciprocal_group"]) <= 1e-5 * abs(want["reciprocal_group"])
    assert abs(e["direct_group"] - want["direct_group"]) <= 1e-4 * abs(want["direct_group"])
    err = rel_rms(f, wf)
    print("fixture force rel RMS", err)
    assert err <= FORCE_REL_RMS, err
    loop.destroy()


def test_water_forces_and_groups(mdb, oracle, water):
    system, state = water
    loop = make_loop(mdb, system, state)
    e, f = loop.evaluate()
    want, wf = oracle.potential(system, state.positions, grid=(30, 30, 30))
    err = rel_rms(f, wf)
    print("water force rel RMS", err)
    print({k: (e[k], want[k]) for k in want if k in e})
    assert err <= FORCE_REL_RMS, err
    assert abs(e["direct_group"] - want["direct_group"]) <= 1e-4 * abs(want["direct_group"])
    assert abs(e["reciprocal_group"] - want["reciprocal_group"]) <= 1e-5 * abs(want["reciprocal_group"])
    assert abs(e["direct_coulomb"] - want["direct_coulomb"]) <= 1e-4 * abs(want["direct_coulomb"]) + 1e-3
    assert abs(e["direct_lj"] - want["direct_lj"]) <= 1e-4 * abs(want["direct_lj"])
    loop.destroy()


def test_one_step_matches_oracle(mdb, oracle, water):
    """validate-loop.ts:90-94: one LFMiddle step, friction on, same Threefry stream."""
    system, state = water
    loop = make_loop(mdb, system, state, seed=11)
    loop.run(1)
    p, v = loop.positions(), loop.velocities()
    op, ov, _ = oracle.run(system, state, 1, seed=11, grid=(30, 30, 30))
    dp = np.abs(p - op).max()
    dv = np.abs(v - ov).max()
    print("one step: max |dx|", dp, "max |dv|", dv)
    assert dp <= 4e-7, dp
    assert dv <= 4e-4, dv
    loop.destroy()


def test_repeat_runs_are_bit_identical(mdb, water):
    system, state = water
    out = []
    for _ in range(2):
        loop = make_loop(mdb, system, state, seed=3)
        loop.run(50)
        out.append((loop.positions(), loop.velocities()))
        loop.destroy()
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])


def test_graph_and_direct_launch_agree(mdb, water):
    system, state = water
    res = []
    for graphs in (True, False):
        loop = make_loop(mdb, system, state, seed=3, graphs=graphs, max_batch=7)
        loop.run(20)
        res.append(loop.positions())
        loop.destroy()
    assert np.array_equal(res[0], res[1])


def test_batch_equals_single(mdb, water):
    """Two systems in one engine advance exactly as each does alone."""
    from mdb200 import synth

    system, state = water
    other_sys, other_state = synth.water_box(n_waters=600, width=2.8, seed=7, grid=(28, 28, 28))
    single = []
    for s, st in ((system, state), (other_sys, other_state)):
        loop = make_loop(mdb, s, st, seed=5)
        loop.run(20)
        single.append(loop.positions())
        loop.destroy()
    batch = mdb.StepLoop.batch([system, other_sys], [state, other_state], mdb.RunOptions(seed=5))
    batch.run(20)
    assert np.array_equal(batch.positions(0), single[0])
    assert np.array_equal(batch.positions(1), single[1])
    batch.destroy()


def test_slot_ordered_spread_equals_atom_ordered_spread(mdb):
    """An engine of 80k atoms spreads PME charges by slot through shared-memory
    mesh patches, a single 10k-atom system by atom straight into the grid: the
    same fixed-point sums, so eight systems batched advance exactly as each
    does alone -- through steps that rebuild the list, whose snapshot of the
    slot order the spread reads."""
    from mdb200 import synth

    members = [synth.water_box(width=4.6, seed=20 + k) for k in range(8)]
    assert sum(m[0].particle_count for m in members) >= 148 * 128  # the slot-ordered spread's threshold
    assert members[0][0].particle_count < 148 * 128 - 128  # alone, each spreads by atom
    single = []
    for system, state in members:
        loop = make_loop(mdb, system, state, seed=6)
        loop.run(30)
        single.append(loop.positions())
        loop.destroy()
    batch = mdb.StepLoop.batch([m[0] for m in members], [m[1] for m in members], mdb.RunOptions(seed=6))
    batch.run(30)
    rebuilds = [batch.verlet_flags(k)["rebuilds"] for k in range(len(members))]
    print("rebuilds per system", rebuilds)
    for k in range(len(members)):
        assert np.array_equal(batch.positions(k), single[k]), k
    batch.destroy()


def test_set_box_equals_an_engine_created_at_that_box(mdb):
    """A box set on an engine -- its PME influence table, which the force
    steps read, is refilled; the list is rebuilt -- gives the trajectory of an
    engine created at that box and those positions, to the bit."""
    from mdb200 import synth
    from mdb200.system import State

    system, state = synth.water_box(n_waters=900, width=3.1, seed=8, grid=(32, 32, 32))
    scale = 1.004
    box2 = np.asarray(state.box, dtype=np.float64) * scale
    pos2 = np.asarray(state.positions, dtype=np.float64) * scale
    moved = make_loop(mdb, system, state, seed=9)
    moved.set_box(box2)
    moved.set_positions(pos2)
    moved.run(20)
    fresh = make_loop(mdb, system, State(positions=pos2, box=box2, velocities=state.velocities, step=state.step),
                      seed=9)
    fresh.run(20)
    assert np.array_equal(moved.positions(), fresh.positions())
    moved.destroy()
    fresh.destroy()


def test_potential_leaves_state_and_matches_evaluate(mdb, water):
    system, state = water
    loop = make_loop(mdb, system, state)
    before = loop.positions()
    # One whole mesh cell (3.0 nm / 30): PME is invariant under translations
    # by mesh cells only, so all that may move is f32 rounding.
    shifted = state.positions + np.array([0.1, 0.0, 0.0])
    e_shift, f_shift = loop.potential(shifted)
    assert np.array_equal(loop.positions(), before)
    e0, f0 = loop.evaluate()
    assert abs(e_shift - e0["potential"]) < 1e-7 * abs(e0["exclusion_correction"])
    assert rel_rms(f_shift, f0) < 2e-6
    loop.destroy()


def test_dynamics_stay_bounded(mdb, water):
    """The lattice-built box relaxes (about 24,000 kJ/mol of potential energy
    becomes heat, ~1,100 K worth over its 5,301 degrees of freedom) while the
    constraints hold and the thermostat starts to cool it."""
    system, state = water
    loop = make_loop(mdb, system, state, seed=2)
    e0 = loop.report().potential_energy
    loop.run(300)
    r = loop.report()
    print("after 300 steps", r.temperature, r.potential_energy, loop.verlet_flags())
    assert np.isfinite(r.potential_energy) and np.isfinite(r.kinetic_energy)
    assert r.potential_energy < e0 - 10000
    assert 100 < r.temperature < 1500
    p = loop.positions()
    d = np.linalg.norm(p[system.constraint_p1] - p[system.constraint_p2], axis=1)
    assert np.max(np.abs(d / system.constraint_distance - 1)) < 1e-5
    assert loop.verlet_flags()["rebuilds"] >= 1
    assert not loop.verlet_flags()["overflowed"]
    loop.destroy()


def test_cutoff_too_large_is_refused(mdb):
    from mdb200 import synth

    system, state = synth.water_box(n_waters=100, width=1.5, seed=1, grid=(16, 16, 16))
    with pytest.raises(mdb.CutoffTooLargeForBox):
        make_loop(mdb, system, state)


@pytest.fixture(scope="module")
def peptide():
    from mdb200 import synth

    return synth.config_peptide_12k()


def test_peptide_forces_and_groups(mdb, oracle, peptide):
    """The 12k-atom solvated Ala20 helix: bonded, exceptions, PME, SHAKE clusters."""
    system, state = peptide
    loop = make_loop(mdb, system, state)
    e, f = loop.evaluate()
    want, wf = oracle.potential(system, state.positions, grid=(50, 50, 50), threads=8)
    err = rel_rms(f, wf)
    print("peptide force rel RMS", err)
    assert err <= FORCE_REL_RMS, err
    for key in ("bond", "angle", "torsion"):
        assert abs(e[key] - want[key]) <= 1e-5 * abs(want[key]) + 1e-4, (key, e[key], want[key])
    assert abs(e["direct_group"] - want["direct_group"]) <= 1e-4 * abs(want["direct_group"])
    assert abs(e["reciprocal_group"] - want["reciprocal_group"]) <= 1e-5 * abs(want["reciprocal_group"])
    assert abs(e["exceptions"] - want["exceptions"]) <= 1e-5 * abs(want["exceptions"])
    assert e["pairs_within_cutoff"] == want["pairs_within_cutoff"]
    loop.destroy()


def test_peptide_one_step_with_shake(mdb, oracle, peptide):
    system, state = peptide
    loop = make_loop(mdb, system, state, seed=4)
    loop.run(1)
    p, v = loop.positions(), loop.velocities()
    op, ov, _ = oracle.run(system, state, 1, seed=4, grid=(50, 50, 50), threads=8)
    dp = np.abs(p - op).max()
    dv = np.abs(v - ov).max()
    print("peptide one step: max |dx|", dp, "max |dv|", dv)
    assert dp <= 4e-7, dp
    assert dv <= 4e-4, dv
    # every constraint holds to the SHAKE tolerance
    d = np.linalg.norm(p[system.constraint_p1] - p[system.constraint_p2], axis=1)
    assert np.max(np.abs(d / system.constraint_distance - 1)) < 2e-6
    loop.destroy()


@pytest.fixture(scope="module")
def octahedron():
    from mdb200 import synth

    return synth.config_octahedron_27k()


def test_octahedron_10k_steps_then_groups_match_oracle(mdb, oracle, octahedron):
    """The 27k-atom truncated octahedron, 10,000 LFMiddle steps, with the
    per-force-group energies and the forces checked against the f64 oracle on
    the same positions at steps 0, 1, 10 and every 1,000 (the configuration's
    schedule)."""
    system, state = octahedron
    loop = make_loop(mdb, system, state, seed=5)
    mesh = tuple(loop.mesh())
    checks = [0, 1, 10] + list(range(1000, 10001, 1000))
    done = 0
    for step in checks:
        loop.run(step - done)
        done = step
        e, f = loop.evaluate()
        pos, box = loop.positions(), loop.box_vectors()
        want, wf = oracle.potential(system, pos, box=box, grid=mesh, threads=8)
        err, change = force_error_allowing_cutoff_shell(oracle, system, pos, box, f, wf)
        print(f"octahedron step {step}: force rel RMS {err:.2e} (raw {rel_rms(f, wf):.2e}, "
              f"{change:+d} pairs at the cutoff), T {e['temperature']:.1f}")
        assert err <= FORCE_REL_RMS, (step, err)
        for key in ("bond", "angle", "torsion"):
            assert abs(e[key] - want[key]) <= 1e-5 * abs(want[key]) + 1e-3, (step, key, e[key], want[key])
        assert abs(e["direct_group"] - want["direct_group"]) <= 1e-4 * abs(want["direct_group"]), step
        assert abs(e["reciprocal_group"] - want["reciprocal_group"]) <= 1e-5 * abs(want["reciprocal_group"]), step
        assert abs(e["exceptions"] - want["exceptions"]) <= 1e-5 * abs(want["exceptions"]), step
        assert e["pairs_within_cutoff"] == want["pairs_within_cutoff"] + change, step
    assert loop.steps == state.step + 10000
    assert 200.0 < e["temperature"] < 400.0
    loop.destroy()


def test_autotune_picks_a_candidate_and_tuned_batch_equals_tuned_single(mdb):
    """The autotuner returns one of its candidates; a tuning passed per system
    to a batch gives the same trajectory as the same tuning on a single engine
    (the batch takes the first system's tile shape, so the single engines get
    it too)."""
    from mdb200 import synth

    a = synth.water_box(n_waters=700, width=2.8, seed=3, grid=(28, 28, 28))
    b = synth.water_box(n_waters=900, width=3.1, seed=4, grid=(32, 32, 32))
    best = mdb.autotune(*a, steps=50)
    print("autotune", best)
    assert best["candidates"] == 32
    assert best["verlet_skin"] in (0.15, 0.20, 0.30, 0.40, 0.50) and best["sort_cell"] in (0.20, 0.25, 0.35)
    assert best["tile_atoms"] in (8, 32) and best["prune_tiles"] in (1, 2)
    assert best["inner_skin"] in (-1.0, 0.08, 0.10)
    tuning = [(best["verlet_skin"], best["sort_cell"], best["tile_atoms"], best["prune_tiles"], best["inner_skin"]),
              (0.20, 0.35, 0, 0)]
    single = []
    for (s, st), t in zip((a, b), tuning):
        t = (t[0], t[1], tuning[0][2], tuning[0][3], t[4] if len(t) > 4 else 0.0)
        loop = mdb.StepLoop.from_parsed(s, st, mdb.RunOptions(seed=5, tuning=[t]))
        loop.run(30)
        single.append(loop.positions())
        assert abs(loop.verlet_flags()["skin"] - t[0]) < 1e-12
        loop.destroy()
    batch = mdb.StepLoop.batch([a[0], b[0]], [a[1], b[1]], mdb.RunOptions(seed=5, tuning=tuning))
    batch.run(30)
    assert np.array_equal(batch.positions(0), single[0])
    assert np.array_equal(batch.positions(1), single[1])
    batch.destroy()


def test_batched_autotune_searches_the_bucket_together(mdb):
    """`autotune_batch` times every candidate on one batched engine of all the
    systems given; `tune_by_bucket(batched=True)` runs it per size bucket on
    the bucket's own systems and hands each system its bucket's choice."""
    from mdb200 import synth

    members = [synth.water_box(n_waters=n, width=w, seed=k, grid=(30, 30, 30))
               for k, (n, w) in enumerate([(700, 2.8), (760, 2.9), (1500, 3.6)])]
    best = mdb.autotune_batch([m[0] for m in members[:2]], [m[1] for m in members[:2]], steps=30)
    print("autotune_batch", best)
    assert best["candidates"] == 20 and best["systems"] == 2  # the batch grid: 8-atom tiles only
    assert best["verlet_skin"] in (0.15, 0.20, 0.25, 0.30, 0.35, 0.40, 0.50) and best["tile_atoms"] == 8
    assert best["inner_skin"] in (-1.0, 0.06, 0.08, 0.10) and best["prune_tiles"] == 2
    assert best["ms_per_step"] > 0
    tuning, buckets = mdb.tune_by_bucket([m[0] for m in members], [m[1] for m in members], steps=30, batched=True)
    assert len(tuning) == 3 and len(buckets) == 2  # 2,100 and 2,280 atoms share a bucket; 4,500 is the next
    assert tuning[0] == tuning[1]
    assert buckets[mdb.size_bucket(members[0][0].particle_count)]["systems"] == 2


@pytest.mark.parametrize("shape,prune", [(8, 1), (8, 2), (32, 1), (32, 2)])
def test_every_tile_shape_and_pruning_matches_oracle(mdb, oracle, peptide, shape, prune):
    """The tuning options change the list, never the forces: each tile shape,
    with and without pruning, against the oracle on the peptide workload."""
    system, state = peptide
    loop = make_loop(mdb, system, state, tuning=[(0.2, 0.25, shape, prune)])
    e, f = loop.evaluate()
    loop.run(30)  # a few rebuilds' worth of dynamics on the same list settings
    e2, f2 = loop.evaluate()
    p2 = loop.positions()
    want2, wf2 = oracle.potential(system, p2, grid=(50, 50, 50), threads=8)
    loop.destroy()
    want, wf = oracle.potential(system, state.positions, grid=(50, 50, 50), threads=8)
    for got, ref, gf, rf, pos in ((e, want, f, wf, state.positions), (e2, want2, f2, wf2, p2)):
        err, change = force_error_allowing_cutoff_shell(oracle, system, pos, system.box, gf, rf)
        print(f"tiles {shape} prune {prune}: force rel RMS {err:.2e}, pairs {got['pairs_within_cutoff']}")
        assert err <= FORCE_REL_RMS, err
        assert got["pairs_within_cutoff"] == ref["pairs_within_cutoff"] + change


@pytest.mark.parametrize("shape", [8, 32])
def test_inner_list_changes_nothing(mdb, peptide, shape):
    """An inner list re-pruned between rebuilds drops only tiles that cannot
    reach inside the cutoff before the next prune, so the trajectory is
    bit-identical to the one on the whole list -- with fewer tiles read."""
    system, state = peptide
    runs = {}
    for inner in (-1.0, 0.06):
        loop = make_loop(mdb, system, state, seed=9, tuning=[(0.4, 0.2, shape, 2, inner)])
        loop.run(300)
        runs[inner] = (loop.positions(), loop.velocities(), loop.verlet_flags())
        loop.destroy()
    (p0, v0, f0), (p1, v1, f1) = runs[-1.0], runs[0.06]
    print("whole list", f0, "inner list", f1)
    assert f1["prunes"] > 10 and f1["rebuilds"] == f0["rebuilds"]
    assert f1["innerTiles"] < (0.8 if shape == 8 else 1.0) * f1["tiles"]
    assert np.array_equal(p0, p1) and np.array_equal(v0, v1)


def test_inner_list_on_a_small_cell_changes_nothing(mdb):
    """A 2.8 nm water box: every tile needs per-pair images (the cell is too
    small for one shift per tile); the inner prune takes those images too, drops
    tiles, and the trajectory stays bit-identical to the whole list's."""
    from mdb200 import synth

    system, state = synth.water_box(n_waters=700, width=2.8, seed=3, grid=(28, 28, 28))
    runs = {}
    for inner in (-1.0, 0.06):
        loop = make_loop(mdb, system, state, seed=9, tuning=[(0.4, 0.2, 8, 2, inner)])
        loop.run(300)
        runs[inner] = (loop.positions(), loop.velocities(), loop.verlet_flags())
        loop.destroy()
    (p0, v0, f0), (p1, v1, f1) = runs[-1.0], runs[0.06]
    print("small cell: whole list", f0, "inner list", f1)
    assert f1["prunes"] > 10 and f1["innerTiles"] < 0.9 * f1["tiles"]
    assert np.array_equal(p0, p1) and np.array_equal(v0, v1)


def test_tile_list_overflow_is_grown_and_rebuilt(mdb, oracle, peptide):
    """The reference never loses a pair when its list overflows
    (src/gpu/loop.ts:380-392).  Here a list that outgrows its capacity stops
    the integrator at that step; the host grows the list, rebuilds it and runs
    the remaining steps, so no step runs on a cut list.  The engine starts
    from a tiny capacity on the peptide box expanded by 25% per axis (molecule
    centres scaled, as the barostat moves them), so its list is grown while
    the engine is created; then it is given the real box and positions back,
    half again as dense as the capacity was grown for, so the first rebuild of
    the next run overflows mid-stride.  The forces match the oracle both times
    and the step count is exact."""
    from mdb200.system import State

    system, state = peptide
    scale = 1.25
    dilute = State(positions=oracle.scale_molecules(system, state.positions, scale),
                   box=np.asarray(state.box) * scale, velocities=state.velocities, step=state.step)
    loop = make_loop(mdb, system, dilute, seed=4, tile_row_capacity=16)
    flags = loop.verlet_flags()
    print("after creation", flags)
    assert flags["listGrown"] >= 1 and flags["overflowed"]
    e, f = loop.evaluate()
    want, wf = oracle.potential(system, dilute.positions, box=dilute.box, grid=(50, 50, 50), threads=8)
    err, change = force_error_allowing_cutoff_shell(oracle, system, dilute.positions, dilute.box, f, wf)
    print("grown list: force rel RMS", err)
    assert err <= FORCE_REL_RMS, err
    assert e["pairs_within_cutoff"] == want["pairs_within_cutoff"] + change
    loop.set_box(state.box)
    loop.set_positions(state.positions)
    grown = loop.verlet_flags()["listGrown"]
    loop.run(5)
    assert loop.steps == state.step + 5
    flags = loop.verlet_flags()
    print("back at the real density, after 5 steps", flags)
    assert flags["listGrown"] > grown
    e2, f2 = loop.evaluate()
    pos, box = loop.positions(), loop.box_vectors()
    want2, wf2 = oracle.potential(system, pos, box=box, grid=(50, 50, 50), threads=8)
    err2, change2 = force_error_allowing_cutoff_shell(oracle, system, pos, box, f2, wf2)
    print("after the mid-run growth: force rel RMS", err2)
    assert err2 <= FORCE_REL_RMS, err2
    assert e2["pairs_within_cutoff"] == want2["pairs_within_cutoff"] + change2
    loop.destroy()


def test_cell_geometry_and_passes_per_step(mdb, water):
    """`cellGeometry()` (loop.ts:894) gives the sort grid the list was built on
    -- divisions of the 3.0 nm box into cells of at least the 0.25 nm sort
    width, and their extent -- and `passesPerStep` (loop.ts:1105) the launches
    of one step, the same count the stage profile reports."""
    system, state = water
    loop = make_loop(mdb, system, state)
    cg = loop.cell_geometry()
    assert cg["divisions"] == (12, 12, 12)
    assert np.allclose(cg["extent"], 0.25)
    passes = loop.passes_per_step
    assert 8 <= passes <= 30
    assert loop.profile_step(repeats=2)["launches_per_step"] == passes
    loop.destroy()

