"""Host-side logic without a GPU: the OpenMM XML contract, the synthetic
workload builders, and the peptide parameterisation, checked against the
reference's rules and against the f64 oracle."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import golden_nonbonded_system


def test_system_xml_round_trip():
    """parseSystem / serialiseSystem (src/engine/system.ts:521, :619)."""
    from mdb200 import peptide, synth
    from mdb200.system import parse_system, serialise_system

    solute, pos = peptide.helix(["ALA"] * 3)
    system, state = synth.solvated(solute, pos, width=3.0, seed=2, grid=(30, 30, 30))
    again = parse_system(serialise_system(system))
    assert again.particle_count == system.particle_count
    assert np.array_equal(again.masses, system.masses)
    assert np.array_equal(again.constraint_p1, system.constraint_p1)
    assert np.allclose(again.constraint_distance, system.constraint_distance, rtol=0, atol=0)
    for a, b in zip(again.torsions, system.torsions):
        assert np.array_equal(np.asarray(a), np.asarray(b))
    assert np.array_equal(again.nonbonded.exception_charge_prod, system.nonbonded.exception_charge_prod)
    assert again.com_frequency == system.com_frequency


def test_state_xml_round_trip():
    from mdb200 import synth
    from mdb200.system import parse_state, serialise_state

    _, state = synth.water_box(n_waters=30, width=2.2, seed=5)
    state.step = 1234
    again = parse_state(serialise_state(state))
    assert again.step == 1234
    assert np.array_equal(again.positions, state.positions)
    assert np.array_equal(again.velocities, state.velocities)


@pytest.mark.parametrize("force,detail", [
    ('<Force type="AndersenThermostat"/>', "AndersenThermostat"),
    ('<Force type="NonbondedForce" method="5" cutoff="1" ewaldTolerance="0.0005"><Particles/></Force>', "LJ-PME"),
    ('<Force type="CustomExternalForce" energy="k*x^2"><PerParticleParameters/><Particles/></Force>', "energy expression"),
])
def test_unsupported_forces_are_refused_by_name(force, detail):
    """UnsupportedForce, src/engine/system.ts:178."""
    from mdb200.system import UnsupportedForce, parse_system

    xml = ('<System><PeriodicBoxVectors><A x="3" y="0" z="0"/><B x="0" y="3" z="0"/><C x="0" y="0" z="3"/>'
           '</PeriodicBoxVectors><Particles><Particle mass="1"/></Particles><Constraints/>'
           f'<Forces>{force}</Forces></System>')
    with pytest.raises(UnsupportedForce, match=detail):
        parse_system(xml)


def test_reference_fixture_parses_to_the_golden_system():
    from mdb200.system import parse_system
    from pathlib import Path

    system, state, g = golden_nonbonded_system()
    assert system.particle_count == 10
    assert system.nonbonded.cutoff == g["cutoff"]


def test_water_box_is_rigid_and_neutral():
    from mdb200 import synth

    system, state = synth.config_water_2652()
    assert system.particle_count == 2652
    p = state.positions
    d = np.linalg.norm(p[system.constraint_p1] - p[system.constraint_p2], axis=1)
    assert np.max(np.abs(d - system.constraint_distance)) < 1e-12
    assert abs(system.nonbonded.charge.sum()) < 1e-9
    assert len(system.nonbonded.exception_p1) == 3 * 884


def test_peptide_workload_matches_the_configuration():
    """The peptide workload: Ala20 helix + caps, 5 nm TIP3P cube, 0.15 M NaCl, ~12,000 atoms."""
    from mdb200 import synth
    from oracle import oracle

    system, state = synth.config_peptide_12k()
    assert 11_500 < system.particle_count < 12_800
    assert abs(system.nonbonded.charge.sum()) < 1e-9
    status, (settle, shake, atoms, constraints) = oracle.split_counts(system)
    assert status == 0 and settle > 3900 and shake > 50
    assert atoms <= 8 and constraints <= 8
    p = state.positions
    d = np.linalg.norm(p[system.constraint_p1] - p[system.constraint_p2], axis=1)
    assert np.max(np.abs(d - system.constraint_distance)) < 1e-9


def test_helix_parameters_follow_ff14sb():
    from mdb200 import peptide

    system, pos = peptide.helix(["ALA"] * 20)
    assert system.particle_count == 212  # 20 x 10 + ACE 6 + NME 6
    p1, p2, length, k = system.bonds
    d = np.linalg.norm(pos[p1] - pos[p2], axis=1)
    assert np.max(np.abs(d - length)) < 2e-3
    # every X-H bond is a constraint (HBonds), none of them a harmonic term
    ff = peptide.forcefield()
    assert system.constraint_count == 107
    # 1-4 exceptions carry the ff14SB scale factors
    q = system.nonbonded.charge
    for a, b, qq, s, e in zip(system.nonbonded.exception_p1, system.nonbonded.exception_p2,
                              system.nonbonded.exception_charge_prod, system.nonbonded.exception_sigma,
                              system.nonbonded.exception_epsilon):
        if qq != 0.0:
            assert abs(qq - q[a] * q[b] * ff["coulomb14scale"]) < 1e-12


def test_helix_potential_is_sane_in_the_oracle():
    from mdb200 import peptide
    from oracle import oracle

    system, pos = peptide.helix(["ALA"] * 8)
    system.box = np.eye(3) * 4.0
    e, f = oracle.potential(system, pos + 2.0, box=np.eye(3) * 4.0, grid=(40, 40, 40))
    assert np.isfinite(e["potential"]) and np.abs(f).max() < 5e3
    assert e["bond"] < 10 and e["angle"] < 50


def test_oracle_verlet_conserves_energy_without_friction():
    """A short NVE run of a small box through the oracle's loop (integrator.ts:68)."""
    from mdb200 import synth
    from oracle import oracle
    from mdb200.system import State

    g = (24, 24, 24)
    system, state = synth.water_box(n_waters=300, width=2.2, seed=4, grid=g, com_frequency=0)
    # relax the lattice first with a friction run
    p, v, step = oracle.run(system, state, 30, friction=50.0, seed=1, grid=g, threads=4)
    st = State(positions=p, box=state.box, velocities=v, step=step)
    e0 = oracle.potential(system, p, grid=g, forces=False)[0]["potential"] + oracle.kinetic_energy(system, v)
    p2, v2, _ = oracle.run(system, st, 20, friction=0.0, integrator=1, time_step=0.0005, grid=g, threads=4)
    e1 = oracle.potential(system, p2, grid=g, forces=False)[0]["potential"] + oracle.kinetic_energy(system, v2)
    assert abs(e1 - e0) < 0.05 * abs(oracle.kinetic_energy(system, v2))


def test_ions_for_concentration():
    from mdb200 import synth

    assert synth.ions_for(125.0, 0.15) == 11
    assert synth.ions_for(1000.0, 0.15) == 90


def test_octahedron_workload_matches_the_configuration(oracle):
    """60-residue (AGKE)15 coil, truncated octahedron at 1.0 nm padding, ~27k atoms."""
    from mdb200 import peptide, synth

    solute, x = peptide.coil()
    radius = peptide.bounding_radius(x)
    assert 2.95 <= radius <= 3.1
    system, state = synth.config_octahedron_27k()
    box = np.asarray(state.box)
    width = 2 * radius + 1.0  # solvate.ts:390
    assert np.allclose(box, synth.box_vectors("octahedron", width))
    assert 25000 <= system.particle_count <= 29000
    assert abs(system.nonbonded.charge.sum()) < 1e-9
    names = [a[2] for a in peptide.build_chain(peptide.AGKE60, 0.0, 0.0)]
    assert solute.particle_count == len(names) == 822
    # no clashes: every solute pair at least two residues apart keeps its distance
    res = np.array([a[0] for a in peptide.build_chain(peptide.AGKE60, 0.0, 0.0)])
    d = np.linalg.norm(x[:, None] - x[None], axis=-1)
    assert d[np.abs(res[:, None] - res[None]) >= 2].min() >= 0.2
    status, (settle, iterative, largest_atoms, largest_constraints) = oracle.split_counts(system)
    assert status == 0 and iterative > 0
    assert largest_atoms <= 4 and largest_constraints <= 3
