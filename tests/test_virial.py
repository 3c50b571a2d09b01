"""The virial tensor W_ab = sum r_a F_b = -dU/d eps_ab (strain x -> (1 + eps) x).

The reference has no virial; the engine reports one for the barostat's
screening network and for pressure.  The f64 oracle's analytic virial is
pinned here against central finite differences of its own energy under small
symmetric strains of positions and box (re-rotated into OpenMM's reduced box
form, which leaves the energy unchanged); the GPU test compares the engine
with that oracle.
"""

from __future__ import annotations

import numpy as np
import pytest


def _reduced(box, pos):
    """Rotate so a lies along x and b in the xy plane (QR of the box)."""
    q, r = np.linalg.qr(box.T)
    sign = np.sign(np.diag(r))
    rot = (q * sign).T
    return (rot @ box.T).T, pos @ rot.T


def _finite_difference_virial(oracle, system, pos, box, grid, h=1e-7):
    fd = np.zeros((3, 3))
    for a in range(3):
        for b in range(a, 3):
            eps = np.zeros((3, 3))
            eps[a, b] += h / 2
            eps[b, a] += h / 2
            u = []
            for sgn in (1.0, -1.0):
                t = np.eye(3) + sgn * eps
                bx, px = _reduced(box @ t.T, pos @ t.T)
                e, _ = oracle.potential(system, px, box=bx, grid=grid, threads=4, forces=False)
                u.append(e["potential"])
            fd[a, b] = fd[b, a] = -(u[0] - u[1]) / (2 * h)
    return fd


def test_oracle_virial_is_minus_the_strain_derivative(oracle):
    """Solvated Ala4 (bonds, angles, torsions, exceptions, PME, dispersion)."""
    from mdb200 import peptide, synth

    solute, x = peptide.helix(["ALA"] * 4)
    system, state = synth.solvated(solute, x, width=2.6, seed=2, grid=(26, 26, 26))
    box = np.asarray(state.box)
    _, _, w = oracle.potential_virial(system, state.positions, box=box, grid=(26, 26, 26), threads=4)
    assert np.abs(w - w.T).max() < 1e-8 * np.abs(w).max()
    fd = _finite_difference_virial(oracle, system, state.positions, box, (26, 26, 26))
    print("analytic\n", w, "\nfinite difference\n", fd)
    assert np.abs(0.5 * (w + w.T) - fd).max() < 2e-6 * np.abs(w).max()


@pytest.mark.gpu
@pytest.mark.parametrize("workload", ["water", "peptide"])
def test_engine_virial_matches_oracle(oracle, workload):
    from mdb200 import steploop, synth

    if workload == "water":
        system, state = synth.config_water_2652()
        grid = (30, 30, 30)
    else:
        system, state = synth.config_peptide_12k()
        grid = (50, 50, 50)
    loop = steploop.StepLoop.from_parsed(system, state, steploop.RunOptions())
    e, _ = loop.evaluate()
    loop.destroy()
    _, _, want = oracle.potential_virial(system, state.positions, grid=grid, threads=8)
    got = np.array(e["virial"]).reshape(3, 3)
    err = np.abs(got - want).max() / np.abs(want).max()
    print(workload, "virial\n", got, "\noracle\n", want, "\nmax rel", err)
    assert err < 2e-5, err


@pytest.mark.gpu
def test_engine_molecular_virial_is_the_molecular_scaling_derivative(oracle):
    """tr(W_mol) = -dU/d ln s under scaling of molecule centres by s (the
    barostat's move), by central differences of the oracle's energy."""
    from mdb200 import steploop, synth

    system, state = synth.water_box(n_waters=700, width=2.8, seed=5, grid=(28, 28, 28))
    loop = steploop.StepLoop.from_parsed(system, state, steploop.RunOptions(mesh=(28, 28, 28)))
    e, _ = loop.evaluate()
    loop.destroy()
    w_mol = np.array(e["molecular_virial"]).reshape(3, 3)
    box = np.asarray(state.box)
    h = 1e-7
    u = []
    for sgn in (1.0, -1.0):
        s = np.exp(sgn * h)
        p = oracle.scale_molecules(system, state.positions, s).reshape(-1, 3)
        en, _ = oracle.potential(system, p, box=box * s, grid=(28, 28, 28), threads=8, forces=False)
        u.append(en["potential"])
    fd = -(u[0] - u[1]) / (2 * h)
    print("tr W_mol", np.trace(w_mol), "finite difference", fd, "tr W (atomic)", sum(e["virial"][::4]))
    assert abs(np.trace(w_mol) - fd) < 2e-5 * abs(fd) + 0.5
