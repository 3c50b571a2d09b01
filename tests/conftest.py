"""Shared test set-up: import paths, the `gpu` marker, and golden fixtures."""

from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT / "making-it-rain-webgpu_b200"))
sys.path.insert(0, str(ROOT))
GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built engine")
    config.addinivalue_line("markers", "slow: long CPU oracle runs")


def golden(name: str) -> dict:
    return json.loads((GOLDEN / f"{name}.json").read_text())


def golden_nonbonded_system():
    """The reference's committed 10-particle fixture as a System and State."""
    from mdb200.system import Nonbonded, State, System

    g = golden("nonbonded")
    parts = np.array(g["particles"], dtype=np.float64)
    exc = g["exceptions"]
    system = System(
        masses=np.array(g["masses"]),
        box=np.array(g["box"]),
        nonbonded=Nonbonded(
            cutoff=g["cutoff"], ewald_tolerance=g["ewald_tolerance"],
            charge=parts[:, 0].copy(), sigma=parts[:, 1].copy(), epsilon=parts[:, 2].copy(),
            exception_p1=np.array([e[0] for e in exc], dtype=np.int32),
            exception_p2=np.array([e[1] for e in exc], dtype=np.int32),
            exception_charge_prod=np.array([e[2] for e in exc]),
            exception_sigma=np.array([e[3] for e in exc]),
            exception_epsilon=np.array([e[4] for e in exc]),
            use_dispersion_correction=g["dispersion_correction"],
        ),
    )
    state = State(positions=np.array(g["positions"]), box=np.array(g["box"]))
    return system, state, g


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as orc

    orc.lib()
    return orc


def rel_rms(a, b) -> float:
    a = np.asarray(a).reshape(-1)
    b = np.asarray(b).reshape(-1)
    return float(np.sqrt(((a - b) ** 2).sum() / (b**2).sum()))


# Pair coordinates are int32 at 2^-26 nm or finer and pair distances are f32,
# so a pair closer than this to the cutoff may fall on either side of it.
CUTOFF_SHELL_NM = 2e-7


def force_error_allowing_cutoff_shell(orc, system, positions, box, forces, want_forces):
    """Relative RMS force error against the oracle, where each pair within
    CUTOFF_SHELL_NM of the cutoff counts as inside or outside, whichever the
    engine's forces agree with (the truncated potential jumps there, by up to
    ~0.3 kJ/mol/nm for a water O-O pair, so one such pair alone can exceed the
    whole force budget).  Returns (error, pair-count change): the engine's
    pairs_within_cutoff must equal the oracle's plus that change."""
    first, second, pair_force, inside = orc.cutoff_shell(system, positions, box=box, eps=CUTOFF_SHELL_NM)
    f = np.asarray(forces, dtype=np.float64).reshape(-1, 3)
    want = np.array(want_forces, dtype=np.float64).reshape(-1, 3)
    change = 0
    for a, b, g, ins in zip(first, second, pair_force, inside):
        if not np.any(g):
            continue
        sign = -1.0 if ins else 1.0
        now = ((f[a] - want[a]) ** 2).sum() + ((f[b] - want[b]) ** 2).sum()
        other = ((f[a] - want[a] - sign * g) ** 2).sum() + ((f[b] - want[b] + sign * g) ** 2).sum()
        if other < now:
            want[a] += sign * g
            want[b] -= sign * g
            change += -1 if ins else 1
    return rel_rms(f, want), change
