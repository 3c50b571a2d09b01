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
