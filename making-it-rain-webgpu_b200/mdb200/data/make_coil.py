"""Write coil_angles.json: the backbone angles of the seeded AGKE60 coil.

The growth search (`peptide.coil_angles`) takes a while, so this script runs
it once: seeds from 11 upwards, each with a bounded number of draws, and the
first seed that converges is stored with its angles next to this script for
`peptide.coil` to read.  Re-running reproduces the file exactly.

    python making-it-rain-webgpu_b200/mdb200/data/make_coil.py
"""

from __future__ import annotations

import json
import sys
from pathlib import Path

sys.path.insert(0, str(Path(__file__).resolve().parents[2]))

from mdb200 import peptide  # noqa: E402


def main() -> None:
    for seed in range(11, 60):
        try:
            phi, psi = peptide.coil_angles(peptide.AGKE60, seed)
        except RuntimeError:
            continue
        table = {"sequence": list(peptide.AGKE60), "seed": seed,
                 "phi": [round(float(v), 12) for v in phi], "psi": [round(float(v), 12) for v in psi]}
        peptide.COIL_DATA.write_text(json.dumps(table) + "\n")
        print("wrote", peptide.COIL_DATA, "seed", seed)
        return
    raise SystemExit("no seed converged")


if __name__ == "__main__":
    main()
