"""Regenerate the golden fixtures in this folder from the reference's own tests.

  python tests/golden/make_golden.py <making-it-rain-webgpu checkout>

The argument is the root of a checkout of the reference project (read only).
Every value written here is read out of the reference's committed test data
or test source, as text; nothing is computed.

  nonbonded.json   test/fixtures/nonbonded-{system,state}.xml and
                   nonbonded-facts.json: OpenMM 8.4 PME and Ewald group
                   energies, per-atom forces, the term decomposition, and the
                   dispersion value asserted at test/nonbonded-reference.test.ts:95.
  random_kat.json  the threefry2x32 known-answer rows of test/random.test.ts
                   (Random123's own tests/kat_vectors).
  erf.json         the mpmath-pinned erf/erfc table of test/erf.test.ts.
  fixed_words.json the exact word layouts asserted in test/fixed-point.test.ts.
  triclinic.json   test/fixtures/triclinic-openmm.json, cases and separations.
"""

from __future__ import annotations

import argparse
import json
import re
import xml.etree.ElementTree as ET
from pathlib import Path

REFERENCE = Path(".")  # set by main() from the command line
OUT = Path(__file__).resolve().parent


def nonbonded() -> dict:
    system = ET.parse(REFERENCE / "test/fixtures/nonbonded-system.xml").getroot()
    state = ET.parse(REFERENCE / "test/fixtures/nonbonded-state.xml").getroot()
    facts = json.loads((REFERENCE / "test/fixtures/nonbonded-facts.json").read_text())
    force = [f for f in system.iter("Force") if f.get("type") == "NonbondedForce"][0]
    box = [[float(v.get(a)) for a in "xyz"] for v in system.find("PeriodicBoxVectors")]
    out = {
        "source": "test/fixtures/nonbonded-{system,state}.xml + nonbonded-facts.json",
        "box": box,
        "masses": [float(p.get("mass")) for p in system.find("Particles")],
        "cutoff": float(force.get("cutoff")),
        "ewald_tolerance": float(force.get("ewaldTolerance")),
        "dispersion_correction": force.get("dispersionCorrection") == "1",
        "particles": [[float(p.get(k)) for k in ("q", "sig", "eps")]
                      for p in force.find("Particles")],
        "exceptions": [[int(e.get("p1")), int(e.get("p2"))] + [float(e.get(k)) for k in ("q", "sig", "eps")]
                       for e in force.find("Exceptions")],
        "positions": [[float(p.get(a)) for a in "xyz"] for p in state.find("Positions")],
        "state_forces": [[float(p.get(a)) for a in "xyz"] for p in state.find("Forces")],
        "PME": facts["PME"],
        "Ewald": facts["Ewald"],
        "decomposition": facts["decomposition"],
        # test/nonbonded-reference.test.ts:95 -- measured against OpenMM.
        "dispersion_openmm": -0.020466041,
    }
    return out


def random_kat() -> dict:
    text = (REFERENCE / "test/random.test.ts").read_text()
    rows = re.findall(r'\[\s*(\d+),\s*"([0-9a-f ]+)",\s*"([0-9a-f ]+)"\s*\]', text)
    cases = [{"rounds": int(r), "input": [int(w, 16) for w in i.split()],
              "output": [int(w, 16) for w in o.split()]} for r, i, o in rows]
    return {"source": "test/random.test.ts KNOWN_ANSWERS (Random123 tests/kat_vectors)", "cases": cases}


def erf_table() -> dict:
    text = (REFERENCE / "test/erf.test.ts").read_text()
    block = text[text.index("const KNOWN"):text.index("];", text.index("const KNOWN"))]
    rows = re.findall(r"\[\s*([0-9.e+-]+),\s*([0-9.e+-]+),\s*([0-9.e+-]+)\s*\]", block)
    return {"source": "test/erf.test.ts KNOWN (mpmath, 30 digits)",
            "rows": [[float(a), float(b), float(c)] for a, b, c in rows]}


def fixed_words() -> dict:
    text = (REFERENCE / "test/fixed-point.test.ts").read_text()
    rows = re.findall(r"fixedWords\((-?[0-9.]+)\)\)\.toEqual\(\{ lo: ([^,]+), hi: (-?\d+) \}\)", text)

    def value(expr: str) -> int:
        expr = expr.strip()
        m = re.fullmatch(r"2 \*\* (\d+)", expr)
        return 2 ** int(m.group(1)) if m else int(expr)

    return {"source": "test/fixed-point.test.ts", "cases": [
        {"value": float(v), "lo": value(lo), "hi": int(hi)} for v, lo, hi in rows]}


def triclinic() -> dict:
    data = json.loads((REFERENCE / "test/fixtures/triclinic-openmm.json").read_text())
    cases = []
    for case in data["cases"]:
        cases.append({k: case[k] for k in ("shape", "width_nm", "cutoff_nm", "reduced_vectors", "pairs")})
    return {"source": "test/fixtures/triclinic-openmm.json", "openmm_version": data["openmm_version"],
            "cases": cases}


def main() -> None:
    global REFERENCE
    ap = argparse.ArgumentParser(description="regenerate the golden fixtures from the reference's tests")
    ap.add_argument("reference", type=Path, help="root of a making-it-rain-webgpu checkout")
    REFERENCE = ap.parse_args().reference
    for name, make in (("nonbonded", nonbonded), ("random_kat", random_kat), ("erf", erf_table),
                       ("fixed_words", fixed_words), ("triclinic", triclinic)):
        path = OUT / f"{name}.json"
        path.write_text(json.dumps(make(), indent=1) + "\n")
        print(f"wrote {path} ({path.stat().st_size} bytes)")


if __name__ == "__main__":
    main()
