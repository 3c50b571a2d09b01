"""Write ff14sb_subset.json: the AMBER ff14SB residues and parameters the
synthetic peptide workloads use.

  python making-it-rain-webgpu_b200/mdb200/data/make_forcefield.py <making-it-rain-webgpu checkout>

Reads OpenMM's force-field XML as the reference project vendors it
(vendor/ffxml/protein.ff14SB.xml, MIT-licensed, from OpenMM) from the given
checkout of the reference, and keeps only what the builders in
mdb200/peptide.py need: the ALA, GLY, LYS, GLU, ACE and NME templates, the
atom types they use, and every bond, angle, proper/improper torsion and
Lennard-Jones entry whose types are among those (or wildcards).  The JSON it
writes is committed next to this script.
"""

from __future__ import annotations

import argparse
import json
import xml.etree.ElementTree as ET
from pathlib import Path

FFXML = Path("vendor/ffxml/protein.ff14SB.xml")  # inside the reference checkout
OUT = Path(__file__).resolve().parent / "ff14sb_subset.json"
RESIDUES = ("ALA", "GLY", "LYS", "GLU", "ACE", "NME")


def main() -> None:
    ap = argparse.ArgumentParser(description="write ff14sb_subset.json from the reference's vendored ff14SB")
    ap.add_argument("reference", type=Path, help="root of a making-it-rain-webgpu checkout")
    root = ET.parse(ap.parse_args().reference / FFXML).getroot()
    types = {t.get("name"): {"class": t.get("class"), "element": t.get("element"), "mass": float(t.get("mass"))}
             for t in root.find("AtomTypes")}
    residues = {}
    used = set()
    for r in root.find("Residues"):
        name = r.get("name")
        if name not in RESIDUES:
            continue
        atoms = [{"name": a.get("name"), "type": a.get("type"), "charge": float(a.get("charge"))}
                 for a in r.findall("Atom")]
        bonds = [[b.get("atomName1"), b.get("atomName2")] for b in r.findall("Bond")]
        external = [e.get("atomName") for e in r.findall("ExternalBond")]
        residues[name] = {"atoms": atoms, "bonds": bonds, "external": external}
        used.update(a["type"] for a in atoms)

    def ok(*names):
        return all(n == "" or n in used for n in names)

    bonds = [{"types": [b.get("type1"), b.get("type2")], "length": float(b.get("length")), "k": float(b.get("k"))}
             for b in root.find("HarmonicBondForce") if ok(b.get("type1"), b.get("type2"))]
    angles = [{"types": [a.get(f"type{i}") for i in (1, 2, 3)], "angle": float(a.get("angle")),
               "k": float(a.get("k"))}
              for a in root.find("HarmonicAngleForce") if ok(*(a.get(f"type{i}") for i in (1, 2, 3)))]

    def terms(e):
        out = []
        i = 1
        while e.get(f"k{i}") is not None:
            out.append([int(e.get(f"periodicity{i}")), float(e.get(f"phase{i}")), float(e.get(f"k{i}"))])
            i += 1
        return out

    torsion = root.find("PeriodicTorsionForce")
    propers = [{"types": [p.get(f"type{i}") for i in (1, 2, 3, 4)], "terms": terms(p)}
               for p in torsion.findall("Proper") if ok(*(p.get(f"type{i}") for i in (1, 2, 3, 4)))]
    impropers = [{"types": [p.get(f"type{i}") for i in (1, 2, 3, 4)], "terms": terms(p)}
                 for p in torsion.findall("Improper") if ok(*(p.get(f"type{i}") for i in (1, 2, 3, 4)))]
    nb = root.find("NonbondedForce")
    lj = {a.get("type"): {"sigma": float(a.get("sigma")), "epsilon": float(a.get("epsilon"))}
          for a in nb.findall("Atom") if a.get("type") in used}
    data = {
        "source": "vendor/ffxml/protein.ff14SB.xml (OpenMM's AMBER ff14SB), subset",
        "types": {k: v for k, v in types.items() if k in used},
        "residues": residues,
        "bonds": bonds,
        "angles": angles,
        "propers": propers,
        "impropers": impropers,
        "improper_ordering": torsion.get("ordering"),
        "lj": lj,
        "coulomb14scale": float(nb.get("coulomb14scale")),
        "lj14scale": float(nb.get("lj14scale")),
    }
    OUT.write_text(json.dumps(data, indent=0) + "\n")
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes): {len(bonds)} bonds, {len(angles)} angles, "
          f"{len(propers)} propers, {len(impropers)} impropers")


if __name__ == "__main__":
    main()
