"""Capped peptides with AMBER ff14SB parameters, built from scratch.

The synthetic solute of the benchmark workloads: ACE-(residues)-NME chains of
ALA, GLY, LYS and GLU with ideal internal geometry, placed by the
natural-extension reference frame (NeRF) method from bond lengths, angles and
dihedrals, then parameterised the way OpenMM's `ForceField.createSystem`
parameterises a protein (bonds, angles, proper torsions with the fewest
wildcards winning, AMBER-ordered impropers, 1-2/1-3 exclusions, scaled 1-4
exceptions, HBond constraints in place of X-H bonds).  Parameters come from
data/ff14sb_subset.json, a subset of vendor/ffxml/protein.ff14SB.xml.
"""

from __future__ import annotations

import itertools
import json
import math
from functools import lru_cache
from pathlib import Path

import numpy as np

from .system import Nonbonded, System

DATA = Path(__file__).resolve().parent / "data" / "ff14sb_subset.json"
ANGSTROM = 0.1


@lru_cache(maxsize=1)
def forcefield() -> dict:
    return json.loads(DATA.read_text())


def place(a, b, c, bond, angle_deg, dihedral_deg):
    """NeRF: the point d with |cd| = bond, angle(b, c, d), dihedral(a, b, c, d)."""
    angle, dih = math.radians(angle_deg), math.radians(dihedral_deg)
    bc = c - b
    bc /= np.linalg.norm(bc)
    n = np.cross(b - a, bc)
    n /= np.linalg.norm(n)
    m = np.cross(n, bc)
    d2 = np.array([-bond * math.cos(angle), bond * math.sin(angle) * math.cos(dih),
                   bond * math.sin(angle) * math.sin(dih)])
    return c + d2[0] * bc + d2[1] * m + d2[2] * n


def build_chain(sequence, phi, psi, omega=180.0):
    """Atoms (residue index, residue name, atom name, xyz nm) of ACE-seq-NME.

    `phi` and `psi` are per-residue lists (degrees) or scalars.
    """
    n = len(sequence)
    phi = [phi] * n if np.isscalar(phi) else list(phi)
    psi = [psi] * n if np.isscalar(psi) else list(psi)
    atoms = []

    def add(res, rname, name, xyz):
        atoms.append((res, rname, name, np.asarray(xyz, dtype=np.float64)))
        return atoms[-1][3]

    # ACE: methyl carbon at the origin, carbonyl along x, a reference point in the plane
    ch3 = add(0, "ACE", "CH3", [0.0, 0.0, 0.0])
    c_prev = add(0, "ACE", "C", [1.522 * ANGSTROM, 0.0, 0.0])
    ref = np.array([-0.5 * ANGSTROM, 1.0 * ANGSTROM, 0.0])
    n_prev, ca_prev = ref, ch3
    psi_prev = 180.0
    backbone = []
    for i, rname in enumerate(sequence):
        res = i + 1
        N = place(n_prev, ca_prev, c_prev, 1.335 * ANGSTROM, 116.2, psi_prev)
        CA = place(ca_prev, c_prev, N, 1.458 * ANGSTROM, 121.7, omega)
        C = place(c_prev, N, CA, 1.525 * ANGSTROM, 111.2, phi[i])
        backbone.append((res, rname, N, CA, C))
        n_prev, ca_prev, c_prev = N, CA, C
        psi_prev = psi[i]
    N_nme = place(n_prev, ca_prev, c_prev, 1.335 * ANGSTROM, 116.2, psi_prev)
    CH3_nme = place(ca_prev, c_prev, N_nme, 1.449 * ANGSTROM, 121.9, omega)

    # ACE carbonyl O and methyl hydrogens
    first_N, first_CA = backbone[0][2], backbone[0][3]
    O_ace = add(0, "ACE", "O", place(first_CA, first_N, c_prev if n == 0 else atoms[1][3], 1.229 * ANGSTROM, 122.9, 0.0))
    for k, d in enumerate((60.0, 180.0, 300.0)):
        add(0, "ACE", f"HH3{k + 1}", place(first_N, atoms[1][3], ch3, 1.09 * ANGSTROM, 109.5, d))

    prev_C, prev_O = atoms[1][3], O_ace
    for idx, (res, rname, N, CA, C) in enumerate(backbone):
        nxt_N = backbone[idx + 1][2] if idx + 1 < n else N_nme
        add(res, rname, "N", N)
        add(res, rname, "H", place(prev_O, prev_C, N, 1.01 * ANGSTROM, 119.8, 180.0))
        add(res, rname, "CA", CA)
        if rname == "GLY":
            add(res, rname, "HA2", place(N, C, CA, 1.09 * ANGSTROM, 109.5, 122.6))
            add(res, rname, "HA3", place(N, C, CA, 1.09 * ANGSTROM, 109.5, -118.0))
        else:
            add(res, rname, "HA", place(N, C, CA, 1.09 * ANGSTROM, 109.5, -118.0))
            CB = add(res, rname, "CB", place(N, C, CA, 1.526 * ANGSTROM, 110.1, 122.6))
            if rname == "ALA":
                for k, d in enumerate((60.0, 180.0, 300.0)):
                    add(res, rname, f"HB{k + 1}", place(N, CA, CB, 1.09 * ANGSTROM, 109.5, d))
            else:
                CG = place(N, CA, CB, 1.53 * ANGSTROM, 113.8, 180.0)
                add(res, rname, "HB2", place(N, CA, CB, 1.09 * ANGSTROM, 109.5, 60.0))
                add(res, rname, "HB3", place(N, CA, CB, 1.09 * ANGSTROM, 109.5, 300.0))
                add(res, rname, "CG", CG)
                add(res, rname, "HG2", place(CA, CB, CG, 1.09 * ANGSTROM, 109.5, 60.0))
                add(res, rname, "HG3", place(CA, CB, CG, 1.09 * ANGSTROM, 109.5, 300.0))
                if rname == "LYS":
                    CD = add(res, rname, "CD", place(CA, CB, CG, 1.53 * ANGSTROM, 111.8, 180.0))
                    add(res, rname, "HD2", place(CB, CG, CD, 1.09 * ANGSTROM, 109.5, 60.0))
                    add(res, rname, "HD3", place(CB, CG, CD, 1.09 * ANGSTROM, 109.5, 300.0))
                    CE = add(res, rname, "CE", place(CB, CG, CD, 1.53 * ANGSTROM, 111.8, 180.0))
                    add(res, rname, "HE2", place(CG, CD, CE, 1.09 * ANGSTROM, 109.5, 60.0))
                    add(res, rname, "HE3", place(CG, CD, CE, 1.09 * ANGSTROM, 109.5, 300.0))
                    NZ = add(res, rname, "NZ", place(CG, CD, CE, 1.47 * ANGSTROM, 111.5, 180.0))
                    for k, d in enumerate((60.0, 180.0, 300.0)):
                        add(res, rname, f"HZ{k + 1}", place(CD, CE, NZ, 1.01 * ANGSTROM, 109.5, d))
                elif rname == "GLU":
                    CD = add(res, rname, "CD", place(CA, CB, CG, 1.52 * ANGSTROM, 113.0, 180.0))
                    add(res, rname, "OE1", place(CB, CG, CD, 1.25 * ANGSTROM, 118.4, 90.0))
                    add(res, rname, "OE2", place(CB, CG, CD, 1.25 * ANGSTROM, 118.4, -90.0))
                else:
                    raise ValueError(f"no builder for residue {rname}")
        add(res, rname, "C", C)
        O = add(res, rname, "O", place(nxt_N, CA, C, 1.229 * ANGSTROM, 120.5, 180.0))
        prev_C, prev_O = C, O
    last = n + 1
    add(last, "NME", "N", N_nme)
    add(last, "NME", "H", place(prev_O, prev_C, N_nme, 1.01 * ANGSTROM, 119.8, 180.0))
    add(last, "NME", "CH3", CH3_nme)
    for k, d in enumerate((60.0, 180.0, 300.0)):
        add(last, "NME", f"HH3{k + 1}", place(prev_C, N_nme, CH3_nme, 1.09 * ANGSTROM, 109.5, d))
    return atoms


def _match(pattern, types):
    return all(p == "" or p == t for p, t in zip(pattern, types))


def parameterise(atoms, constrain_hbonds: bool = True, cutoff: float = 1.0, ewald_tolerance: float = 5e-4):
    """A System for the chain, parameterised from the ff14SB subset."""
    ff = forcefield()
    n = len(atoms)
    index = {}
    types, charges = [], []
    for i, (res, rname, name, _) in enumerate(atoms):
        tpl = {a["name"]: a for a in ff["residues"][rname]["atoms"]}
        if name not in tpl:
            raise ValueError(f"{rname} has no atom {name}")
        types.append(tpl[name]["type"])
        charges.append(tpl[name]["charge"])
        index[(res, name)] = i
    bonds = set()
    residues = sorted({a[0] for a in atoms})
    rname_of = {a[0]: a[1] for a in atoms}
    for res in residues:
        for a, b in ff["residues"][rname_of[res]]["bonds"]:
            bonds.add(tuple(sorted((index[(res, a)], index[(res, b)]))))
        if res + 1 in rname_of:
            bonds.add(tuple(sorted((index[(res, "C")], index[(res + 1, "N")]))))
    adj = [set() for _ in range(n)]
    for a, b in bonds:
        adj[a].add(b)
        adj[b].add(a)
    element = [ff["types"][t]["element"] for t in types]
    masses = np.array([ff["types"][t]["mass"] for t in types])

    def bond_param(a, b):
        for d in ff["bonds"]:
            if _match(d["types"], (types[a], types[b])) or _match(d["types"], (types[b], types[a])):
                return d["length"], d["k"]
        raise ValueError(f"no bond parameters for {types[a]}-{types[b]}")

    bp1, bp2, blen, bk = [], [], [], []
    cp1, cp2, cd = [], [], []
    for a, b in sorted(bonds):
        length, k = bond_param(a, b)
        if constrain_hbonds and (element[a] == "H" or element[b] == "H"):
            cp1.append(a)
            cp2.append(b)
            cd.append(length)
        else:
            bp1.append(a)
            bp2.append(b)
            blen.append(length)
            bk.append(k)

    angles = []
    for b in range(n):
        for a, c in itertools.combinations(sorted(adj[b]), 2):
            for d in ff["angles"]:
                if _match(d["types"], (types[a], types[b], types[c])) or _match(d["types"], (types[c], types[b], types[a])):
                    angles.append((a, b, c, d["angle"], d["k"]))
                    break
            else:
                raise ValueError(f"no angle parameters for {types[a]}-{types[b]}-{types[c]}")

    torsions = []
    seen = set()
    for b, c in sorted(bonds):
        for a in sorted(adj[b] - {c}):
            for d in sorted(adj[c] - {b}):
                if a == d:
                    continue
                key = (a, b, c, d) if a < d else (d, c, b, a)
                if key in seen:
                    continue
                seen.add(key)
                best, best_wild = None, 99
                fwd = (types[a], types[b], types[c], types[d])
                rev = fwd[::-1]
                for defn in ff["propers"]:
                    if _match(defn["types"], fwd) or _match(defn["types"], rev):
                        wild = sum(1 for t in defn["types"] if t == "")
                        if wild < best_wild:
                            best, best_wild = defn, wild
                if best is None:
                    raise ValueError(f"no proper torsion for {fwd}")
                for per, phase, k in best["terms"]:
                    if k != 0.0:
                        torsions.append((key[0], key[1], key[2], key[3], per, phase, k))
    # impropers: definitions name the central atom first; AMBER order puts it third
    for c in range(n):
        if len(adj[c]) != 3:
            continue
        best, best_score, best_order = None, -1, None
        for defn in ff["impropers"]:
            t = defn["types"]
            if t[0] != "" and t[0] != types[c]:
                continue
            for perm in itertools.permutations(sorted(adj[c])):
                if all(t[k + 1] == "" or t[k + 1] == types[perm[k]] for k in range(3)):
                    score = sum(1 for k in range(4) if t[k] != "")
                    if score > best_score:
                        # wildcard slots take their atoms in ascending index order
                        wild = sorted(perm[k] for k in range(3) if t[k + 1] == "")
                        order = list(perm)
                        w = iter(wild)
                        for k in range(3):
                            if t[k + 1] == "":
                                order[k] = next(w)
                        best, best_score, best_order = defn, score, order
        if best is not None:
            a1, a2, a4 = best_order
            for per, phase, k in best["terms"]:
                if k != 0.0:
                    torsions.append((a1, a2, c, a4, per, phase, k))

    # exclusions and 1-4 exceptions from the bond graph (createExceptionsFromBonds)
    lj = ff["lj"]
    sigma = np.array([lj[t]["sigma"] for t in types])
    eps = np.array([lj[t]["epsilon"] for t in types])
    q = np.array(charges)
    near = set()
    for a in range(n):
        for b in adj[a]:
            near.add(tuple(sorted((a, b))))
            for c in adj[b]:
                if c != a:
                    near.add(tuple(sorted((a, c))))
    fourteen = set()
    for a, b, c, d, *_ in torsions:
        pass
    for b, c in bonds:
        for a in adj[b] - {c}:
            for d in adj[c] - {b}:
                if a != d:
                    pair = tuple(sorted((a, d)))
                    if pair not in near:
                        fourteen.add(pair)
    e1, e2, eq, es, ee = [], [], [], [], []
    for a, b in sorted(near):
        e1.append(a); e2.append(b); eq.append(0.0); es.append(1.0); ee.append(0.0)
    for a, b in sorted(fourteen):
        e1.append(a); e2.append(b)
        eq.append(q[a] * q[b] * ff["coulomb14scale"])
        es.append(0.5 * (sigma[a] + sigma[b]))
        ee.append(math.sqrt(eps[a] * eps[b]) * ff["lj14scale"])
    tor = list(zip(*torsions)) if torsions else [[]] * 7
    system = System(
        masses=masses, box=np.eye(3) * 10.0,
        constraint_p1=np.array(cp1, dtype=np.int32), constraint_p2=np.array(cp2, dtype=np.int32),
        constraint_distance=np.array(cd),
        nonbonded=Nonbonded(cutoff=cutoff, ewald_tolerance=ewald_tolerance, charge=q, sigma=sigma, epsilon=eps,
                            exception_p1=np.array(e1, dtype=np.int32), exception_p2=np.array(e2, dtype=np.int32),
                            exception_charge_prod=np.array(eq), exception_sigma=np.array(es),
                            exception_epsilon=np.array(ee)),
        bonds=(np.array(bp1, dtype=np.int32), np.array(bp2, dtype=np.int32), np.array(blen), np.array(bk)),
        angles=tuple(np.array(x, dtype=(np.int32 if i < 3 else np.float64)) for i, x in enumerate(zip(*angles))),
        torsions=tuple(np.array(x, dtype=(np.int32 if i < 5 else np.float64)) for i, x in enumerate(tor)),
    )
    positions = np.array([a[3] for a in atoms])
    return system, positions


def helix(sequence, phi=-57.0, psi=-47.0):
    return parameterise(build_chain(sequence, phi, psi))


# -------------------------------------------------------------- random coil --
# The 27k-atom workload's solute: a seeded 60-residue Ala-Gly-Lys-Glu chain
# whose backbone angles come from the extended basins (beta, polyproline II)
# and right-handed alpha turns, grown so that no two atoms of residues two or
# more apart clash and its bounding sphere fits a truncated octahedron of
# about 7.15 nm at OpenMM's 1.0 nm padding (src/prep/solvate.ts:390).
AGKE60 = ("ALA", "GLY", "LYS", "GLU") * 15
COIL_BASINS = np.array([[-120.0, 135.0], [-70.0, 145.0], [-63.0, -43.0]])
COIL_WEIGHTS = np.array([0.33, 0.22, 0.45])
COIL_DATA = Path(__file__).resolve().parent / "data" / "coil_angles.json"


def bounding_radius(xyz) -> float:
    """Radius of the sphere about the bounding box centre (solvate.ts:364)."""
    xyz = np.asarray(xyz)
    centre = 0.5 * (xyz.min(axis=0) + xyz.max(axis=0))
    return float(np.linalg.norm(xyz - centre, axis=1).max())


def _clashes(atoms, new_residue: int) -> bool:
    """Does any atom of `new_residue` come too close to an atom of a residue at
    least two before it (0.30 nm between heavy atoms, 0.20 nm otherwise)?"""
    xyz = np.array([a[3] for a in atoms])
    res = np.array([a[0] for a in atoms])
    heavy = np.array([not a[2].startswith("H") for a in atoms])
    new = res == new_residue
    old = res <= new_residue - 2
    if not old.any():
        return False
    d = np.linalg.norm(xyz[new][:, None] - xyz[old][None], axis=-1)
    limit = np.where(heavy[new][:, None] & heavy[old][None], 0.30, 0.20)
    return bool((d < limit).any())


def coil_angles(sequence, seed: int, min_radius: float = 2.95, max_radius: float = 3.1, confine: float = 3.0,
                tries: int = 24, budget: int = 20000):
    """Per-residue (phi, psi) of a clash-free coil, grown with backtracking.

    Residue k takes up to `tries` basin draws; a draw is kept when none of the
    residue's atoms clashes with residues two or more before it and all stay
    within `confine` nm of the first atom; when every draw fails the growth
    backs up two residues.  A finished chain whose bounding radius exceeds
    `max_radius` or falls short of `min_radius` (or whose caps clash) is
    regrown.  Deterministic for a seed.
    """
    rng = np.random.default_rng(seed)
    n = len(sequence)
    phi, psi = np.zeros(n), np.zeros(n)
    draws = 0
    while draws < budget:
        k = 0
        while k < n and draws < budget:
            placed = False
            for _ in range(tries):
                draws += 1
                phi[k], psi[k] = COIL_BASINS[rng.choice(3, p=COIL_WEIGHTS)] + rng.normal(0, 12, 2)
                atoms = [a for a in build_chain(sequence[:k + 1], phi[:k + 1], psi[:k + 1]) if a[0] <= k + 1]
                xyz = np.array([a[3] for a in atoms if a[0] == k + 1])
                if np.linalg.norm(xyz - atoms[0][3], axis=1).max() > confine or _clashes(atoms, k + 1):
                    continue
                placed = True
                break
            k = k + 1 if placed else max(0, k - 2)
        if k < n:
            break
        atoms = build_chain(sequence, phi, psi)
        xyz = np.array([a[3] for a in atoms])
        if min_radius <= bounding_radius(xyz) <= max_radius and not _clashes(atoms, n + 1):
            return phi.copy(), psi.copy()
    raise RuntimeError(f"no clash-free coil of radius {min_radius}-{max_radius} nm after {draws} draws")


def coil():
    """The parameterised AGKE60 coil with the angles data/make_coil.py found
    and stored in data/coil_angles.json (the seed is recorded there)."""
    table = json.loads(COIL_DATA.read_text())
    return parameterise(build_chain(tuple(table["sequence"]), np.array(table["phi"]), np.array(table["psi"])))
