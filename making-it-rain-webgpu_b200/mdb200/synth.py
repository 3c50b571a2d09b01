"""Seeded synthetic inputs with the shapes of the benchmark configurations.

The reference's realistic fixtures (1L2Y, 3HTB) are not committed and need
OpenMM plus network access to regenerate, so the workloads here are built by
this module: rigid TIP3P water boxes (cubic, rhombic dodecahedral, truncated
octahedral), optionally with ions, with the water model's published
parameters.  TIP3P as OpenMM's amber14 distributes it (vendor/ffxml/
amber14-tip3p.xml:71-72 masses, :247-249 charges, :255/:258 geometry,
:319-320 Lennard-Jones; Na+/Cl- Joung-Cheatham :263/:268).

Every builder is deterministic in its seed.
"""

from __future__ import annotations

import math

import numpy as np

from .system import Nonbonded, State, System

# TIP3P (Jorgensen et al. 1983) as in amber14-tip3p.xml
MASS_O, MASS_H = 15.99943, 1.007947
Q_O, Q_H = -0.834, 0.417
SIGMA_O, EPS_O = 0.31507524065751241, 0.635968
R_OH = 0.09572
THETA_HOH = 1.82421813418
D_HH = 2 * R_OH * math.sin(THETA_HOH / 2)
# Joung-Cheatham ions for TIP3P
NA = dict(mass=22.99, q=1.0, sigma=0.2439280690268249, eps=0.3658460312)
CL = dict(mass=35.45, q=-1.0, sigma=0.4477656957373345, eps=0.14891274399999999)

WATER_DENSITY_PER_NM3 = 33.42  # 0.997 g/cm^3 of H2O


def box_vectors(shape: str, width: float) -> np.ndarray:
    """`boxVectorsForShape`, src/reference/triclinic.ts:359."""
    if shape == "cube":
        return np.diag([width, width, width]).astype(np.float64)
    if shape == "dodecahedron":
        return np.array([[width, 0, 0], [0, width, 0], [width / 2, width / 2, width * math.sqrt(2) / 2]])
    if shape == "octahedron":
        return np.array([[width, 0, 0], [width / 3, width * 2 * math.sqrt(2) / 3, 0],
                         [-width / 3, width * math.sqrt(2) / 3, width * math.sqrt(6) / 3]])
    raise ValueError(f"unknown box shape {shape!r}")


def _water_template() -> np.ndarray:
    """O, H1, H2 relative to the molecule's centre of mass."""
    o = np.zeros(3)
    h1 = np.array([R_OH, 0.0, 0.0])
    h2 = np.array([R_OH * math.cos(THETA_HOH), R_OH * math.sin(THETA_HOH), 0.0])
    xyz = np.stack([o, h1, h2])
    com = (MASS_O * o + MASS_H * (h1 + h2)) / (MASS_O + 2 * MASS_H)
    return xyz - com


def _random_rotations(rng: np.random.Generator, n: int) -> np.ndarray:
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    return np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
        np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
        np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1),
    ], 1)


def _lattice_sites(box: np.ndarray, count: int, rng: np.random.Generator, exclude=None, min_gap=0.0):
    """`count` sites on a uniform fractional lattice of the cell, chosen at random."""
    volume = abs(np.linalg.det(box))
    per_axis = max(1, math.ceil(count ** (1 / 3)))
    inv = np.linalg.inv(box)
    for _ in range(64):
        g = (np.arange(per_axis) + 0.5) / per_axis
        frac = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
        jitter = rng.uniform(-0.05, 0.05, size=frac.shape) / per_axis
        cart = (frac + jitter) @ box
        if exclude is not None and len(exclude):
            keep = np.ones(len(cart), dtype=bool)
            for p in exclude:
                f = (cart - p) @ inv
                f -= np.round(f)
                keep &= np.linalg.norm(f @ box, axis=1) > min_gap
            cart = cart[keep]
        if len(cart) >= count:
            break
        per_axis += 1
    else:
        raise ValueError(f"no lattice leaves {count} free sites (volume {volume:.2f} nm^3)")
    pick = np.sort(rng.choice(len(cart), size=count, replace=False))
    return cart[pick]


def water_box(n_waters: int | None = None, width: float = 3.0, shape: str = "cube", seed: int = 1,
              n_na: int = 0, n_cl: int = 0, cutoff: float = 1.0, ewald_tolerance: float = 5e-4,
              grid=(0, 0, 0), temperature: float | None = 300.0, com_frequency: int = 1,
              barostat=None, solute=None) -> tuple[System, State]:
    """Rigid TIP3P (plus ions, plus an optional pre-built solute) in a periodic cell.

    `solute`, when given, is (System, positions): its atoms come first and the
    water sites keep 0.25 nm clear of them.
    """
    rng = np.random.default_rng(seed)
    box = box_vectors(shape, width)
    volume = abs(np.linalg.det(box))
    if n_waters is None:
        n_waters = int(round(WATER_DENSITY_PER_NM3 * volume))
    masses, charges, sigmas, epsilons, positions = [], [], [], [], []
    cp1, cp2, cd = [], [], []
    e1, e2, eq, es, ee = [], [], [], [], []
    bonds = angles = torsions = None
    base = 0
    solute_xyz = None
    if solute is not None:
        s_sys, s_pos = solute
        solute_xyz = np.asarray(s_pos, dtype=np.float64)
        nb = s_sys.nonbonded
        masses += list(s_sys.masses)
        charges += list(nb.charge)
        sigmas += list(nb.sigma)
        epsilons += list(nb.epsilon)
        positions += list(solute_xyz)
        cp1 += list(s_sys.constraint_p1)
        cp2 += list(s_sys.constraint_p2)
        cd += list(s_sys.constraint_distance)
        e1 += list(nb.exception_p1)
        e2 += list(nb.exception_p2)
        eq += list(nb.exception_charge_prod)
        es += list(nb.exception_sigma)
        ee += list(nb.exception_epsilon)
        bonds, angles, torsions = s_sys.bonds, s_sys.angles, s_sys.torsions
        base = s_sys.particle_count
    n_mol = n_waters + n_na + n_cl
    sites = _lattice_sites(box, n_mol, rng, exclude=solute_xyz, min_gap=0.3)
    order = rng.permutation(n_mol)
    ion_sites = sites[order[:n_na + n_cl]]
    water_sites = sites[np.sort(order[n_na + n_cl:])]
    tpl = _water_template()
    rot = _random_rotations(rng, n_waters)
    for k in range(n_waters):
        xyz = water_sites[k] + tpl @ rot[k].T
        o = base + 3 * k
        masses += [MASS_O, MASS_H, MASS_H]
        charges += [Q_O, Q_H, Q_H]
        sigmas += [SIGMA_O, 1.0, 1.0]
        epsilons += [EPS_O, 0.0, 0.0]
        positions += list(xyz)
        cp1 += [o, o, o + 1]
        cp2 += [o + 1, o + 2, o + 2]
        cd += [R_OH, R_OH, D_HH]
        e1 += [o, o, o + 1]
        e2 += [o + 1, o + 2, o + 2]
        eq += [0.0, 0.0, 0.0]
        es += [1.0, 1.0, 1.0]
        ee += [0.0, 0.0, 0.0]
    for k in range(n_na + n_cl):
        ion = NA if k < n_na else CL
        masses.append(ion["mass"])
        charges.append(ion["q"])
        sigmas.append(ion["sigma"])
        epsilons.append(ion["eps"])
        positions.append(ion_sites[k])
    n = len(masses)
    system = System(
        masses=np.array(masses),
        box=box,
        constraint_p1=np.array(cp1, dtype=np.int32),
        constraint_p2=np.array(cp2, dtype=np.int32),
        constraint_distance=np.array(cd),
        nonbonded=Nonbonded(
            cutoff=cutoff, ewald_tolerance=ewald_tolerance, grid=tuple(grid),
            charge=np.array(charges), sigma=np.array(sigmas), epsilon=np.array(epsilons),
            exception_p1=np.array(e1, dtype=np.int32), exception_p2=np.array(e2, dtype=np.int32),
            exception_charge_prod=np.array(eq), exception_sigma=np.array(es), exception_epsilon=np.array(ee),
            use_dispersion_correction=True,
        ),
        bonds=bonds, angles=angles, torsions=torsions,
        com_frequency=com_frequency,
        barostat=barostat,
    )
    pos = np.array(positions, dtype=np.float64).reshape(n, 3)
    velocities = None
    if temperature is not None:
        velocities = maxwell_boltzmann(system, temperature, rng)
    return system, State(positions=pos, box=box.copy(), velocities=velocities)


def maxwell_boltzmann(system: System, temperature: float, rng: np.random.Generator) -> np.ndarray:
    """Thermal velocities, sqrt(kT/m) N(0,1) per component; zero for frozen atoms.

    Not projected onto the constraints: the LFMiddle step RATTLEs/SETTLEs the
    velocities right after its first kick.
    """
    kt = 0.008314462618153242 * temperature
    m = np.asarray(system.masses)
    scale = np.where(m > 0, np.sqrt(kt / np.where(m > 0, m, 1.0)), 0.0)
    v = rng.normal(size=(len(m), 3)) * scale[:, None]
    total = m.sum()
    if total > 0:
        v -= (m[:, None] * v).sum(0) / total
    return v


def config_water_2652(seed: int = 1):
    """2,652-atom cubic 3.0 nm TIP3P box, 884 waters, mesh pinned 30^3 (0.1 nm)."""
    return water_box(n_waters=884, width=3.0, seed=seed, grid=(30, 30, 30))


def config_water_cube(width: float, seed: int = 1, grid=(0, 0, 0), **kw):
    return water_box(width=width, seed=seed, grid=grid, **kw)


def ions_for(volume_nm3: float, molar: float = 0.15) -> int:
    """Ion pairs for a salt concentration: c * V * N_A, rounded."""
    return int(round(molar * volume_nm3 * 1e-24 * 6.02214076e23))


def solvated(solute_system: System, solute_positions, width: float, shape: str = "cube", seed: int = 1,
             grid=(0, 0, 0), molar: float = 0.15, **kw):
    """A solute centred in a TIP3P cell with NaCl at `molar`, neutralised."""
    from .system import Nonbonded  # noqa: F401  (kept for symmetry with water_box)

    box = box_vectors(shape, width)
    centre = 0.5 * box.sum(axis=0)
    pos = np.asarray(solute_positions, dtype=np.float64)
    pos = pos - pos.mean(axis=0) + centre
    volume = abs(np.linalg.det(box))
    pairs = ions_for(volume, molar)
    net = float(np.round(solute_system.nonbonded.charge.sum()))
    n_na = pairs + max(0, int(-net))
    n_cl = pairs + max(0, int(net))
    solute_volume = 0.02 * solute_system.particle_count
    n_waters = int(round(WATER_DENSITY_PER_NM3 * (volume - solute_volume))) - (n_na + n_cl)
    return water_box(n_waters=n_waters, width=width, shape=shape, seed=seed, n_na=n_na, n_cl=n_cl, grid=grid,
                     solute=(solute_system, pos), **kw)


def config_peptide_12k(seed: int = 1):
    """Ala20 alpha-helix (phi -57, psi -47) with ACE/NME caps, ff14SB, HBond
    constraints, in a 5.0 nm TIP3P cube with 0.15 M NaCl; mesh 50^3 (0.1 nm)."""
    from . import peptide

    solute, positions = peptide.helix(["ALA"] * 20)
    return solvated(solute, positions, width=5.0, seed=seed, grid=(50, 50, 50))


def config_octahedron_27k(seed: int = 1):
    """60-residue (Ala-Gly-Lys-Glu)15 coil with ACE/NME caps, ff14SB, HBond
    constraints, in a TIP3P truncated octahedron sized by OpenMM's padding
    rule at 1.0 nm (src/prep/solvate.ts:390: width = 2 R + padding, R the
    bounding-sphere radius), 0.15 M NaCl; mesh by the reference's rule from
    the box diagonal.  About 27,000 atoms."""
    from . import peptide

    solute, positions = peptide.coil()
    width = max(2.0 * peptide.bounding_radius(positions) + 1.0, 2.0)
    return solvated(solute, positions, width=width, shape="octahedron", seed=seed)


def _perpendicular_min(box: np.ndarray) -> float:
    a, b, c = box
    v = abs(np.linalg.det(box))
    return float(min(v / np.linalg.norm(np.cross(b, c)), v / np.linalg.norm(np.cross(c, a)),
                     v / np.linalg.norm(np.cross(a, b))))


def ensemble_member(rng: np.random.Generator, seed: int, cutoff: float = 1.0, barostat=None):
    """One system of the batched ensemble: a target atom count drawn
    log-uniformly from 2,000 to 30,000, a cubic or rhombic-dodecahedral cell of
    TIP3P sized to it, and, half the time, an Ala helix of 10-40 residues when
    one fits the cell at OpenMM's 1.0 nm padding (otherwise the longest that
    fits, or none).  Returns (system, state, description)."""
    from . import peptide

    target = math.exp(rng.uniform(math.log(2000), math.log(30000)))
    shape = "cube" if rng.random() < 0.5 else "dodecahedron"
    volume = target / (3 * WATER_DENSITY_PER_NM3)
    unit = abs(np.linalg.det(box_vectors(shape, 1.0)))
    width = (volume / unit) ** (1 / 3)
    # the cutoff must stay below half the narrowest perpendicular width
    width = max(width, 2.02 * cutoff / _perpendicular_min(box_vectors(shape, 1.0)))
    residues = int(rng.integers(10, 41)) if rng.random() < 0.5 else 0
    room = _perpendicular_min(box_vectors(shape, width))
    while residues >= 10:
        solute, x = peptide.helix(["ALA"] * residues)
        if 2 * peptide.bounding_radius(x) + 1.0 <= room:
            break
        residues -= 5
    if residues < 10:
        residues = 0
    if residues:
        system, state = solvated(solute, x, width=width, shape=shape, seed=seed, barostat=barostat)
    else:
        system, state = water_box(width=width, shape=shape, seed=seed, barostat=barostat)
    return system, state, {"shape": shape, "width": width, "helix_residues": residues,
                           "atoms": system.particle_count}


def config_ensemble_64(seed: int = 1, count: int = 64, barostat=None):
    """The batched ensemble: `count` independent systems of uneven sizes."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        out.append(ensemble_member(rng, seed=seed * 1000 + k, barostat=barostat))
    return out


def config_npt_ensemble_64(seed: int = 1, count: int = 64, frequency: int = 25):
    """The batched ensemble under NPT: the same 64 systems, each with a Monte
    Carlo barostat at 1 bar and 300 K, a volume move every 25 steps."""
    return config_ensemble_64(seed=seed, count=count, barostat=(1.0, 300.0, frequency))


def config_npt_100k(seed: int = 1, width: float = 10.0, frequency: int = 25):
    """NPT: a cubic 10 nm TIP3P box (about 100,000 atoms) at 300 K and 1 bar,
    Monte Carlo volume moves every 25 steps; mesh by the reference's rule."""
    return water_box(width=width, seed=seed, barostat=(1.0, 300.0, frequency))
