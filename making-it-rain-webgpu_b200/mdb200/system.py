"""OpenMM System and State, as flat arrays, with their XML form.

The input contract of the step engine: mirrors `OpenMMSystem`, the force
interfaces, `parseSystem` and `parseState` of src/engine/system.ts:41-620 and
src/engine/state.ts:60-235 (paths relative to the reference project root),
including the refusals by name (`UnsupportedForce`, system.ts:178).

`System.desc()` builds the `mdb_system_desc` the C ABI takes; the arrays it
points into are kept alive by the returned object.
"""

from __future__ import annotations

import ctypes as C
import dataclasses
import xml.etree.ElementTree as ET
from typing import Optional

import numpy as np

from . import abi

# NonbondedMethod values (system.ts: OpenMM's enum); only PME runs here.
NO_CUTOFF, CUTOFF_NON_PERIODIC, CUTOFF_PERIODIC, EWALD, PME, LJPME = range(6)

RESTRAINT_EXPRESSION = "k*periodicdistance(x,y,z,x0,y0,z0)^2"


class UnsupportedForce(ValueError):
    """A force this engine does not implement (system.ts:178)."""

    def __init__(self, force_type: str, detail: str | None = None):
        message = f"{force_type} is not implemented by this engine"
        if detail:
            message += f": {detail}"
        message += (
            ". The supported set is HarmonicBondForce, HarmonicAngleForce, "
            "PeriodicTorsionForce, NonbondedForce (PME), CMMotionRemover, "
            "MonteCarloBarostat, and a CustomExternalForce holding exactly "
            f'"{RESTRAINT_EXPRESSION}".'
        )
        super().__init__(message)
        self.force_type = force_type


def _f64(values) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(values, dtype=np.float64))


def _i32(values) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(values, dtype=np.int32))


@dataclasses.dataclass
class Nonbonded:
    cutoff: float
    ewald_tolerance: float
    charge: np.ndarray
    sigma: np.ndarray
    epsilon: np.ndarray
    exception_p1: np.ndarray
    exception_p2: np.ndarray
    exception_charge_prod: np.ndarray
    exception_sigma: np.ndarray
    exception_epsilon: np.ndarray
    alpha: float = 0.0
    grid: tuple = (0, 0, 0)
    use_dispersion_correction: bool = True
    method: int = PME


@dataclasses.dataclass
class System:
    """An OpenMM System (system.ts:161)."""

    masses: np.ndarray
    box: np.ndarray  # (3, 3) rows a, b, c
    constraint_p1: np.ndarray = dataclasses.field(default_factory=lambda: _i32([]))
    constraint_p2: np.ndarray = dataclasses.field(default_factory=lambda: _i32([]))
    constraint_distance: np.ndarray = dataclasses.field(default_factory=lambda: _f64([]))
    nonbonded: Optional[Nonbonded] = None
    bonds: Optional[tuple] = None  # (p1, p2, length, k)
    angles: Optional[tuple] = None  # (p1, p2, p3, theta, k)
    torsions: Optional[tuple] = None  # (p1, p2, p3, p4, periodicity, phase, k)
    com_frequency: int = 0
    barostat: Optional[tuple] = None  # (pressure bar, temperature K, frequency)
    restraints: Optional[tuple] = None  # (particle, k, x0, y0, z0)

    @property
    def particle_count(self) -> int:
        return int(self.masses.shape[0])

    @property
    def constraint_count(self) -> int:
        return int(self.constraint_p1.shape[0])

    def desc(self) -> "SystemDescHandle":
        return SystemDescHandle(self)


class SystemDescHandle:
    """An `mdb_system_desc` plus the arrays it points into."""

    def __init__(self, system: System):
        keep = []

        def dp(a):
            a = _f64(a)
            keep.append(a)
            return a.ctypes.data_as(C.POINTER(C.c_double))

        def ip(a):
            a = _i32(a)
            keep.append(a)
            return a.ctypes.data_as(C.POINTER(C.c_int32))

        d = abi.SystemDesc()
        n = system.particle_count
        d.n_particles = n
        d.masses = dp(system.masses)
        d.box[:] = [float(v) for v in np.asarray(system.box, dtype=np.float64).reshape(9)]
        d.n_constraints = system.constraint_count
        d.constraint_p1 = ip(system.constraint_p1)
        d.constraint_p2 = ip(system.constraint_p2)
        d.constraint_distance = dp(system.constraint_distance)
        nb = system.nonbonded
        if nb is not None:
            d.has_nonbonded = 1
            d.cutoff = nb.cutoff
            d.ewald_tolerance = nb.ewald_tolerance
            d.alpha = nb.alpha
            d.grid[:] = [int(g) for g in nb.grid]
            d.use_dispersion_correction = int(bool(nb.use_dispersion_correction))
            d.charge = dp(nb.charge)
            d.sigma = dp(nb.sigma)
            d.epsilon = dp(nb.epsilon)
            d.n_exceptions = int(len(nb.exception_p1))
            d.exception_p1 = ip(nb.exception_p1)
            d.exception_p2 = ip(nb.exception_p2)
            d.exception_charge_prod = dp(nb.exception_charge_prod)
            d.exception_sigma = dp(nb.exception_sigma)
            d.exception_epsilon = dp(nb.exception_epsilon)
        if system.bonds is not None:
            p1, p2, length, k = system.bonds
            d.n_bonds = len(p1)
            d.bond_p1, d.bond_p2 = ip(p1), ip(p2)
            d.bond_length, d.bond_k = dp(length), dp(k)
        if system.angles is not None:
            p1, p2, p3, theta, k = system.angles
            d.n_angles = len(p1)
            d.angle_p1, d.angle_p2, d.angle_p3 = ip(p1), ip(p2), ip(p3)
            d.angle_theta, d.angle_k = dp(theta), dp(k)
        if system.torsions is not None:
            p1, p2, p3, p4, per, phase, k = system.torsions
            d.n_torsions = len(p1)
            d.torsion_p1, d.torsion_p2, d.torsion_p3, d.torsion_p4 = ip(p1), ip(p2), ip(p3), ip(p4)
            d.torsion_periodicity = ip(per)
            d.torsion_phase, d.torsion_k = dp(phase), dp(k)
        d.com_frequency = int(system.com_frequency)
        if system.barostat is not None:
            pressure, temperature, frequency = system.barostat
            d.barostat_pressure = float(pressure)
            d.barostat_temperature = float(temperature)
            d.barostat_frequency = int(frequency)
        if system.restraints is not None:
            particle, k, x0, y0, z0 = system.restraints
            d.n_restraints = len(particle)
            d.restraint_particle = ip(particle)
            d.restraint_k, d.restraint_x0 = dp(k), dp(x0)
            d.restraint_y0, d.restraint_z0 = dp(y0), dp(z0)
        self.desc = d
        self._keep = keep
        self.system = system

    def pointer(self):
        return C.pointer(self.desc)


@dataclasses.dataclass
class State:
    """An OpenMM State (state.ts:18): positions, velocities, box, step."""

    positions: np.ndarray  # (N, 3) nm
    box: np.ndarray  # (3, 3)
    velocities: Optional[np.ndarray] = None  # (N, 3) nm/ps
    step: int = 0
    time: float = 0.0

    def desc(self) -> "StateDescHandle":
        return StateDescHandle(self)


class StateDescHandle:
    def __init__(self, state: State):
        self.positions = _f64(state.positions).reshape(-1)
        self.velocities = None if state.velocities is None else _f64(state.velocities).reshape(-1)
        d = abi.StateDesc()
        d.positions = self.positions.ctypes.data_as(C.POINTER(C.c_double))
        d.velocities = (
            self.velocities.ctypes.data_as(C.POINTER(C.c_double))
            if self.velocities is not None
            else C.POINTER(C.c_double)()
        )
        d.box[:] = [float(v) for v in np.asarray(state.box, dtype=np.float64).reshape(9)]
        d.step = int(state.step)
        self.desc = d

    def pointer(self):
        return C.pointer(self.desc)


# ------------------------------------------------------------------ XML ----


def _box_from(element) -> np.ndarray:
    box = element.find("PeriodicBoxVectors")
    if box is None:
        raise ValueError("expected <PeriodicBoxVectors>")
    rows = []
    for tag in ("A", "B", "C"):
        v = box.find(tag)
        if v is None:
            raise ValueError(f"expected three box vectors, missing <{tag}>")
        rows.append([float(v.get("x")), float(v.get("y")), float(v.get("z"))])
    return np.array(rows, dtype=np.float64)


def _flag(element, name: str, default: bool = False) -> bool:
    value = element.get(name)
    if value is None:
        return default
    return value.strip() not in ("0", "false", "False")


def parse_system(text: str) -> System:
    """`parseSystem`, src/engine/system.ts:521."""
    root = ET.fromstring(text)
    if root.tag != "System":
        raise ValueError(f"expected <System>, found <{root.tag}>")
    box = _box_from(root)
    masses = _f64([float(p.get("mass")) for p in root.find("Particles").findall("Particle")])
    p1, p2, dist = [], [], []
    constraints = root.find("Constraints")
    if constraints is not None:
        for c in constraints.findall("Constraint"):
            p1.append(int(c.get("p1")))
            p2.append(int(c.get("p2")))
            dist.append(float(c.get("d")))
    system = System(masses=masses, box=box, constraint_p1=_i32(p1), constraint_p2=_i32(p2),
                    constraint_distance=_f64(dist))
    forces = root.find("Forces")
    for force in [] if forces is None else forces.findall("Force"):
        kind = force.get("type")
        if kind == "HarmonicBondForce":
            rows = force.find("Bonds").findall("Bond") if force.find("Bonds") is not None else []
            system.bonds = (
                _i32([int(b.get("p1")) for b in rows]), _i32([int(b.get("p2")) for b in rows]),
                _f64([float(b.get("d")) for b in rows]), _f64([float(b.get("k")) for b in rows]))
            if _flag(force, "usesPeriodic"):
                raise UnsupportedForce(kind, "usesPeriodic bonded terms are not produced by this workflow")
        elif kind == "HarmonicAngleForce":
            rows = force.find("Angles").findall("Angle") if force.find("Angles") is not None else []
            system.angles = (
                _i32([int(a.get("p1")) for a in rows]), _i32([int(a.get("p2")) for a in rows]),
                _i32([int(a.get("p3")) for a in rows]), _f64([float(a.get("a")) for a in rows]),
                _f64([float(a.get("k")) for a in rows]))
            if _flag(force, "usesPeriodic"):
                raise UnsupportedForce(kind, "usesPeriodic bonded terms are not produced by this workflow")
        elif kind == "PeriodicTorsionForce":
            rows = force.find("Torsions").findall("Torsion") if force.find("Torsions") is not None else []
            system.torsions = (
                _i32([int(t.get("p1")) for t in rows]), _i32([int(t.get("p2")) for t in rows]),
                _i32([int(t.get("p3")) for t in rows]), _i32([int(t.get("p4")) for t in rows]),
                _i32([int(t.get("periodicity")) for t in rows]),
                _f64([float(t.get("phase")) for t in rows]), _f64([float(t.get("k")) for t in rows]))
            if _flag(force, "usesPeriodic"):
                raise UnsupportedForce(kind, "usesPeriodic bonded terms are not produced by this workflow")
        elif kind == "NonbondedForce":
            method = int(force.get("method", "4"))
            if method == LJPME:
                raise UnsupportedForce(kind, "LJ-PME is not implemented")
            if method != PME:
                raise UnsupportedForce(kind, f"nonbonded method {method}; this engine runs PME (4) only")
            offsets = 0
            for tag in ("ParticleOffsets", "ExceptionOffsets"):
                block = force.find(tag)
                if block is not None:
                    offsets += len(list(block))
            if offsets:
                raise UnsupportedForce(kind, f"it carries {offsets} parameter offset(s)")
            if _flag(force, "useSwitchingFunction"):
                raise UnsupportedForce(kind, "a switching function is not implemented")
            parts = force.find("Particles").findall("Particle")
            excs = force.find("Exceptions").findall("Exception") if force.find("Exceptions") is not None else []
            system.nonbonded = Nonbonded(
                cutoff=float(force.get("cutoff")),
                ewald_tolerance=float(force.get("ewaldTolerance")),
                alpha=float(force.get("alpha", "0")),
                grid=(int(force.get("nx", "0")), int(force.get("ny", "0")), int(force.get("nz", "0"))),
                use_dispersion_correction=_flag(force, "dispersionCorrection"),
                charge=_f64([float(p.get("q")) for p in parts]),
                sigma=_f64([float(p.get("sig")) for p in parts]),
                epsilon=_f64([float(p.get("eps")) for p in parts]),
                exception_p1=_i32([int(e.get("p1")) for e in excs]),
                exception_p2=_i32([int(e.get("p2")) for e in excs]),
                exception_charge_prod=_f64([float(e.get("q")) for e in excs]),
                exception_sigma=_f64([float(e.get("sig")) for e in excs]),
                exception_epsilon=_f64([float(e.get("eps")) for e in excs]),
            )
        elif kind == "CMMotionRemover":
            system.com_frequency = int(float(force.get("frequency", "1")))
        elif kind == "MonteCarloBarostat":
            system.barostat = (float(force.get("pressure")), float(force.get("temperature")),
                               int(force.get("frequency", "25")))
        elif kind == "CustomExternalForce":
            expression = (force.get("energy") or "").replace(" ", "").replace(";", "")
            if expression != RESTRAINT_EXPRESSION:
                raise UnsupportedForce(kind, f'its energy expression is "{force.get("energy")}"')
            names = [p.get("name") for p in force.find("PerParticleParameters").findall("Parameter")]
            rows = force.find("Particles").findall("Particle")
            col = {name: i for i, name in enumerate(names)}
            for want in ("k", "x0", "y0", "z0"):
                if want not in col:
                    raise UnsupportedForce(kind, f'it has no per-particle parameter "{want}"')
            vals = [[float(r.get(f"param{i + 1}")) for i in range(len(names))] for r in rows]
            particle = _i32([int(r.get("index")) for r in rows])
            arr = np.array(vals, dtype=np.float64).reshape(len(rows), len(names))
            system.restraints = (particle, arr[:, col["k"]].copy(), arr[:, col["x0"]].copy(),
                                 arr[:, col["y0"]].copy(), arr[:, col["z0"]].copy())
        else:
            raise UnsupportedForce(kind or "(untyped force)")
    return system


def parse_state(text: str) -> State:
    """`parseState`, src/engine/state.ts:60."""
    root = ET.fromstring(text)
    if root.tag != "State":
        raise ValueError(f"expected <State>, found <{root.tag}>")
    box = _box_from(root)
    pos = np.array([[float(p.get("x")), float(p.get("y")), float(p.get("z"))]
                    for p in root.find("Positions").findall("Position")], dtype=np.float64)
    vel = None
    vnode = root.find("Velocities")
    if vnode is not None:
        vel = np.array([[float(v.get("x")), float(v.get("y")), float(v.get("z"))]
                        for v in vnode.findall("Velocity")], dtype=np.float64)
    return State(positions=pos, box=box, velocities=vel, step=int(root.get("stepCount", "0")),
                 time=float(root.get("time", "0")))


def _fmt(v: float) -> str:
    return repr(float(v))


def serialise_state(state: State) -> str:
    """`serialiseState`, src/engine/state.ts:203: a checkpoint an OpenMM reader accepts."""
    lines = ['<?xml version="1.0" ?>',
             f'<State openmmVersion="8.4" stepCount="{int(state.step)}" time="{_fmt(state.time)}" '
             'type="State" version="1">', "\t<PeriodicBoxVectors>"]
    for tag, row in zip("ABC", np.asarray(state.box).reshape(3, 3)):
        lines.append(f'\t\t<{tag} x="{_fmt(row[0])}" y="{_fmt(row[1])}" z="{_fmt(row[2])}"/>')
    lines.append("\t</PeriodicBoxVectors>")
    lines.append("\t<Positions>")
    for p in np.asarray(state.positions).reshape(-1, 3):
        lines.append(f'\t\t<Position x="{_fmt(p[0])}" y="{_fmt(p[1])}" z="{_fmt(p[2])}"/>')
    lines.append("\t</Positions>")
    if state.velocities is not None:
        lines.append("\t<Velocities>")
        for v in np.asarray(state.velocities).reshape(-1, 3):
            lines.append(f'\t\t<Velocity x="{_fmt(v[0])}" y="{_fmt(v[1])}" z="{_fmt(v[2])}"/>')
        lines.append("\t</Velocities>")
    lines.append("</State>")
    return "\n".join(lines) + "\n"


def serialise_system(system: System) -> str:
    """`serialiseSystem`, src/engine/system.ts:619: the XML `parse_system` reads back."""
    out = ['<?xml version="1.0" ?>', '<System openmmVersion="8.4" type="System" version="1">',
           "\t<PeriodicBoxVectors>"]
    for tag, row in zip("ABC", np.asarray(system.box).reshape(3, 3)):
        out.append(f'\t\t<{tag} x="{_fmt(row[0])}" y="{_fmt(row[1])}" z="{_fmt(row[2])}"/>')
    out.append("\t</PeriodicBoxVectors>")
    out.append("\t<Particles>")
    out += [f'\t\t<Particle mass="{_fmt(m)}"/>' for m in system.masses]
    out.append("\t</Particles>")
    out.append("\t<Constraints>")
    out += [f'\t\t<Constraint d="{_fmt(d)}" p1="{a}" p2="{b}"/>'
            for a, b, d in zip(system.constraint_p1, system.constraint_p2, system.constraint_distance)]
    out.append("\t</Constraints>")
    out.append("\t<Forces>")
    if system.bonds is not None:
        out.append('\t\t<Force type="HarmonicBondForce" usesPeriodic="0" version="2"><Bonds>')
        out += [f'\t\t\t<Bond d="{_fmt(d)}" k="{_fmt(k)}" p1="{a}" p2="{b}"/>' for a, b, d, k in zip(*system.bonds)]
        out.append("\t\t</Bonds></Force>")
    if system.angles is not None:
        out.append('\t\t<Force type="HarmonicAngleForce" usesPeriodic="0" version="2"><Angles>')
        out += [f'\t\t\t<Angle a="{_fmt(t)}" k="{_fmt(k)}" p1="{a}" p2="{b}" p3="{c}"/>'
                for a, b, c, t, k in zip(*system.angles)]
        out.append("\t\t</Angles></Force>")
    if system.torsions is not None:
        out.append('\t\t<Force type="PeriodicTorsionForce" usesPeriodic="0" version="2"><Torsions>')
        out += [f'\t\t\t<Torsion k="{_fmt(k)}" p1="{a}" p2="{b}" p3="{c}" p4="{d}" periodicity="{n}" '
                f'phase="{_fmt(ph)}"/>' for a, b, c, d, n, ph, k in zip(*system.torsions)]
        out.append("\t\t</Torsions></Force>")
    nb = system.nonbonded
    if nb is not None:
        out.append(f'\t\t<Force type="NonbondedForce" method="{PME}" cutoff="{_fmt(nb.cutoff)}" '
                   f'ewaldTolerance="{_fmt(nb.ewald_tolerance)}" alpha="{_fmt(nb.alpha)}" '
                   f'nx="{nb.grid[0]}" ny="{nb.grid[1]}" nz="{nb.grid[2]}" '
                   f'dispersionCorrection="{int(bool(nb.use_dispersion_correction))}" '
                   'useSwitchingFunction="0" version="4">')
        out.append("\t\t\t<Particles>")
        out += [f'\t\t\t\t<Particle eps="{_fmt(e)}" q="{_fmt(q)}" sig="{_fmt(s)}"/>'
                for q, s, e in zip(nb.charge, nb.sigma, nb.epsilon)]
        out.append("\t\t\t</Particles>")
        out.append("\t\t\t<Exceptions>")
        out += [f'\t\t\t\t<Exception eps="{_fmt(e)}" p1="{a}" p2="{b}" q="{_fmt(q)}" sig="{_fmt(s)}"/>'
                for a, b, q, s, e in zip(nb.exception_p1, nb.exception_p2, nb.exception_charge_prod,
                                         nb.exception_sigma, nb.exception_epsilon)]
        out.append("\t\t\t</Exceptions>")
        out.append("\t\t</Force>")
    if system.com_frequency:
        out.append(f'\t\t<Force type="CMMotionRemover" frequency="{int(system.com_frequency)}" version="1"/>')
    if system.barostat is not None:
        p, t, f = system.barostat
        out.append(f'\t\t<Force type="MonteCarloBarostat" pressure="{_fmt(p)}" temperature="{_fmt(t)}" '
                   f'frequency="{int(f)}" version="2"/>')
    out.append("\t</Forces>")
    out.append("</System>")
    return "\n".join(out) + "\n"
