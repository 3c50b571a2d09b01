"""Initial velocities as `Context.setVelocitiesToTemperature` sets them.

Mirrors src/reference/velocities.ts:78 `velocitiesAtTemperature`: a
Maxwell-Boltzmann draw per moving particle from the counter-based generator
on its own domain (Threefry-2x32-20, counter (2 i + axis / 2, seed), key
(seed, 0xbb67ae85), Box-Muller on open-interval uniforms, src/reference/
random.ts), shifted by -(offset / m) F -- the integrator's velocity time
offset, dt / 2 for the LFMiddle and Verlet integrators -- and projected onto
the constraints with the fixed tolerance 1e-5 that OpenMM uses here.

Host code, like the reference's; the forces come from the device.
"""

from __future__ import annotations

import numpy as np

from .system import System

BOLTZMANN_KJ_PER_MOL_K = 0.008314462618153242
VELOCITY_DOMAIN = 0xBB67AE85
# the projection tolerance setVelocitiesToTemperature uses, whatever the integrator's
VELOCITY_CONSTRAINT_TOLERANCE = 1e-5
_ROTATIONS = (13, 15, 26, 6, 17, 29, 16, 24)


def threefry2x32(c0, c1, k0, k1, rounds: int = 20):
    """Threefry-2x32 (Salmon et al., SC'11) on uint32 arrays: the two output words."""
    u = np.uint32
    c0 = np.asarray(c0, dtype=u)
    c1 = np.asarray(c1, dtype=u)
    ks = (u(k0), u(k1), u(0x1BD11BDA ^ int(k0) ^ int(k1)))
    with np.errstate(over="ignore"):
        x0 = c0 + ks[0]
        x1 = c1 + ks[1]
        for r in range(rounds):
            x0 = x0 + x1
            b = _ROTATIONS[r % 8]
            x1 = ((x1 << u(b)) | (x1 >> u(32 - b))) ^ x0
            if (r + 1) % 4 == 0:
                inj = (r + 1) // 4
                x0 = x0 + ks[inj % 3]
                x1 = x1 + ks[(inj + 1) % 3] + u(inj)
    return x0, x1


def open_unit(bits) -> np.ndarray:
    """A uniform in (0, 1) from the top 23 bits: ((b >> 9) + 0.5) 2^-23."""
    return ((np.asarray(bits, dtype=np.uint32) >> np.uint32(9)).astype(np.float64) + 0.5) * 2.0**-23


def domain_normals(domain: int, seed: int, count: int) -> np.ndarray:
    """Standard normals for particles 0..count-1, axes x, y, z: (count, 3)."""
    particle = np.arange(count, dtype=np.uint64)
    out = np.empty((count, 3))
    for pair in range(2):  # axes (0, 1) share a counter, axis 2 takes the next
        c0 = (particle * 2 + pair).astype(np.uint32)
        c1 = np.full(count, seed & 0xFFFFFFFF, dtype=np.uint32)
        b0, b1 = threefry2x32(c0, c1, seed & 0xFFFFFFFF, domain)
        radius = np.sqrt(-2.0 * np.log(open_unit(b0)))
        angle = 2.0 * np.pi * open_unit(b1)
        out[:, 2 * pair] = radius * np.cos(angle)
        if pair == 0:
            out[:, 1] = radius * np.sin(angle)
    return out


def constrain_velocities(system: System, positions: np.ndarray, velocities: np.ndarray, tolerance: float,
                         max_iterations: int = 10000) -> np.ndarray:
    """Remove the velocity along every constraint, mass-weighted, until the
    relative velocity along each bond is below `tolerance` (nm/ps per nm of
    bond); all constraints at once per sweep, each atom's correction shared
    among its constraints.  The projection is unique, so this meets the
    reference's SETTLE-v / RATTLE result to the tolerance."""
    v = np.array(velocities, dtype=np.float64).reshape(-1, 3)
    if system.constraint_count == 0:
        return v
    p = np.asarray(positions, dtype=np.float64).reshape(-1, 3)
    i, j = system.constraint_p1, system.constraint_p2
    m = np.asarray(system.masses, dtype=np.float64)
    inv = np.where(m > 0, 1.0 / np.where(m > 0, m, 1.0), 0.0)
    r = p[j] - p[i]
    r2 = np.einsum("ij,ij->i", r, r)
    share = np.bincount(np.concatenate([i, j]), minlength=v.shape[0]).astype(np.float64)
    w = inv[i] + inv[j]
    for _ in range(max_iterations):
        rv = np.einsum("ij,ij->i", r, v[j] - v[i])
        if np.max(np.abs(rv) / r2) <= tolerance:
            break
        lam = np.where(w > 0, rv / (np.where(w > 0, w, 1.0) * r2), 0.0)
        delta = np.zeros_like(v)
        np.add.at(delta, i, (lam * inv[i] / share[i])[:, None] * r)
        np.add.at(delta, j, -(lam * inv[j] / share[j])[:, None] * r)
        v += delta
    return v


def velocities_at_temperature(system: System, positions: np.ndarray, temperature: float, seed: int,
                              time_offset: float, forces: np.ndarray | None = None) -> np.ndarray:
    """`velocitiesAtTemperature` (src/reference/velocities.ts:78): (N, 3) nm/ps.
    A non-zero `time_offset` needs the forces at `positions` (kJ/mol/nm)."""
    if time_offset != 0 and forces is None:
        raise ValueError("a non-zero velocity time offset needs the forces at these positions: the draw is "
                         "shifted by -(offset/m) F; pass the forces, or time_offset=0")
    n = system.particle_count
    m = np.asarray(system.masses, dtype=np.float64)
    moving = m > 0
    kt = BOLTZMANN_KJ_PER_MOL_K * temperature
    v = np.zeros((n, 3))
    scale = np.sqrt(kt / np.where(moving, m, 1.0))
    v[moving] = (scale[:, None] * domain_normals(VELOCITY_DOMAIN, seed, n))[moving]
    if time_offset != 0:
        f = np.asarray(forces, dtype=np.float64).reshape(-1, 3)
        v[moving] -= (time_offset / m[moving])[:, None] * f[moving]
    return constrain_velocities(system, positions, v, VELOCITY_CONSTRAINT_TOLERANCE)


# the tolerance OpenMM re-constrains shifted velocities to (src/reference/kinetic.ts:28)
SHIFTED_VELOCITY_TOLERANCE = 1e-4


def kinetic_energy(system: System, velocities: np.ndarray) -> float:
    """(1/2) sum m v^2 over the moving particles (kinetic.ts:31), kJ/mol."""
    m = np.asarray(system.masses, dtype=np.float64)
    v = np.asarray(velocities, dtype=np.float64).reshape(-1, 3)
    moving = m > 0
    return 0.5 * float(np.sum(m[moving, None] * v[moving] * v[moving]))


def shifted_kinetic_energy(system: System, positions: np.ndarray, velocities: np.ndarray, forces: np.ndarray,
                           time_shift: float, tolerance: float = SHIFTED_VELOCITY_TOLERANCE) -> float:
    """`shiftedKineticEnergy` (kinetic.ts:87): the kinetic energy of the
    velocities advanced by `time_shift` (v + time_shift F / m) and projected
    back onto the constraints; a zero shift is the plain kinetic energy.  With
    time_shift = dt / 2 this is the kinetic energy a leapfrog integrator's
    conserved total needs, which `StepLoop.report` carries."""
    if time_shift == 0:
        return kinetic_energy(system, velocities)
    m = np.asarray(system.masses, dtype=np.float64)
    v = np.array(velocities, dtype=np.float64).reshape(-1, 3)
    f = np.asarray(forces, dtype=np.float64).reshape(-1, 3)
    moving = m > 0
    v[moving] += f[moving] * (time_shift / m[moving])[:, None]
    return kinetic_energy(system, constrain_velocities(system, positions, v, tolerance))
