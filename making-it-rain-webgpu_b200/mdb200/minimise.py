"""Local energy minimisation with the forces from the device.

Mirrors the reference's minimiser (src/reference/minimise.ts:164 `minimise`,
src/reference/lbfgs.ts:102 `lbfgs`, src/gpu/minimise.ts:33
`minimiseOnDevice`), which follows OpenMM's `ReferenceMinimize`: the search
runs on the host, every evaluation sets positions on the device and reads
back the energy and forces (`StepLoop.potential`, one `mdb_potential` call).

The objective is the potential plus the constraints turned into springs,
E(x) = U(x) + sum (k/2)(r - d)^2 with k = 100 / max(1e-4, constraint
tolerance); an outer loop multiplies k by ten until every constrained distance
is within max(1e-4, tolerance) of its target, and gives up -- returning the
starting configuration, as OpenMM does -- when stiffening stops helping.  The
search is L-BFGS with libLBFGS's backtracking strong-Wolfe line search and
its default parameters (memory 6, ftol 1e-4, wolfe 0.9, 40 trials, step
factors 0.5 / 2.1).  The tolerance is a root-mean-square force per particle
(kJ/mol/nm): OpenMM passes epsilon = tolerance / max(rms |x_i|, 1) to
libLBFGS's |g| / max(|x|, 1) test.

Positions on the device are 2^-32 nm fixed point, so a line search whose
trial step falls below that resolution sees no change and stops
("line-search-failed" or "step-too-small"): a property of the format, which
the reference documents the same way.
"""

from __future__ import annotations

import dataclasses
from typing import Callable, Optional

import numpy as np

from .system import System

# (energy, forces (N, 3)) at positions (N, 3)
Potential = Callable[[np.ndarray], tuple]
# value at x, gradient written into g
Objective = Callable[[np.ndarray, np.ndarray], float]


@dataclasses.dataclass
class LbfgsResult:
    value: float
    iterations: int
    evaluations: int
    status: str  # converged | max-iterations | line-search-failed | not-a-descent-direction | step-too-small | step-too-large
    gradient_ratio: float


def lbfgs(x: np.ndarray, objective: Objective, *, memory: int = 6, epsilon: float = 1e-5, max_iterations: int = 0,
          max_line_search: int = 40, ftol: float = 1e-4, wolfe: float = 0.9, min_step: float = 1e-20,
          max_step: float = 1e20) -> LbfgsResult:
    """Minimise `objective` from `x` (1-D float64, changed in place);
    src/reference/lbfgs.ts:102.  Stops when |g| / max(|x|, 1) <= epsilon, after
    `max_iterations` (0: no limit), or when the line search makes no progress,
    which is reported in `status` rather than raised."""
    n = x.size
    g = np.zeros(n)
    s = np.zeros((memory, n))
    y = np.zeros((memory, n))
    ys = np.zeros(memory)
    alpha = np.zeros(memory)
    evaluations = 1
    value = float(objective(x, g))

    def ratio() -> float:
        return float(np.linalg.norm(g) / max(np.linalg.norm(x), 1.0))

    if ratio() <= epsilon:
        return LbfgsResult(value, 0, evaluations, "converged", ratio())
    d = -g
    step = 1.0 / float(np.linalg.norm(d))  # the first step is scaled to the gradient
    end = stored = 0
    iteration = 0
    while True:
        iteration += 1
        x0, g0, f0 = x.copy(), g.copy(), value
        slope0 = float(g @ d)
        if slope0 > 0:
            return LbfgsResult(value, iteration - 1, evaluations, "not-a-descent-direction", ratio())
        outcome = "line-search-failed"
        for _ in range(max_line_search):
            x[:] = x0 + step * d
            value = float(objective(x, g))
            evaluations += 1
            if value > f0 + step * ftol * slope0:
                factor = 0.5
            else:
                slope = float(g @ d)
                if slope < wolfe * slope0:
                    factor = 2.1
                elif slope > -wolfe * slope0:
                    factor = 0.5  # strong Wolfe: the slope must also be small in magnitude
                else:
                    outcome = "ok"
                    break
            if step < min_step:
                outcome = "step-too-small"
                break
            if step > max_step:
                outcome = "step-too-large"
                break
            step *= factor
        if outcome != "ok":
            x[:] = x0
            g[:] = g0
            return LbfgsResult(f0, iteration - 1, evaluations, outcome, ratio())
        r = ratio()
        if r <= epsilon:
            return LbfgsResult(value, iteration, evaluations, "converged", r)
        if max_iterations and iteration >= max_iterations:
            return LbfgsResult(value, iteration, evaluations, "max-iterations", r)
        # newest correction pair, then the two-loop recursion d = -H g
        s[end] = x - x0
        y[end] = g - g0
        sy = float(y[end] @ s[end])
        yy = float(y[end] @ y[end])
        ys[end] = sy
        stored = min(stored + 1, memory)
        end = (end + 1) % memory
        d = -g.copy()
        j = end
        for _ in range(stored):
            j = (j - 1) % memory
            alpha[j] = float(s[j] @ d) / ys[j]
            d -= alpha[j] * y[j]
        d *= sy / yy
        for _ in range(stored):
            beta = float(y[j] @ d) / ys[j]
            d += (alpha[j] - beta) * s[j]
            j = (j + 1) % memory
        step = 1.0


def max_constraint_error(system: System, positions: np.ndarray) -> float:
    """The worst relative violation of a constrained distance
    (src/reference/minimise.ts `maxConstraintError`)."""
    if system.constraint_count == 0:
        return 0.0
    p = np.asarray(positions, dtype=np.float64).reshape(-1, 3)
    r = np.linalg.norm(p[system.constraint_p2] - p[system.constraint_p1], axis=1)
    return float(np.max(np.abs(r - system.constraint_distance) / system.constraint_distance))


def constrain_positions(system: System, positions: np.ndarray, tolerance: float,
                        max_iterations: int = 10000) -> np.ndarray:
    """Project `positions` (N, 3) onto the constraints to relative `tolerance`
    by mass-weighted SHAKE along the starting bond vectors, all constraints at
    once per sweep (Jacobi).  The reference projects with its SETTLE/SHAKE
    split (src/reference/constraints.ts); any projection that meets the
    tolerance serves the minimiser, whose answer is set by the objective."""
    x = np.array(positions, dtype=np.float64).reshape(-1, 3)
    if system.constraint_count == 0:
        return x
    i, j = system.constraint_p1, system.constraint_p2
    dist = system.constraint_distance
    m = np.asarray(system.masses, dtype=np.float64)
    inv = np.where(m > 0, 1.0 / np.where(m > 0, m, 1.0), 0.0)
    ref = x[j] - x[i]
    # atoms in several constraints take each correction in part, so the sweep converges
    share = np.bincount(np.concatenate([i, j]), minlength=x.shape[0]).astype(np.float64)
    for _ in range(max_iterations):
        cur = x[j] - x[i]
        r2 = np.einsum("ij,ij->i", cur, cur)
        diff = dist * dist - r2
        if np.max(np.abs(diff) / (2 * dist * dist)) <= tolerance:
            break
        proj = np.einsum("ij,ij->i", cur, ref)
        w = inv[i] + inv[j]
        ok = (proj != 0) & (w > 0)
        lam = np.where(ok, diff / (2 * np.where(ok, w * proj, 1.0)), 0.0)
        delta = np.zeros_like(x)
        np.add.at(delta, i, -(lam * inv[i] / share[i])[:, None] * ref)
        np.add.at(delta, j, (lam * inv[j] / share[j])[:, None] * ref)
        x += delta
    return x


def _springs(system: System, x: np.ndarray, grad: np.ndarray, k: float) -> float:
    """Spring energy k/2 (r - d)^2 of every constraint, its gradient added to
    `grad` (N, 3); frozen (massless) particles get no gradient."""
    if system.constraint_count == 0:
        return 0.0
    i, j = system.constraint_p1, system.constraint_p2
    delta = x[j] - x[i]
    r = np.linalg.norm(delta, axis=1)
    dr = r - system.constraint_distance
    unit = delta / r[:, None]
    mobile = np.asarray(system.masses) != 0
    contrib = (k * dr)[:, None] * unit
    np.add.at(grad, i, -contrib * mobile[i][:, None])
    np.add.at(grad, j, contrib * mobile[j][:, None])
    return float(0.5 * k * np.sum(dr * dr))


@dataclasses.dataclass
class MinimiseResult:
    positions: np.ndarray          # (N, 3) nm
    energy: float                  # kJ/mol, the potential alone
    restraint_energy: float        # kJ/mol, the constraint springs at the end
    max_constraint_error: float    # before the final projection
    restraint_strength: float
    initial_restraint_strength: float
    force_rms: float               # objective gradient, kJ/mol/nm per particle
    potential_force_rms: float     # potential forces only
    rounds: int
    iterations: int
    evaluations: int
    gave_up: bool
    status: str


def minimise(system: System, positions: np.ndarray, potential: Potential, *, tolerance: float = 10.0,
             max_iterations: int = 0, constraint_tolerance: float = 1e-6) -> MinimiseResult:
    """OpenMM's minimisation (src/reference/minimise.ts:164) with `potential`
    as the force field."""
    n = system.particle_count
    working = max(1e-4, constraint_tolerance)
    k = 100.0 / working
    k0 = k
    x = constrain_positions(system, positions, working).reshape(-1)
    initial = x.copy()
    mean_square = float(np.mean(np.sum(x.reshape(-1, 3) ** 2, axis=1)))
    epsilon = tolerance / (1.0 if mean_square < 1 else np.sqrt(mean_square))
    frozen = np.asarray(system.masses) == 0
    last = {"energy": 0.0, "restraint": 0.0, "grad": np.zeros(3 * n), "forces": np.zeros((n, 3))}

    def objective(xv: np.ndarray, gv: np.ndarray) -> float:
        p = xv.reshape(-1, 3)
        energy, forces = potential(p)
        forces = np.asarray(forces, dtype=np.float64).reshape(-1, 3)
        grad = -forces
        grad[frozen] = 0.0
        restraint = _springs(system, p, grad, k)
        gv[:] = grad.reshape(-1)
        last.update(energy=float(energy), restraint=restraint, grad=gv.copy(), forces=forces.copy())
        return float(energy) + restraint

    previous1 = previous2 = 1e10
    rounds = iterations = evaluations = 0
    gave_up = False
    status = "converged"
    error = 0.0
    while True:
        rounds += 1
        result = lbfgs(x, objective, epsilon=epsilon, max_iterations=max_iterations, memory=6)
        iterations += result.iterations
        evaluations += result.evaluations
        status = result.status
        error = max_constraint_error(system, x)
        if error <= working:
            break
        if error >= previous2:
            x[:] = initial  # OpenMM restores the start before it gives up
            gave_up = True
            break
        previous2, previous1 = previous1, error
        k *= 10.0
        if error > 100 * working:
            x[:] = initial
    out = x.reshape(-1, 3)
    if constraint_tolerance < working:
        out = constrain_positions(system, out, constraint_tolerance)

    def rms(v) -> float:
        return float(np.sqrt(np.sum(np.asarray(v) ** 2) / n))

    return MinimiseResult(positions=out, energy=last["energy"], restraint_energy=last["restraint"],
                          max_constraint_error=error, restraint_strength=k, initial_restraint_strength=k0,
                          force_rms=rms(last["grad"]), potential_force_rms=rms(last["forces"]), rounds=rounds,
                          iterations=iterations, evaluations=evaluations, gave_up=gave_up, status=status)
