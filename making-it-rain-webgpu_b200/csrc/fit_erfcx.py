"""Coefficients of the screened-Coulomb polynomial in k_nonbonded.cu.

The pair kernel needs erfc(x) and exp(-x^2) for x = alpha r in [0, alpha rc].
It evaluates exp(-x^2) once and writes erfc(x) = exp(-x^2) P(u), where P fits
the scaled complementary error function erfcx(x) = exp(x^2) erfc(x), a smooth
function that falls from 1 to 0.15 on [0, 3.6], as a polynomial in

    u = (2 t - (1 + t_min)) / (1 - t_min),   t = 1 / (1 + x/2),

so u runs over [-1, 1].  The fit is a relative-error-weighted least-squares
Chebyshev fit in f64 (numpy), converted to monomials in u for Horner
evaluation.  Degree 7 keeps the fit error below 5e-7 relative, under the f32
rounding of the pair arithmetic around it; the resulting direct-space force
error was measured against f64 at 6.0e-7 relative RMS versus 5.9e-7 with a
correctly rounded erfc (2,652-atom water box).

    python making-it-rain-webgpu_b200/csrc/fit_erfcx.py
"""

import numpy as np
from scipy.special import erfcx

X_MAX = 3.6  # alpha * cutoff ceiling; the host checks every system against it
DEGREE = 7


def main() -> None:
    x = np.linspace(0.0, X_MAX, 400001)
    t = 1.0 / (1.0 + 0.5 * x)
    t_min = 1.0 / (1.0 + 0.5 * X_MAX)
    u = (2 * t - (1 + t_min)) / (1 - t_min)
    y = erfcx(x)
    V = np.polynomial.chebyshev.chebvander(u, DEGREE)
    c, *_ = np.linalg.lstsq(V / y[:, None], np.ones_like(y), rcond=None)
    mono = np.polynomial.Chebyshev(c).convert(kind=np.polynomial.Polynomial).coef
    print(f"u = t * {2 / (1 - t_min)!r}f + {-(1 + t_min) / (1 - t_min)!r}f")
    print("coefficients, highest degree first:")
    for k in range(DEGREE, -1, -1):
        print(f"  {mono[k]!r}f")
    fit = np.polyval(mono[::-1], u)
    print("max relative error (f64):", float(np.max(np.abs(fit / y - 1))))


if __name__ == "__main__":
    main()
