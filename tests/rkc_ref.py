"""CPU restatement of the RKC2 base step (test infrastructure): the damped
second-order Runge-Kutta-Chebyshev method (Sommeijer, Shampine & Verwer
1998), eps = 2/13, coefficients by the Chebyshev three-term recurrences, the
stage right-hand side from the oracle's Cahn-Hilliard RHS, and every stage
combination rounded in the library's order, so FP64 results are comparable
bit for bit."""
import numpy as np


def coeffs(s: int) -> dict:
    eps = 2.0 / 13.0
    w0 = 1.0 + eps / (float(s) * s)
    T, d1, d2 = [1.0, w0], [0.0, 1.0], [0.0, 0.0]
    for j in range(2, s + 1):
        T.append(2.0 * w0 * T[j - 1] - T[j - 2])
        d1.append(2.0 * T[j - 1] + 2.0 * w0 * d1[j - 1] - d1[j - 2])
        d2.append(4.0 * d1[j - 1] + 2.0 * w0 * d2[j - 1] - d2[j - 2])
    w1 = d1[s] / d2[s]
    b = [0.0] * (s + 1)
    for j in range(2, s + 1):
        b[j] = d2[j] / (d1[j] * d1[j])
    b[0] = b[1] = b[2]
    a = [1.0 - b[j] * T[j] for j in range(s + 1)]
    out = {"s": s, "mt1": b[1] * w1, "mu": {}, "nu": {}, "mt": {}, "gt": {},
           "beta": (w0 + 1.0) * d2[s] / d1[s]}
    for j in range(2, s + 1):
        out["mu"][j] = 2.0 * b[j] * w0 / b[j - 1]
        out["nu"][j] = -b[j] / b[j - 2]
        out["mt"][j] = 2.0 * b[j] * w1 / b[j - 1]
        out["gt"][j] = -a[j - 1] * out["mt"][j]
    return out


def stability_polynomial(s: int, z: complex) -> complex:
    """R(z) of one step on y' = lambda y, z = lambda dt."""
    c = coeffs(s)
    y0 = 1.0
    f0 = z * y0
    ym2, ym1 = y0, y0 + c["mt1"] * f0
    for j in range(2, s + 1):
        yj = ((1.0 - c["mu"][j] - c["nu"][j]) * y0 + c["mu"][j] * ym1 + c["nu"][j] * ym2
              + c["mt"][j] * z * ym1 + c["gt"][j] * f0)
        ym2, ym1 = ym1, yj
    return ym1


def step(rhs, psi: np.ndarray, dt: float, s: int) -> np.ndarray:
    """One RKC2 step; rhs(y) -> f(y) (float64 arrays)."""
    c = coeffs(s)
    y0 = psi
    f0 = rhs(y0)
    ym2, ym1 = y0, y0 + (c["mt1"] * dt) * f0
    for j in range(2, s + 1):
        r = (1.0 - c["mu"][j] - c["nu"][j], c["mu"][j], c["nu"][j], c["mt"][j] * dt, c["gt"][j] * dt)
        f = rhs(ym1)
        acc = r[0] * y0
        acc = acc + r[1] * ym1
        acc = acc + r[2] * ym2
        acc = acc + r[3] * f
        yj = acc + r[4] * f0
        ym2, ym1 = ym1, yj
    return ym1
