"""Fits the rational approximation of the Ewald real-space correction used by the pair kernel.

    G(z) = [erf(x) - 2x exp(-x^2)/sqrt(pi)] / x^3,   x = sqrt(z) = beta*r

so that the Coulomb part of the pair force scalar is  qq * (1/r^3 - beta^3 G(beta^2 r^2))
(equal to qq [erfc(br) + 2br/sqrt(pi) e^{-b^2r^2}] / r^3) and the exclusion correction is
-qq beta^3 G.  G is entire and even in x; on z in [0, 9] (beta*r <= 3; an Ewald tolerance of
1e-5 puts beta*rc near 2.8) a degree-(5,4) rational P(z)/Q(z), Q(0) = 1, fitted by linearised
least squares with Loeb reweighting and an error-proportional weight, has max |error| 3.3e-8 in
FP64 and 1.1e-7 when evaluated in FP32 (Horner, FP32 coefficients), the floor of FP32 Horner
evaluation here, with one multiply-add fewer than a (5,5) fit on [0, 12]; its denominator has no
zero for z >= 0. Run this file to regenerate the coefficients written into sb_ewald.cuh and
sb_pair_x2.cuh.
"""
import numpy as np
from math import factorial
from scipy.special import erf

ZMAX = 9.0


def G(z):
    z = np.asarray(z, np.float64)
    out = np.empty_like(z)
    small = z < 1e-3
    x = np.sqrt(z[~small])
    out[~small] = (erf(x) - 2 * x / np.sqrt(np.pi) * np.exp(-z[~small])) / x ** 3
    zs = z[small]
    s = np.zeros_like(zs)
    for n in range(12):
        a = (-1) ** (n + 1) / (factorial(n + 1) * (2 * n + 3)) - (-1) ** (n + 1) / factorial(n + 1)
        s += a * zs ** n
    out[small] = 2 / np.sqrt(np.pi) * s
    return out


def fit(m=5, n=4, iters=40):
    z = np.linspace(0, ZMAX, 20001)
    g = G(z)
    w = np.ones_like(z)
    for _ in range(iters):
        A = np.concatenate([np.vander(z, m + 1, increasing=True),
                            -(g[:, None] * np.vander(z, n + 1, increasing=True)[:, 1:])], axis=1)
        coef, *_ = np.linalg.lstsq(A * w[:, None], g * w, rcond=None)
        p, q = coef[:m + 1], np.concatenate([[1.0], coef[m + 1:]])
        Q = np.polyval(q[::-1], z)
        err = np.polyval(p[::-1], z) / Q - g
        w = (1 / np.abs(Q)) * (1 + 3 * np.abs(err) / np.abs(err).max())
    return p, q, np.abs(err).max()


if __name__ == "__main__":
    p, q, e = fit()
    print("// max abs error (FP64) %.3e on z in [0, %g]" % (e, ZMAX))
    print("P:", ", ".join("%.9ef" % c for c in p))
    print("Q:", ", ".join("%.9ef" % c for c in q))
