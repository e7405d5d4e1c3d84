"""Coefficients of the FP64 and FP32 sine / cosine polynomials in fastmath.cuh.

Method: Chebyshev approximation (mpmath.chebyfit, 50 significant digits) of
    g(t) = (sin(sqrt t) - sqrt t) / t^(3/2)   so that sin x = x + x^3 P(x^2),
    h(t) = (cos(sqrt t) - 1) / t              so that cos x = 1 + x^2 Q(x^2),
on t in [0, a^2] for the three argument ranges used by the kernels:
    a = 1/2   (sincos_half64: phase offsets |k| (R_i + R_j) <= 1/2)
    a = 1     (sincos_small64: offsets <= 1)
    a = pi/4  (sincos_cw64: after Cody-Waite reduction).
The coefficients are rounded to double; the script prints them (highest degree
first, as the Horner loops consume them) with the maximum absolute error of the
rounded polynomial against the 50-digit function over 4001 points of [0, a].

FP32 (the mixed-precision kernels: sincos_half32 / small32 / cw32 and the
packed f32x2 forms in dp0.cuh): the same polynomial shapes with fewer terms,
sin x = x + x^3 P(x^2) with 2 / 3 / 3 coefficients and cos x = 1 + x^2 Q(x^2)
with 3 / 4 / 4, on |x| <= 1/2, 1 and pi/4.  Each is a minimax fit of the
absolute error of sin / cos itself (not of P or Q) by Lawson's algorithm:
iteratively reweighted least squares on 2000 Chebyshev-spaced points of
[0, a], weights multiplied by the pointwise error each step, 400 steps (C. L.
Lawson, "Contributions to the theory of linear least maximum approximation",
1961).  The coefficients are rounded to float; the script reports the maximum
absolute error of the polynomial evaluated in float arithmetic with fused
multiply-adds (each fma emulated as one rounding of the exact double result)
against the 50-digit function over 20001 points of [0, a].

Run: python fit_sincos.py
"""

import mpmath as mp
import numpy as np

mp.mp.dps = 50

# (name, a, number of sine coefficients, number of cosine coefficients)
CLASSES = (("half64", mp.mpf(1) / 2, 5, 6), ("small64", mp.mpf(1), 7, 7), ("cw64", mp.pi / 4, 6, 7))


def _g(t):
    if t == 0:
        return mp.mpf(-1) / 6
    s = mp.sqrt(t)
    return (mp.sin(s) - s) / (t * s)


def _h(t):
    if t == 0:
        return mp.mpf(-1) / 2
    return (mp.cos(mp.sqrt(t)) - 1) / t


def fit(kind, a, ncoeff):
    poly = mp.chebyfit(_g if kind == "sin" else _h, [mp.mpf(0), a * a], ncoeff)
    coeffs = [float(c) for c in poly]
    worst = mp.mpf(0)
    for i in range(4001):
        x = a * i / 4000
        t = x * x
        p = mp.mpf(0)
        for c in coeffs:
            p = p * t + mp.mpf(c)
        v, ref = (x + x**3 * p, mp.sin(x)) if kind == "sin" else (1 + t * p, mp.cos(x))
        worst = max(worst, abs(v - ref))
    return coeffs, float(worst)


# (name, a, number of sine coefficients, number of cosine coefficients) of the FP32 polynomials
CLASSES32 = (("half32", 0.5, 2, 3), ("small32", 1.0, 3, 4), ("cw32", float(mp.pi / 4), 3, 4))


def fit32(kind, a, ncoeff, points=2000, steps=400):
    """Lawson minimax fit of x^3 P(x^2) to sin x - x (or x^2 Q(x^2) to cos x - 1) on [0, a]."""
    x = a * (1.0 - np.cos(np.pi * np.arange(points + 1) / points)) / 2.0
    x = x[1:]
    t = x * x
    if kind == "sin":
        target = np.array([float(mp.sin(mp.mpf(v)) - mp.mpf(v)) for v in x])
        basis = np.stack([x**3 * t ** (ncoeff - 1 - i) for i in range(ncoeff)], axis=1)
    else:
        target = np.array([float(mp.cos(mp.mpf(v)) - 1) for v in x])
        basis = np.stack([t ** (ncoeff - i) for i in range(ncoeff)], axis=1)
    w = np.full(len(x), 1.0 / len(x))
    for _ in range(steps):
        sw = np.sqrt(w)
        c = np.linalg.lstsq(basis * sw[:, None], target * sw, rcond=None)[0]
        w *= np.abs(basis @ c - target)
        w /= w.sum()
    return [np.float32(v) for v in c]


def error32(kind, a, coeffs, samples=20001):
    """Max absolute error of the float evaluation (Horner with fused multiply-adds)."""

    def fma(p, q, r):
        return np.float32(np.float64(p) * np.float64(q) + np.float64(r))

    worst = 0.0
    for i in range(samples):
        x = np.float32(a * i / (samples - 1))
        x2 = np.float32(x * x)
        p = coeffs[0]
        for c in coeffs[1:]:
            p = fma(p, x2, c)
        if kind == "sin":
            v, ref = fma(np.float32(x * x2), p, x), mp.sin(mp.mpf(float(x)))
        else:
            v, ref = fma(x2, p, np.float32(1.0)), mp.cos(mp.mpf(float(x)))
        worst = max(worst, abs(float(v) - float(ref)))
    return worst


if __name__ == "__main__":
    for name, a, ns, nc in CLASSES:
        for kind, n in (("sin", ns), ("cos", nc)):
            coeffs, err = fit(kind, a, n)
            print("%s %s (max abs error %.2e): {%s}" % (name, kind, err, ", ".join(repr(c) for c in coeffs)))
    for name, a, ns, nc in CLASSES32:
        for kind, n in (("sin", ns), ("cos", nc)):
            coeffs = fit32(kind, a, n)
            err = error32(kind, a, coeffs)
            print("%s %s (max abs error %.2e in float): {%s}"
                  % (name, kind, err, ", ".join(repr(float(c)) + "f" for c in coeffs)))
