"""Coefficients of the FP64 sine / cosine polynomials in fastmath.cuh.

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

Run: python fit_sincos.py
"""

import mpmath as mp

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


if __name__ == "__main__":
    for name, a, ns, nc in CLASSES:
        for kind, n in (("sin", ns), ("cos", nc)):
            coeffs, err = fit(kind, a, n)
            print("%s %s (max abs error %.2e): {%s}" % (name, kind, err, ", ".join(repr(c) for c in coeffs)))
