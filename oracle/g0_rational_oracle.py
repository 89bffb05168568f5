"""CPU restatement of the closed-form transforms of baths with a rational hybridisation
(test infrastructure only): keldy's contour method (c++/keldy/impurity_oneband/
model.cpp:326-426) integrates g(t) = int dw/2pi e^{-iwt} g(w) numerically along a contour;
for the flat band and the Lorentzian bath that integral has a closed form at each pole of
the rational functions R_l of keldy_b200.g0_tables.rational_terms, with scipy's principal
E1 (exp1) and a Gauss-Legendre quadrature of the Fermi correction (scipy / numpy)."""
from __future__ import annotations

import numpy as np
from scipy.special import exp1, expi


def _term(mu, poles, res, t, beta, nodes=240):
    """(K, F, C) of one term at t >= 0."""
    K = F = C = 0j
    for z, r in zip(poles, res):
        if t == 0.0:
            s = 1.0 if z.imag < 0 else -1.0
            K += r * (np.log(mu - z) - 1j * np.pi * s)
            if z.imag < 0:
                F += r * (-2j * np.pi)
            continue
        v = 1j * (mu - z) * t
        if z.imag < 0 and mu == z.real:
            e1 = -expi(-z.imag * t) + 1j * np.pi
        else:
            e1 = exp1(v)
            if z.imag < 0 and mu > z.real:
                e1 = e1 + 2j * np.pi
        K += r * (-np.exp(-1j * z * t) * e1)
        if z.imag < 0:
            F += r * (-2j * np.pi) * np.exp(-1j * z * t)
    if np.isfinite(beta):
        W = 36.0 / beta
        x, w = np.polynomial.legendre.leggauss(nodes)
        for a, b in ((-W, 0.0), (0.0, W)):
            xs = 0.5 * (b - a) * x + 0.5 * (b + a)
            ws = 0.5 * (b - a) * w
            dn = np.sign(xs) * np.exp(-beta * np.abs(xs)) / (1.0 + np.exp(-beta * np.abs(xs)))
            om = mu + xs
            R = sum(r / (om - z) for z, r in zip(poles, res))
            C += np.sum(ws * dn * R * np.exp(-1j * om * t))
    return K, F, C


def transform(terms, beta, times):
    """(lesser, greater) at the given times."""
    gl, gg = [], []
    for t in np.atleast_1d(times):
        less = great = 0j
        for mu, poles, res in terms:
            poles, res = np.asarray(poles), np.asarray(res)
            if t < 0:
                K, F, C = (np.conj(v) for v in _term(mu, np.conj(poles), np.conj(res), -t, beta))
            else:
                K, F, C = _term(mu, poles, res, t, beta)
            less += K + C
            great -= F - K - C
        gl.append(less / (2 * np.pi))
        gg.append(great / (2 * np.pi))
    return np.array(gl), np.array(gg)
