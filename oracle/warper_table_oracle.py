"""CPU restatement of keldy's tabulated product warpers and of make_warper_from_proj
(test infrastructure only; the package never imports it).

* table(u, f1): warper_product_1d_simple_interp_nearest_t::integrate_and_inverse
  (warpers/product_1d_simple.hpp:219-253): F[n-1] = 0, F[i] = F[i+1] - (f1[i+1] + f1[i])/2
  (u[i+1] - u[i]), normalised by -F[0] (then F[0] = -1), cut = first index of F's
  trailing zeros; f1 on an interval = the mean of its ends (:197-204).
* reverse / forward: GSL linear interpolation (index by bisection, last point in the last
  interval) of u(F) on F[0..cut] and of F(u) (:206-217, 322-330).
* projection(...): gather_data (make_warper_from_proj.hpp:68-98), kernel_smoothing
  (:40-66) with the local linear regression of interfaces/gsl_fit_linear_wrap.hpp:66-113
  (weighted least squares, weights <= 0 left out), f1 points (:135-150).
"""
from __future__ import annotations

import numpy as np


def table(u, f1):
    u = np.asarray(u, dtype=np.float64)
    f = np.array(f1, dtype=np.float64)
    n = len(u)
    F = np.zeros(n)
    cut, found = n - 1, False
    for i in range(n - 2, -1, -1):
        F[i] = F[i + 1] - 0.5 * (f[i + 1] + f[i]) * (u[i + 1] - u[i])
        found = found or F[i] != 0
        if not found:
            cut = i
    if not found:
        raise RuntimeError("Model function is flat zero.")
    norm = -F[0]
    F /= norm
    f /= norm
    F[0] = -1.0
    fm = 0.5 * (f[:-1] + f[1:])
    return dict(u=u, F=F, fm=fm, cut=cut, norm=norm)


def _interval(a, lo, hi, v):
    while hi > lo + 1:
        m = (lo + hi) >> 1
        if a[m] > v:
            hi = m
        else:
            lo = m
    return lo


def _lerp(x, x0, x1, y0, y1):
    dx = x1 - x0
    return y0 + (x - x0) / dx * (y1 - y0) if dx > 0 else y0


def reverse(t, l):
    y = -l
    i = _interval(t["F"], 0, t["cut"], y)
    u = _lerp(y, t["F"][i], t["F"][i + 1], t["u"][i], t["u"][i + 1])
    return u, 1.0 / t["fm"][_interval(t["u"], 0, len(t["u"]) - 1, u)]


def forward(t, u):
    i = _interval(t["u"], 0, len(t["u"]) - 1, u)
    return -_lerp(u, t["u"][i], t["u"][i + 1], t["F"][i], t["F"][i + 1]), t["fm"][i]


def map_reverse(tables, li):
    li = np.atleast_2d(li)
    out = np.empty_like(li)
    jac = np.ones(len(li))
    for p in range(len(li)):
        for j in range(li.shape[1]):
            t = tables[0] if len(tables) == 1 else tables[j]
            out[p, j], jj = reverse(t, li[p, j])
            jac[p] *= jj
    return out, jac


def kernel_smoothing(y, sigma):
    y = np.asarray(y, dtype=np.float64)
    N = len(y)
    H = max(min(int(3 * sigma), N), 1)
    K = 2 * H + 1
    ker = np.exp(-(((np.arange(K) - H) / sigma) ** 2) / 2)
    with np.errstate(divide="ignore", invalid="ignore"):
        logy = np.log(y)
    out = np.empty(N)
    for i in range(N):
        sk, ek = max(0, H - i), min(N + H - i - 1, K - 1)
        sx = sk - H + i
        x = np.arange(sx, sx + ek - sk + 1, dtype=np.float64)
        w = ker[sk:ek + 1].copy()
        w[y[sx:sx + len(x)] <= 0] = 0.0
        keep = w > 0
        xm = np.sum(w[keep] * x[keep]) / np.sum(w[keep])
        ym = np.sum(w[keep] * logy[sx:sx + len(x)][keep]) / np.sum(w[keep])
        dx = x[keep] - xm
        c1 = np.sum(w[keep] * dx * (logy[sx:sx + len(x)][keep] - ym)) / np.sum(w[keep] * dx * dx)
        out[i] = np.exp((ym - xm * c1) + i * c1)
    return out


def projection(li, values, num_bins, sigma):
    """Per axis: the tabulated warper's (u, f1) points from samples li [n, order] with values |f J|."""
    li = np.atleast_2d(li)
    bin_size = 1.0 / num_bins
    u = np.arange(num_bins + 1) * bin_size
    u[-1] = 1.0
    out = []
    for axis in range(li.shape[1]):
        x = li[:, axis]
        b = np.where(x == 1.0, num_bins - 1, np.minimum((x / bin_size).astype(np.int64), num_bins - 1))
        s = np.bincount(b, weights=values, minlength=num_bins)
        c = np.bincount(b, minlength=num_bins)
        avg = np.where(c > 0, s / np.maximum(c, 1), s)
        sm = kernel_smoothing(avg, sigma / bin_size)
        f1 = np.zeros(num_bins + 1)
        for i in range(num_bins):
            f1[i + 1] = 2 * sm[i] - f1[i]
        out.append((u.copy(), f1))
    return out
