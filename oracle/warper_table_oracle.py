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


# ---------------------------------------------------------------------------------------
# warper_projection_t (warpers/projection.hpp:176-382) and the hybrid warper
# (product_1d_simple.hpp:381-554), restated with the published methods they rest on:
# local linear regression (weighted least squares), Brent's minimisation, Akima's and
# Steffen's interpolation.

def gaussian_kernel(H, sigma):
    return np.exp(-(((np.arange(2 * H + 1) - H) / sigma) ** 2) / 2)


def local_linear_reg(y, kernel, dead):
    """interfaces/gsl_fit_linear_wrap.hpp:66-113 on x = 0..N-1: the weighted linear fit
    over the kernel window centred on each point, dead points left out."""
    y = np.asarray(y, dtype=np.float64)
    N, K = len(y), len(kernel)
    H = K // 2
    out = np.empty(N)
    for i in range(N):
        sk, ek = max(0, H - i), min(N + H - i - 1, K - 1)
        sx = sk - H + i
        n = ek - sk + 1
        x = np.arange(sx, sx + n, dtype=np.float64)
        w = np.where(dead[sx:sx + n], 0.0, kernel[sk:ek + 1])
        keep = w > 0
        W = w[keep].sum()
        xm = np.sum(w[keep] * x[keep]) / W
        ym = np.sum(w[keep] * y[sx:sx + n][keep]) / W
        dx = x[keep] - xm
        c1 = np.sum(w[keep] * dx * (y[sx:sx + n][keep] - ym)) / np.sum(w[keep] * dx * dx)
        out[i] = (ym - xm * c1) + i * c1
    return out


def brent_minimize(f, a, x, b, abstol, max_iter):
    """Brent's minimisation without derivatives (Brent 1973, ch. 5) from the bracket
    (a, x, b); stops when b - a < abstol or after max_iter steps; the best point."""
    golden = 0.5 * (3.0 - np.sqrt(5.0))
    fx, fa, fb = f(x), f(a), f(b)
    if not (fx < fa and fx < fb):
        raise RuntimeError("Endpoints do not enclose a minimum")
    v = w = x
    fv = fw = fx
    d = e = 0.0
    for _ in range(max_iter):
        mid = 0.5 * (a + b)
        tol = np.sqrt(np.finfo(float).eps) * abs(x) + 1e-12
        parabolic = False
        if abs(e) > tol:
            r = (x - w) * (fx - fv)
            q = (x - v) * (fx - fw)
            p = (x - v) * q - (x - w) * r
            q = 2.0 * (q - r)
            if q > 0:
                p = -p
            else:
                q = -q
            e_prev, e = e, d
            if abs(p) < abs(0.5 * q * e_prev) and q * (a - x) < p < q * (b - x):
                d = p / q
                u = x + d
                if u - a < 2 * tol or b - u < 2 * tol:
                    d = tol if x < mid else -tol
                parabolic = True
        if not parabolic:
            e = (b - x) if x < mid else (a - x)
            d = golden * e
        u = x + d if abs(d) >= tol else x + (tol if d > 0 else -tol)
        fu = f(u)
        if fu <= fx:
            if u < x:
                b = x
            else:
                a = x
            v, fv, w, fw, x, fx = w, fw, x, fx, u, fu
        else:
            if u < x:
                a = u
            else:
                b = u
            if fu <= fw or w == x:
                v, fv, w, fw = w, fw, u, fu
            elif fu <= fv or v == x or v == w:
                v, fv = u, fu
        if abs(b - a) < abstol:
            break
    return x


def optimize_sigma(y, sigma, upper):
    """projection.hpp:82-128: the width (bins, >= 0.3) minimising the leave-one-out error
    of the smoothed projection; Brent on [-upper, upper] from sigma, 20 steps, 1e-8."""
    y = np.asarray(y, dtype=np.float64)
    N = len(y)
    dead = ~(y > 0)
    with np.errstate(divide="ignore", invalid="ignore"):
        log_y = np.where(dead, 0.0, np.log(np.where(dead, 1.0, y)))
    H = max(min(int(3 * upper), N), 1)

    def cost(s):
        s = max(abs(s), 0.3)
        k = gaussian_kernel(H, s)
        k[H] = 0.0
        k = k / k[H + 1]
        c = np.sum((np.exp(local_linear_reg(log_y, k, dead)) - y) ** 2)
        if np.isnan(c):
            raise RuntimeError("Smoothing procedure returned a Nan.")
        return c

    return max(abs(brent_minimize(cost, -upper, sigma, upper, 1e-8, 20)), 0.3)


def mesh_eval(g, x):
    """TRIQS gf<retime> on the uniform mesh of [0, 1]: linear interpolation."""
    n = len(g)
    a = x * (1.0 / (1.0 / (n - 1)))
    fi = np.floor(a)
    w = a - fi
    i = int(fi)
    if i == n - 1 and abs(w) < 1e-14:
        i, w = n - 2, 1.0
    if not 0 <= i < n - 1:
        raise RuntimeError("out of window")
    return (1.0 - w) * g[i] + w * g[i + 1]


def hermite(x, x0, x1, y0, y1, d0, d1):
    h = x1 - x0
    s = (y1 - y0) / h
    c2 = (3.0 * s - 2.0 * d0 - d1) / h
    c3 = (d0 + d1 - 2.0 * s) / (h * h)
    dx = x - x0
    return y0 + dx * (d0 + dx * (c2 + dx * c3))


def akima_slopes(x, y):
    """Akima (1970) node slopes, end secants extrapolated linearly."""
    x, y = np.asarray(x, dtype=np.float64), np.asarray(y, dtype=np.float64)
    n = len(x)
    m = np.empty(n + 3)
    m[2:n + 1] = np.diff(y) / np.diff(x)
    m[1] = 2 * m[2] - m[3]
    m[0] = 2 * m[1] - m[2]
    m[n + 1] = 2 * m[n] - m[n - 1]
    m[n + 2] = 2 * m[n + 1] - m[n]
    t = np.empty(n)
    for i in range(n):
        mm2, mm1, m0, mp1 = m[i], m[i + 1], m[i + 2], m[i + 3]
        wl, wr = abs(mp1 - m0), abs(mm1 - mm2)
        t[i] = (wl * mm1 + wr * m0) / (wl + wr) if wl + wr > 0 else 0.5 * (mm1 + m0)
    return t


def steffen_slopes(x, y):
    """Steffen (1990) monotone node slopes, the end secants at both ends."""
    x, y = np.asarray(x, dtype=np.float64), np.asarray(y, dtype=np.float64)
    n = len(x)
    d = np.empty(n)
    d[0] = (y[1] - y[0]) / (x[1] - x[0])
    for i in range(1, n - 1):
        h0, h1 = x[i] - x[i - 1], x[i + 1] - x[i]
        s0, s1 = (y[i] - y[i - 1]) / h0, (y[i + 1] - y[i]) / h1
        p = (s0 * h1 + s1 * h0) / (h0 + h1)
        d[i] = (np.copysign(1.0, s0) + np.copysign(1.0, s1)) * min(abs(s0), abs(s1), 0.5 * abs(p))
    d[n - 1] = (y[n - 1] - y[n - 2]) / (x[n - 1] - x[n - 2])
    return d


def binner_gather(xs, values, xmin, xmax, nb):
    """binner_t<1>: the mean value per bin (x = xmax in the last bin) and the counts."""
    bs = (xmax - xmin) / nb
    data = np.zeros(nb)
    cnt = np.zeros(nb, dtype=np.int64)
    for x, v in zip(xs, values):
        if not xmin <= x <= xmax:
            continue
        b = nb - 1 if x == xmax else min(int((x - xmin) / bs), nb - 1)
        data[b] += v
        cnt[b] += 1
    return np.where(cnt > 0, data / np.maximum(cnt, 1), data), cnt


def projection_warper(li, values, num_bins, sigma, optimize=False):
    """warper_projection_t's constructor (projection.hpp:225-332): per axis a dict with
    fn, fint, inv (the three uniform-mesh tables), norm, sigma (natural units), xi, count."""
    li = np.atleast_2d(li)
    nb = num_bins
    delta = 1.0 / (nb - 1.0)
    xmin, xmax = -delta / 2, 1 + delta / 2
    bs = (xmax - xmin) / nb
    axes = []
    for axis in range(li.shape[1]):
        xi, cnt = binner_gather(li[:, axis], values, xmin, xmax, nb)
        s = sigma / bs
        if optimize:
            s = optimize_sigma(xi, s, 1.0 / bs)
        H = max(min(int(3 * s), nb), 1)
        with np.errstate(divide="ignore", invalid="ignore"):
            sm = np.exp(local_linear_reg(np.log(xi), gaussian_kernel(H, s), ~(xi > 0)))
        times = xmin + (np.arange(nb) + 0.5) * bs
        times[0], times[-1] = 0.0, 1.0
        mdelta = 1.0 / (nb - 1)
        mesh = np.arange(nb) * mdelta
        fn = np.array([_lerp(t, times[i], times[i + 1], sm[i], sm[i + 1])
                       for t in mesh for i in [_interval(times, 0, nb - 1, t)]])
        fint = np.array([0.0] + [mesh_eval(fn, mesh[j] - mdelta / 2) * mdelta for j in range(1, nb)])
        fint = np.cumsum(fint)
        norm = fint[-1]
        fint = fint / norm
        t = akima_slopes(fint, mesh)
        M = 1 + 5 * (nb - 1)
        inv = np.empty(M)
        for k in range(M):
            l = k * (1.0 / (M - 1))
            i = _interval(fint, 0, nb - 1, l)
            inv[k] = hermite(l, fint[i], fint[i + 1], mesh[i], mesh[i + 1], t[i], t[i + 1])
        axes.append(dict(fn=fn, fint=fint, inv=inv, norm=norm, sigma=s * bs, xi=xi, count=cnt))
    return axes


def projection_reverse(axes, l):
    """map_reverse (projection.hpp:330-344, 367-369): u_i = inv_i(l_i), J = prod norm_i / fn_i(u_i)."""
    u = [mesh_eval(a["inv"], x) for a, x in zip(axes, l)]
    jac = 1.0
    for a, x in zip(axes, u):
        jac *= a["norm"] / mesh_eval(a["fn"], x)
    return np.array(u), jac


def projection_forward(axes, u):
    """map_forward (projection.hpp:338-345, 352-358): l_i = fint_i(u_i), J = prod fn_i(u_i)."""
    l = [mesh_eval(a["fint"], x) for a, x in zip(axes, u)]
    jac = 1.0
    for a, x in zip(axes, u):
        jac *= mesh_eval(a["fn"], x)
    return np.array(l), jac


HYBRID_SHAPES = {
    "exponential": lambda w, p: (lambda t: np.exp(-t / w)),
    "inverse": lambda w, p: (lambda t: w / (w + t)),
    "inverse_square": lambda w, p: (lambda t: w * w / ((w + t) * (w + t))),
    "inverse_power": lambda w, p: (lambda t: np.prod([w] * p) / np.prod([w + t] * p)),
    "uniform": lambda w, p: (lambda t: 1.0),
}


def hybrid_table(f1, u_max, n):
    """warper_product_1d_simple_interp_hybrid_t's constructor (product_1d_simple.hpp:424-476):
    Simpson's rule from u_max down, normalised; Steffen slopes of F(u) and of u(F)."""
    delta = u_max / (n - 1)
    u = np.array([delta * i for i in range(n)])
    u[-1] = u_max
    F = np.zeros(n)
    cut, found = n - 1, False
    f2d = f1(u[-1])
    for i in range(n - 2, -1, -1):
        f0d = f2d
        f1d = f1(0.5 * (u[i + 1] + u[i]))
        f2d = f1(u[i])
        F[i] = F[i + 1] - delta / 6.0 * (f0d + 4 * f1d + f2d)
        found = found or F[i] != 0
        if not found:
            cut = i
    norm = -F[0]
    F = F / norm
    F[0] = -1.0
    return dict(u=u, F=F, dF=steffen_slopes(u, F), du=steffen_slopes(F[:cut + 1], u[:cut + 1]), cut=cut,
                norm=norm, f1=f1)


def hybrid_reverse(t, l):
    y = -l
    i = _interval(t["F"], 0, t["cut"], y)
    u = hermite(y, t["F"][i], t["F"][i + 1], t["u"][i], t["u"][i + 1], t["du"][i], t["du"][i + 1])
    return u, 1.0 / (t["f1"](u) / t["norm"])


def hybrid_forward(t, u):
    i = _interval(t["u"], 0, len(t["u"]) - 1, u)
    f = t["f1"](u) / t["norm"]
    return -hermite(u, t["u"][i], t["u"][i + 1], t["F"][i], t["F"][i + 1], t["dF"][i], t["dF"][i + 1]), f
