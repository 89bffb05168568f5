"""Host-side g0 tables of the single-level dot with flat-band leads.

keldy builds g0^<(t), g0^>(t) on the uniform mesh [-time_max, time_max] with an odd
number of points (model.cpp:79-90, 139-177). This module produces the same tables:

* :func:`flatband_analytic` restates keldy's zero-temperature formula
  (``make_flat_band_analytic``, model.cpp:428-466): beta = infinity, bias 0, eps_d 0.
* :func:`flatband` evaluates the Fourier transform of the flat-band dot functions
  (model.hpp:100-112, 129-130; Delta^R = -i Gamma/2 per lead, model.cpp:107-111) for
  any beta, eps_d and bias: the zero-temperature part in closed form through the
  complex exponential integral E1, the finite-temperature correction (localised within
  ~36/beta of each chemical potential) by Gauss-Legendre quadrature. Accurate to
  ~1e-12; keldy's own "fft"/"contour" methods approximate the same functions.

Conventions follow keldy: g(t) = int dw/2pi e^{-iwt} g(w), mu_left = -V/2,
mu_right = +V/2, and t < 0 from g(-t) = -conj(g(t)) (model.cpp:302-314).
"""
from __future__ import annotations

import numpy as np
from scipy.special import exp1, expi


def time_mesh(time_max, npts):
    """keldy's retime mesh: npts points on [-time_max, time_max]; an even count is raised
    by one so that t = 0 is a mesh point (model.cpp:87-90)."""
    if npts % 2 == 0:
        npts += 1
    delta = (time_max - (-time_max)) / (npts - 1)
    return -time_max + np.arange(npts) * delta


def flatband_analytic(gamma, time_max, npts):
    """Zero-temperature flat band, eps_d = 0, bias 0 (model.cpp:428-466):
    g^<(t) = [e^{Gt} Ei(-Gt) - e^{-Gt} Ei(Gt)]/(2 pi) + i/2 e^{-|Gt|}, g^<(0) = i/2,
    g^> = conj(g^<)."""
    t = time_mesh(time_max, npts)
    gt = gamma * t
    with np.errstate(all="ignore"):
        re = (np.exp(gt) * expi(-gt) - np.exp(-gt) * expi(gt)) / (2 * np.pi)
    gl = re + 0.5j * np.exp(-np.abs(gt))
    gl[t == 0.0] = 0.5j
    return t, gl, np.conj(gl)


def _lorentz_below(t, mu, eps, gamma):
    """K(t) = int_{-inf}^{mu} e^{-iwt} / ((w-eps)^2 + gamma^2) dw for t > 0 (array t)."""
    out = np.zeros(t.shape, dtype=np.complex128)
    for sgn in (+1, -1):
        z = eps + 1j * sgn * gamma
        v = 1j * (mu - z) * t
        if sgn < 0 and mu == eps:
            # the path ends on E1's cut (v = -gamma t): take the limit from below
            e1 = -expi(gamma * t) + 1j * np.pi
        else:
            e1 = exp1(v)
            # continuation of E1 across its cut when the path Re v = t Im z < 0 passes Im v = 0
            if sgn < 0 and mu > eps:
                e1 = e1 + 2j * np.pi
        J = -np.exp(-1j * z * t) * e1
        out += sgn * J
    return out / (2j * gamma)


def _fermi_correction(t, mu, eps, gamma, beta, nodes=240):
    """int dx e^{-i(x+mu)t} d(x) / ((x+mu-eps)^2 + gamma^2), d(x) = n_F(x) - theta(-x)."""
    W = 36.0 / beta
    xg, wg = np.polynomial.legendre.leggauss(nodes)
    out = np.zeros(t.shape, dtype=np.complex128)
    for a, b in ((-W, 0.0), (0.0, W)):
        x = 0.5 * (b - a) * xg + 0.5 * (b + a)
        w = 0.5 * (b - a) * wg
        ax = np.abs(x)
        d = np.sign(x) * np.exp(-beta * ax) / (1.0 + np.exp(-beta * ax))
        f = w * d / ((x + mu - eps) ** 2 + gamma ** 2)
        for s in range(0, len(t), 8192):
            ts = t[s:s + 8192]
            out[s:s + 8192] += np.exp(-1j * np.outer(ts, x + mu)) @ f
    return out


def flatband(gamma, eps_d, bias_V, beta, time_max, npts):
    """g^<, g^> of the dot coupled to two flat-band leads (each Delta^R = -i gamma/2) at
    inverse temperature beta (np.inf for zero temperature). Returns (t, lesser, greater)."""
    t = time_mesh(time_max, npts)
    tp = t[t > 0]
    mus = (-bias_V / 2.0, bias_V / 2.0)
    full = np.pi / gamma * np.exp(-1j * eps_d * tp - gamma * tp)
    less = np.zeros(tp.shape, dtype=np.complex128)
    great = np.zeros(tp.shape, dtype=np.complex128)
    for mu in mus:
        below = _lorentz_below(tp, mu, eps_d, gamma)
        corr = _fermi_correction(tp, mu, eps_d, gamma, beta) if np.isfinite(beta) else 0.0
        less += below + corr
        great += full - below - corr
    pref = gamma / (2 * np.pi)
    gl_pos = 1j * pref * less
    gg_pos = -1j * pref * great
    # t = 0: int n(w) / ((w-eps)^2 + gamma^2) dw in closed form at T = 0, plus correction
    occ = 0.0
    for mu in mus:
        k0 = (np.arctan((mu - eps_d) / gamma) + np.pi / 2) / gamma
        c0 = _fermi_correction(np.zeros(1), mu, eps_d, gamma, beta)[0].real if np.isfinite(beta) else 0.0
        occ += k0 + c0
    g0l = 1j * pref * occ
    g0g = -1j * pref * (2 * np.pi / gamma - occ)
    n = len(t)
    mid = n // 2
    gl = np.empty(n, dtype=np.complex128)
    gg = np.empty(n, dtype=np.complex128)
    gl[mid + 1:] = gl_pos
    gg[mid + 1:] = gg_pos
    gl[mid] = g0l
    gg[mid] = g0g
    gl[:mid] = -np.conj(gl_pos[::-1])
    gg[:mid] = -np.conj(gg_pos[::-1])
    return t, gl, gg


def _fermi(x, beta):
    if not np.isfinite(beta):
        return np.where(x < 0, 1.0, np.where(x > 0, 0.0, 0.5))
    return 0.5 * (1.0 - np.tanh(0.5 * beta * x))


def semicircle_nodes(gamma, eps_d, bias_V, beta, half_bandwidth, time_max, nodes=None):
    """Quadrature of the semicircular-bath Fourier integrals (model.cpp:92-105, 220-319):
    Delta^R(w) = Gamma/(2D) (w - i sqrt(D^2 - w^2)) per lead inside the band. As keldy's
    finite-contour method, the integrals run over the band [-D, D]; here in theta with
    w = -D cos(theta), which removes the square-root edges, by Gauss-Legendre panels split
    at the chemical potentials. Returns (w, f_less, f_great, f_l10, f_g10): the nodes and
    the weights of g(t) = sum_k f_k e^{-i w_k t} for the dot's lesser and greater functions
    and for the (right lead, dot) block (model.hpp:94-99)."""
    D = float(half_bandwidth)
    mus = (-bias_V / 2.0, bias_V / 2.0)
    breaks = sorted({0.0, np.pi} | {float(np.arccos(-mu / D)) for mu in mus if abs(mu) < D})
    n = nodes or int(96 + 2.0 * D * time_max)
    xg, wg = np.polynomial.legendre.leggauss(n)
    th_list, w_list = [], []
    for a, b in zip(breaks[:-1], breaks[1:]):
        th_list.append(0.5 * (b - a) * xg + 0.5 * (b + a))
        w_list.append(0.5 * (b - a) * wg)
    th = np.concatenate(th_list)
    wq = np.concatenate(w_list)
    w = -D * np.cos(th)
    jac = D * np.sin(th)
    root = D * np.sin(th)                       # sqrt(D^2 - w^2)
    delta_r = 0.5 * (gamma / D) * (w - 1j * root)  # per lead
    gR = 1.0 / (w - eps_d - 2.0 * delta_r)
    c = (gamma / D) * root                      # -i (Delta^R - Delta^A) per lead
    nl = [_fermi(w - mu, beta) for mu in mus]
    less_w = 1j * c * (nl[0] + nl[1]) * np.abs(gR) ** 2
    great_w = -1j * c * ((1 - nl[0]) + (1 - nl[1])) * np.abs(gR) ** 2
    # right lead - dot (model.hpp:94-99): -s n_R^(s) (Delta^R - Delta^A)_R g^A + Delta^R_R g_dot^(s)
    gA = np.conj(gR)
    l10_w = -(nl[1]) * (-1j * c) * gA + delta_r * less_w
    g10_w = (1 - nl[1]) * (-1j * c) * gA + delta_r * great_w
    k = wq * jac / (2 * np.pi)
    return w, k * less_w, k * great_w, k * l10_w, k * g10_w


def semicircle(gamma, eps_d, bias_V, beta, half_bandwidth, time_max, npts, dot_lead=False, nodes=None):
    """Dot coupled to two semicircular leads of half-bandwidth D (model.cpp:92-105), the
    Fourier sums of semicircle_nodes on the host.

    Returns (t, lesser, greater) for the dot, and with dot_lead=True also the
    (lead, dot) and (dot, lead) blocks: (t, lesser, greater, lesser_10, greater_10,
    lesser_01, greater_01) (right lead, model.hpp:94-99)."""
    t = time_mesh(time_max, npts)
    w, f_less, f_great, f_l10, f_g10 = semicircle_nodes(gamma, eps_d, bias_V, beta, half_bandwidth, time_max, nodes)

    def ft(f, times):
        out = np.empty(len(times), dtype=np.complex128)
        for s in range(0, len(times), 8192):
            out[s:s + 8192] = np.exp(-1j * np.outer(times[s:s + 8192], w)) @ f
        return out

    mid = len(t) // 2

    def dot_block(f):
        pos = ft(f, t[mid + 1:])
        g = np.empty(len(t), dtype=np.complex128)
        g[mid + 1:] = pos
        g[mid] = ft(f, np.zeros(1))[0]
        g[:mid] = -np.conj(pos[::-1])
        return g

    gl, gg = dot_block(f_less), dot_block(f_great)
    if not dot_lead:
        return t, gl, gg
    l10, g10 = ft(f_l10, t), ft(f_g10, t)
    l01 = -np.conj(l10[::-1])
    g01 = -np.conj(g10[::-1])
    return t, gl, gg, l10, g10, l01, g01


# ---------------------------------------------------------------- frequency domain
def bath_hybrid_R(bath_type, gamma, half_bandwidth, w):
    """Retarded hybridisation of one lead at real frequencies w (model.cpp:92-119):
    semicircle Gamma/(2D) (w - i sqrt(D^2 - w^2)) inside the band and
    Gamma/(2D) (w - sgn(w) sqrt(w^2 - D^2)) outside; flatband -i Gamma/2; lorentzian
    Gamma hw/2 / (w + i hw) (half_bandwidth read as the half width at half maximum)."""
    w = np.asarray(w, dtype=np.float64)
    g, D = float(gamma), float(half_bandwidth)
    if bath_type == "semicircle":
        inside = np.abs(w) < D
        root_in = np.sqrt(np.maximum(D * D - w * w, 0.0))
        root_out = np.sqrt(np.maximum(w * w - D * D, 0.0))
        sgn = np.where(np.signbit(w), -1.0, 1.0)
        return np.where(inside, 0.5 * (g / D) * (w - 1j * root_in), 0.5 * (g / D) * (w - sgn * root_out))
    if bath_type == "flatband":
        return np.full(w.shape, -0.5j * g, dtype=np.complex128)
    if bath_type == "lorentzian":
        return g * D / 2.0 / (w + 1j * D)
    raise RuntimeError("bath_type not defined")


def omega_functions(bath_type, gamma, eps_d, bias_V, beta, half_bandwidth, w):
    """keldy's g0_model_omega at real frequencies w (model.hpp:94-170; both leads alike, mu_left
    = -V/2, mu_right = +V/2): (g0_dot_lesser, g0_dot_greater, g0_rightlead_dot_lesser,
    g0_rightlead_dot_greater). On the real axis keldy keeps only i Im of the dot functions."""
    w = np.asarray(w, dtype=np.float64)
    dR = bath_hybrid_R(bath_type, gamma, half_bandwidth, w)
    dA = np.conj(dR)
    hyb = dR - dA                               # per lead, both leads alike
    gR = 1.0 / (w - eps_d - 2.0 * dR)
    gA = 1.0 / (w - eps_d - 2.0 * dA)
    mus = (-bias_V / 2.0, bias_V / 2.0)
    out = []
    for lesser in (True, False):
        s = 1 if lesser else -1
        nl = [_fermi(s * (w - mu), beta) for mu in mus]
        dot = -s * gR * (nl[0] * hyb + nl[1] * hyb) * gA
        out.append(1j * dot.imag)
    dots = list(out)
    for lesser, dot in zip((True, False), dots):
        s = 1 if lesser else -1
        # g0_rightlead_dot (model.hpp:94-99), with the full (complex) dot function
        full = -s * gR * (_fermi(s * (w - mus[0]), beta) * hyb + _fermi(s * (w - mus[1]), beta) * hyb) * gA
        out.append(-s * _fermi(s * (w - mus[1]), beta) * hyb * gA + dR * full)
    return tuple(out)


def adjoint_frequencies(time_max, npts):
    """The frequency mesh adjoint to keldy's time mesh (TRIQS make_adjoint_mesh): npts points
    w_j = (j - c) dw, c = (npts - 1)/2, dw = 2 pi / (npts dt)."""
    t = time_mesh(time_max, npts)
    L = len(t)
    dt = t[1] - t[0]
    return (np.arange(L) - (L - 1) // 2) * (2.0 * np.pi / (L * dt))


def fft_samples(bath_type, gamma, eps_d, bias_V, beta, half_bandwidth, time_max, npts, dot_lead=False):
    """The frequency values keldy's make_g0_by_fft transforms (model.cpp:179-212): on the
    adjoint mesh, the dot block i Im g0_dot^{</>}(w) and, with dot_lead, the (right lead, dot)
    block g0_rightlead_dot^{</>}(w). Returns {(o1, o2): (lesser_w, greater_w)}."""
    w = adjoint_frequencies(time_max, npts)
    dl, dg, ll, lg = omega_functions(bath_type, gamma, eps_d, bias_V, beta, half_bandwidth, w)
    out = {(0, 0): (dl, dg)}
    if dot_lead:
        out[(1, 0)] = (ll, lg)
    return out


# ---------------------------------------------------------------- rational baths
def _pf(c, poles):
    """Residues of c / prod_k (w - z_k) at its simple poles z_k."""
    poles = np.asarray(poles, dtype=np.complex128)
    res = np.empty(len(poles), dtype=np.complex128)
    for k, z in enumerate(poles):
        d = z - np.delete(poles, k)
        if np.any(np.abs(d) < 1e-9 * (1.0 + abs(z))):
            raise RuntimeError("the rational bath functions have a double pole at these parameters")
        res[k] = c / np.prod(d)
    return res


def rational_terms(bath_type, gamma, eps_d, bias_V, half_bandwidth, dot_lead=False):
    """keldy's dot functions for a bath with a rational hybridisation (flatband: Delta^R =
    -i Gamma/2, lorentzian: Gamma hw/2/(w + i hw) per lead; model.cpp:107-118) as sums over
    the leads l of Fermi functions times rational functions with simple poles:
    g^<(w) = sum_l n_F(w - mu_l) R_l(w), g^>(w) = -sum_l (1 - n_F(w - mu_l)) R_l(w)
    (model.hpp:94-112). R_dot = -(Delta^R - Delta^A) g^R g^A for both leads; the (right lead,
    dot) block (model.hpp:94-99) has R_1 + R_2 at mu_R and R_2 at mu_L, R_1 = -(Delta^R -
    Delta^A) g^A, R_2 = Delta^R R_dot. Returns {(o1, o2): [(mu, poles, residues), ...]}."""
    mus = (-bias_V / 2.0, bias_V / 2.0)
    g, eps, hw = float(gamma), float(eps_d), float(half_bandwidth)
    if bath_type == "flatband":
        # R_dot = i Gamma / ((w - eps)^2 + Gamma^2)
        poles = np.array([eps + 1j * g, eps - 1j * g])
        dot = (poles, _pf(1j * g, poles))
        if dot_lead:
            raise RuntimeError("The dot-lead g0 for flatband bath is singular and not implemented accurately.")
        return {(0, 0): [(mus[0], *dot), (mus[1], *dot)]}
    if bath_type != "lorentzian":
        raise RuntimeError("rational_terms: flatband or lorentzian bath")
    # g^R = (w + i hw) / Q(w), Q(w) = (w - eps)(w + i hw) - Gamma hw; R_dot = i Gamma hw^2 / (Q Q*)
    q = np.roots([1.0, 1j * hw - eps, -(1j * eps * hw + g * hw)])
    qs = np.conj(q)
    dpoles = np.concatenate([q, qs])
    dot = (dpoles, _pf(1j * g * hw * hw, dpoles))
    out = {(0, 0): [(mus[0], *dot), (mus[1], *dot)]}
    if dot_lead:
        p1 = np.concatenate([[-1j * hw], qs])
        r1 = _pf(1j * g * hw * hw, p1)                     # R_1 = i Gamma hw^2 / ((w + i hw) Q*)
        p2 = np.concatenate([[-1j * hw], q, qs])
        r2 = _pf(0.5 * g * hw * 1j * g * hw * hw, p2)      # R_2 = (Gamma hw / 2) / (w + i hw) * R_dot
        r12 = r2.copy()
        r12[0] += r1[0]
        r12[3:] += r1[1:]
        out[(1, 0)] = [(mus[1], p2, r12), (mus[0], p2, r2)]
    return out


def rational_reference(terms, beta, t, kind):
    """The transform (1/2pi) int e^{-iwt} g(w) dw of rational_terms' functions by direct
    adaptive quadrature on the real axis, |w| <= 3000 (test helper; kind 'lesser' or 'greater')."""
    from scipy.integrate import quad
    out = []
    for tt in np.atleast_1d(t):
        tot = 0j
        for mu, poles, res in terms:
            def f(w, mu=mu, poles=poles, res=res):
                r = np.sum(res / (w - poles))
                n = _fermi(w - mu, beta)
                return (n * r) if kind == "lesser" else (-(1.0 - n) * r)
            for part in ("real", "imag"):
                for sgn in (1.0, -1.0):
                    fc = (lambda w, s=sgn: getattr(f(s * w) * np.exp(-1j * s * w * tt), part))
                    v = sum(quad(fc, a, b, limit=5000, epsabs=1e-14, epsrel=1e-12)[0]
                            for a, b in ((0.0, 10.0), (10.0, 100.0), (100.0, 3000.0)))
                    tot += v if part == "real" else 1j * v
        out.append(tot / (2 * np.pi))
    return np.array(out)
