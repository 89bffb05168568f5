"""The CPU restatement of keldy's "fft" tables (oracle/g0_fft_oracle.py) against keldy's fft
known answers, on keldy's frequency functions (keldy_b200.g0_tables.fft_samples)."""
import numpy as np

from keldy_b200 import g0_tables
from oracle import g0_fft_oracle


def _tables(p, dot_lead=False):
    beta = p["beta"] if p["beta"] > 0 else np.inf
    npts = int(p["nr_time_points_gf"])
    npts += 1 - npts % 2
    s = g0_tables.fft_samples(p["bath_type"], p["Gamma"], p["eps_d"], p["bias_V"], beta, p.get("half_bandwidth", 2.0),
                              p["time_max"], npts, dot_lead=dot_lead)
    out = {k: tuple(g0_fft_oracle.transform(v, p["time_max"]) for v in vals) for k, vals in s.items()}
    return g0_tables.time_mesh(p["time_max"], npts), out


def test_flatband_fft_known_answers(keldy_tests):
    """model_flatband_test.cpp Flatband_asym_1/2 and Flatband_3 (fft runs): g^<(1) within
    keldy's tolerances, and g(t) = -conj(g(-t)) within 1e-8."""
    for case in keldy_tests["flatband_fft_kat"]:
        t, tabs = _tables(case["params"])
        gl, gg = tabs[(0, 0)]
        for v in case["values"]:
            i = int(np.argmin(np.abs(t - v["t"])))
            assert abs(gl[i] - complex(v["re"], v["im"])) < v["tol"], (case["test"], gl[i])
        for sv in case["symmetry"]:
            g = gl if sv["function"] == "lesser" else gg
            i, j = int(np.argmin(np.abs(t - sv["t"]))), int(np.argmin(np.abs(t + sv["t"])))
            assert abs(g[i] + np.conj(g[j])) < sv["tol"]


def test_flatband_sym_fft_vs_analytic(keldy_tests):
    """model_flatband_test.cpp Flatband_sym: the fft tables at T ~ 0 against the analytic
    zero-temperature formula on t = -100, -98, ..., 100 (t = 0 included), within 1e-3."""
    k = keldy_tests["flatband_sym_kat"]
    p = k["params"]
    t, tabs = _tables(p)
    gl, gg = tabs[(0, 0)]
    _, al, ag = g0_tables.flatband_analytic(p["Gamma"], p["time_max"], len(t))
    for n in range(k["n_times"]):
        i = int(np.argmin(np.abs(t - (k["t0"] + n * k["dt"]))))
        assert abs(gl[i] - al[i]) < k["tol"] and abs(gg[i] - ag[i]) < k["tol"], t[i]


def test_semicircle_fft_known_answers(keldy_tests):
    """model_semicircle_test.cpp Semicirc_fft: dot and dot-lead blocks at t = 1 within keldy's
    1e-3 (the (0,1) block is the transform of -conj of the (1,0) frequency values)."""
    case = keldy_tests["semicircle_kat"][0]
    assert case["params"]["ft_method"] == "fft"
    t, tabs = _tables(case["params"], dot_lead=True)
    l10 = tabs[(1, 0)][0]
    blocks = {(0, 0): tabs[(0, 0)][0], (1, 0): l10, (0, 1): -np.conj(l10[::-1])}
    for v in case["values"]:
        i = int(np.argmin(np.abs(t - v["t"])))
        assert abs(blocks[(v["o1"], v["o2"])][i] - complex(v["re"], v["im"])) < v["tol"]


def test_lorentzian_fft_vs_quadrature():
    """The Lorentzian bath (model.cpp:114-118) has no keldy known answer: its fft table against
    an independent adaptive quadrature of g(t) = int dw/2pi e^{-iwt} g^<(w) (scipy's QUADPACK
    Fourier integrals on each half line), and the sum rule g^<(0) - g^>(0) = i."""
    from scipy.integrate import quad
    args = ("lorentzian", 1.0, 0.3, 0.5, 20.0, 2.0)
    tmax, L = 50.0, 20001
    s = g0_tables.fft_samples(*args, tmax, L)
    gl = g0_fft_oracle.transform(s[(0, 0)][0], tmax)
    gg = g0_fft_oracle.transform(s[(0, 0)][1], tmax)
    t = g0_tables.time_mesh(tmax, L)
    c = (L - 1) // 2
    assert abs((gl[c] - gg[c]) - 1j) < 1e-5

    def im_lesser(w):
        return g0_tables.omega_functions(*args, np.array([w]))[0][0].imag

    for tt in (0.5, 2.0, 7.0):
        i = int(np.argmin(np.abs(t - tt)))
        # g^<(w) = i b(w): g(t) = (1/2pi) int i b(w) (cos wt - i sin wt) dw
        re = sum(quad(lambda w, s=s_: im_lesser(s * w), 0, np.inf, weight="sin", wvar=tt, limlst=200)[0] * s_
                 for s_ in (1.0, -1.0)) / (2 * np.pi)
        im = sum(quad(lambda w, s=s_: im_lesser(s * w), 0, np.inf, weight="cos", wvar=tt, limlst=200)[0]
                 for s_ in (1.0, -1.0)) / (2 * np.pi)
        assert abs(gl[i] - complex(re, im)) < 1e-4, (tt, gl[i], complex(re, im))


def test_rational_oracle_vs_quadrature_and_flatband():
    """The closed-form transforms of the rational baths (oracle/g0_rational_oracle.py) against
    direct adaptive quadrature of int dw/2pi e^{-iwt} g(w) for the Lorentzian bath (dot and
    dot-lead blocks, both signs of t, finite temperature with bias), and against the host's
    closed-form flat-band tables (g0_tables.flatband) for the flat band's two-pole terms."""
    from oracle import g0_rational_oracle as ro
    terms = g0_tables.rational_terms("lorentzian", 1.0, 0.3, 0.5, 2.0, dot_lead=True)
    for blk, tol in (((0, 0), 1e-9), ((1, 0), 1e-6)):
        for tt in (0.0, 0.7, 5.0, -3.0):
            a, b = ro.transform(terms[blk], 20.0, [tt])
            assert abs(a[0] - g0_tables.rational_reference(terms[blk], 20.0, [tt], "lesser")[0]) < tol
            assert abs(b[0] - g0_tables.rational_reference(terms[blk], 20.0, [tt], "greater")[0]) < tol
    ft = g0_tables.rational_terms("flatband", 1.0, 0.4, 0.6, 2.0)
    t, hl, hg = g0_tables.flatband(1.0, 0.4, 0.6, 50.0, 20.0, 401)
    a, b = ro.transform(ft[(0, 0)], 50.0, t)
    assert np.abs(a - hl).max() < 1e-12 and np.abs(b - hg).max() < 1e-12


def test_rational_terms_reproduce_frequency_functions():
    """rational_terms' poles and residues give back keldy's frequency functions
    (omega_functions, model.hpp:94-170) on the real axis to rounding."""
    w = np.linspace(-5, 5, 11)
    for bath, dl in (("flatband", False), ("lorentzian", True)):
        terms = g0_tables.rational_terms(bath, 1.0, 0.3, 0.5, 2.0, dot_lead=dl)
        of = g0_tables.omega_functions(bath, 1.0, 0.3, 0.5, 20.0, 2.0, w)
        for blk, idx in (((0, 0), (0, 1)), ((1, 0), (2, 3))):
            if blk not in terms:
                continue
            for kind, oi in zip(("lesser", "greater"), idx):
                v = np.zeros(len(w), complex)
                for mu, poles, res in terms[blk]:
                    R = np.array([np.sum(res / (x - poles)) for x in w])
                    n = g0_tables._fermi(w - mu, 20.0)
                    v += n * R if kind == "lesser" else -(1 - n) * R
                assert np.abs(v - of[oi]).max() < 1e-13, (bath, blk, kind)
