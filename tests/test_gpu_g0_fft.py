"""keldy's ft_method "fft" tables on the GPU (kb_model_set_fft, G0Model): the discrete
transform against the CPU restatement (oracle/g0_fft_oracle.py, numpy's FFT), and keldy's
fft known answers through keldy's Python names. The CPU restatement itself is pinned to
those known answers in test_g0_fft_oracle.py."""
import numpy as np
import pytest

from keldy_b200 import capi, g0_tables, impurity_oneband as io
from oracle import g0_fft_oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("L", [3, 2001, 10001])
def test_transform_vs_oracle(ctx, L):
    """Random frequency values with 1/w^2 tails: the GPU table equals numpy's FFT of the same
    sum within 1e-11 of the table's largest value (the direct sum of L terms and the FFT
    round differently, ~sqrt(L) ulps); the mirror block is -conj(g(-t))."""
    rng = np.random.default_rng(L)
    w = g0_tables.adjoint_frequencies(7.0, L)
    gl = (rng.normal(size=L) + 1j * rng.normal(size=L)) / (1.0 + w * w)
    gg = (rng.normal(size=L) + 1j * rng.normal(size=L)) / (1.0 + w * w)
    m = capi.Model(ctx, 7.0, None, None, npts=L)
    m.set_fft(1, 0, gl, gg, capi.FT_MIRROR)
    dl, dg = m.table(0, 1, 0)
    wl, wg = g0_fft_oracle.transform(gl, 7.0), g0_fft_oracle.transform(gg, 7.0)
    assert np.abs(dl - wl).max() <= 1e-11 * np.abs(wl).max()
    assert np.abs(dg - wg).max() <= 1e-11 * np.abs(wg).max()
    l01, _ = m.table(0, 0, 1)
    np.testing.assert_array_equal(l01, -np.conj(dl[::-1]))


def test_set_fft_errors(ctx):
    m = capi.Model(ctx, 5.0, None, None, npts=2000)
    v = np.ones(2000, dtype=np.complex128)
    with pytest.raises(capi.KbError, match="odd number"):
        m.set_fft(0, 0, v, v)
    m2 = capi.Model(ctx, 5.0, None, None, npts=2001)
    v = np.ones(2001, dtype=np.complex128)
    with pytest.raises(capi.KbError, match="off-diagonal"):
        m2.set_fft(0, 0, v, v, capi.FT_MIRROR)
    v[3] = np.nan
    with pytest.raises(capi.KbError, match="finite"):
        m2.set_fft(0, 0, v, v)


def _model(p, dot_lead=False):
    p = dict(p)
    p["nr_time_points_gf"] = int(p["nr_time_points_gf"])
    return io.G0Model(p, dot_lead)


def test_flatband_fft_known_answers(keldy_tests):
    """model_flatband_test.cpp Flatband_asym_1/2, Flatband_3 (fft runs) through G0Model."""
    for case in keldy_tests["flatband_fft_kat"]:
        g = _model(case["params"])
        t = g0_tables.time_mesh(case["params"]["time_max"], len(g.g0_lesser))
        for v in case["values"]:
            i = int(np.argmin(np.abs(t - v["t"])))
            assert abs(g.g0_lesser[i] - complex(v["re"], v["im"])) < v["tol"], case["test"]
        for sv in case["symmetry"]:
            tab = g.g0_lesser if sv["function"] == "lesser" else g.g0_greater
            i, j = int(np.argmin(np.abs(t - sv["t"]))), int(np.argmin(np.abs(t + sv["t"])))
            assert abs(tab[i] + np.conj(tab[j])) < sv["tol"]


def test_flatband_sym_fft_vs_analytic(keldy_tests):
    """model_flatband_test.cpp Flatband_sym: 100,001 points on [-1000, 1000] at beta = 1e5,
    against the zero-temperature formula on t = -100, -98, ..., 100 within 1e-3, and equal to
    the CPU restatement within 1e-12 of the table's maximum."""
    k = keldy_tests["flatband_sym_kat"]
    p = k["params"]
    g = _model(p)
    L = len(g.g0_lesser)
    t = g0_tables.time_mesh(p["time_max"], L)
    _, al, ag = g0_tables.flatband_analytic(p["Gamma"], p["time_max"], L)
    for n in range(k["n_times"]):
        i = int(np.argmin(np.abs(t - (k["t0"] + n * k["dt"]))))
        assert abs(g.g0_lesser[i] - al[i]) < k["tol"] and abs(g.g0_greater[i] - ag[i]) < k["tol"], t[i]
    s = g0_tables.fft_samples("flatband", p["Gamma"], p["eps_d"], p["bias_V"], p["beta"], 2.0, p["time_max"], L)
    want = g0_fft_oracle.transform(s[(0, 0)][0], p["time_max"])
    assert np.abs(g.g0_lesser - want).max() <= 1e-12 * np.abs(want).max()


def test_semicircle_fft_known_answers(keldy_tests):
    """model_semicircle_test.cpp Semicirc_fft (10,000 -> 10,001 points, dot-lead blocks) through
    G0Model with keldy's default ft_method, within keldy's tolerances; t <-> -t symmetry of
    the dot block and between the off-diagonal blocks within 1e-8."""
    case = keldy_tests["semicircle_kat"][0]
    assert case["params"]["ft_method"] == "fft"
    g = _model(case["params"], True)
    t = g0_tables.time_mesh(case["params"]["time_max"], len(g.g0_lesser))
    blocks = {(0, 0): g.get_table(0, 0, 0)[0], (0, 1): g.get_table(0, 0, 1)[0], (1, 0): g.get_table(0, 1, 0)[0]}
    for v in case["values"]:
        i = int(np.argmin(np.abs(t - v["t"])))
        assert abs(blocks[(v["o1"], v["o2"])][i] - complex(v["re"], v["im"])) < v["tol"]
    i, j = int(np.argmin(np.abs(t - 1.0))), int(np.argmin(np.abs(t + 1.0)))
    assert abs(blocks[(0, 0)][i] + np.conj(blocks[(0, 0)][j])) < 1e-8
    assert abs(blocks[(0, 1)][i] + np.conj(blocks[(1, 0)][j])) < 1e-8


def test_lorentzian_bath_tables_and_charge(ctx, oracle):
    """bath_type "lorentzian" (model.cpp:114-118) by keldy's default fft method: tables equal
    the CPU restatement, satisfy g^<(0) - g^>(0) = i, and integrate (charge at order 2)
    to the oracle's sum on the same tables."""
    p = io.model_param_t(bath_type="lorentzian", Gamma=1.0, eps_d=0.3, bias_V=0.5, beta=20.0, half_bandwidth=2.0,
                         time_max=20.0, nr_time_points_gf=8001)
    g = io.G0Model(p, False)
    s = g0_tables.fft_samples("lorentzian", 1.0, 0.3, 0.5, 20.0, 2.0, 20.0, 8001)
    want = g0_fft_oracle.transform(s[(0, 0)][0], 20.0)
    assert np.abs(g.g0_lesser - want).max() <= 1e-12 * np.abs(want).max()
    c = len(g.g0_lesser) // 2
    assert abs(g.g0_lesser[c] - g.g0_greater[c] - 1j) < 1e-5
    gm = ctx.model(20.0, g.g0_lesser, g.g0_greater)
    om = oracle.model(20.0, g.g0_lesser, g.g0_greater)
    chain = [(capi.WARPER_PLASMA_UV, 10.0, 0.0), (capi.WARPER_EXPONENTIAL, 10.0, 1.0)]
    A, B = (10.0, 0, 0, 0, 0), (10.0, 0, 1, 0, 0)
    (sm, npts, nd, _), = capi.integrate(ctx, [dict(model=gm, rng=ctx.sobol(2), chain=chain, A=A, B=B, order=2,
                                                   k_first=1, n_points=4096)])
    w, onp, ond, sc = oracle.integrate(om, A, B, chain, 2, 4096)
    assert (npts, nd) == (onp, ond) and abs(sm - w) <= 1e-12 * sc


@pytest.mark.parametrize("beta", [np.inf, 50.0, 5.0])
def test_rational_builder_reproduces_flatband_closed_form(ctx, beta):
    """kb_model_set_rational on the flat band's two-pole terms equals the host's closed-form
    flat-band tables (g0_tables.flatband: E1 at the poles, quadrature of the Fermi correction)
    to 1e-10 of the table's maximum, at zero and finite temperature, with bias."""
    gamma, eps, V, tmax, L = 1.0, 0.4, 0.6, 20.0, 4001
    terms = g0_tables.rational_terms("flatband", gamma, eps, V, 2.0)
    m = capi.Model(ctx, tmax, None, None, npts=L)
    m.set_rational(0, 0, terms[(0, 0)], beta, capi.FT_SYMMETRIC)
    dl, dg = m.table()
    _, hl, hg = g0_tables.flatband(gamma, eps, V, beta, tmax, L)
    scale = max(np.abs(hl).max(), np.abs(hg).max())
    assert np.abs(dl - hl).max() <= 1e-10 * scale and np.abs(dg - hg).max() <= 1e-10 * scale


def test_lorentzian_contour_tables(ctx):
    """bath_type "lorentzian", ft_method "contour" (model.cpp:326-426) through G0Model: the GPU's
    closed form equals the CPU restatement (oracle/g0_rational_oracle.py, pinned to direct
    quadrature in test_g0_fft_oracle.py) on the dot and dot-lead blocks at every mesh point to
    1e-10 of the table maximum, agrees with keldy's default fft tables of the same model
    within the fft's discretisation (2e-4 with the fft on a five times wider window, the same
    time step: the fft's table is periodic in t with the window's length, so near the edges
    of a window as short as the decay of g it aliases), satisfies the sum rule
    g^<(0) - g^>(0) = i, and the (0, 1) block mirrors the (1, 0) block."""
    from oracle import g0_rational_oracle
    p = io.model_param_t(bath_type="lorentzian", ft_method="contour", Gamma=1.0, eps_d=0.3, bias_V=0.5, beta=20.0,
                         half_bandwidth=2.0, time_max=20.0, nr_time_points_gf=801)
    g = io.G0Model(p, True)
    t = g0_tables.time_mesh(20.0, 801)
    terms = g0_tables.rational_terms("lorentzian", 1.0, 0.3, 0.5, 2.0, dot_lead=True)
    l00, g00 = g.get_table(0, 0, 0)
    l10, g10 = g.get_table(0, 1, 0)
    l01, _ = g.get_table(0, 0, 1)
    for (a, b), blk in (((l00, g00), (0, 0)), ((l10, g10), (1, 0))):
        wa, wb = g0_rational_oracle.transform(terms[blk], 20.0, t)
        scale = max(np.abs(wa).max(), np.abs(wb).max())
        assert np.abs(a - wa).max() <= 1e-10 * scale and np.abs(b - wb).max() <= 1e-10 * scale, blk
    c = len(t) // 2
    assert abs(l00[c] - g00[c] - 1j) < 1e-12
    np.testing.assert_array_equal(l01, -np.conj(l10[::-1]))
    gf = io.G0Model(dict(p, ft_method="fft", time_max=100.0, nr_time_points_gf=4001), True)
    sl = slice(1600, 2401)  # t in [-20, 20] on the wider mesh (same step 0.05)
    assert np.abs(gf.get_table(0, 0, 0)[0][sl] - l00).max() < 2e-4
    assert np.abs(gf.get_table(0, 1, 0)[0][sl] - l10).max() < 2e-4


def test_rational_builder_errors(ctx):
    m = capi.Model(ctx, 5.0, None, None, npts=201)
    with pytest.raises(capi.KbError, match="off the real axis"):
        m.set_rational(0, 0, [(0.0, np.array([1.0 + 0j, 1j]), np.array([1.0 + 0j, -1.0 + 0j]))], 10.0)
    with pytest.raises(capi.KbError, match="beta"):
        m.set_rational(0, 0, [(0.0, np.array([1j, -1j]), np.array([1.0 + 0j, -1.0 + 0j]))], -1.0)
    with pytest.raises(capi.KbError, match="1..8 poles"):
        m.set_rational(0, 0, [(0.0, np.full(9, 1j), np.zeros(9, complex))], 10.0)
