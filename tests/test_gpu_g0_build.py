"""g0 tables built on the GPU (kb_models_set_flatband) against the host builder
(g0_tables.flatband) and keldy's flat-band known answers."""
import math

import numpy as np
import pytest

from keldy_b200 import capi, g0_tables

pytestmark = pytest.mark.gpu

CASES = [  # (Gamma, eps_d, V, beta)
    (1.0, 0.0, 0.0, 50.0), (1.0, 0.5, 1.0, 100.0), (1.0, 0.3, 0.4, 20.0), (1.5, -1.0, 2.0, 10.0),
    (0.7, 0.0, 0.0, 200.0), (1.0, 0.0, 0.0, math.inf), (1.0, -0.5, 1.0, math.inf), (1.0, 0.25, 0.5, 10.0),
]


@pytest.mark.parametrize("time_max,npts", [(10.0, 2001), (20.0, 4001), (50.0, 10001)])
def test_gpu_builder_equals_host_builder(ctx, time_max, npts):
    models = capi.flatband_models(ctx, CASES, time_max, npts)
    for m, (g, e, v, b) in zip(models, CASES):
        _, hl, hg = g0_tables.flatband(g, e, v, b, time_max, npts)
        dl, dg = m.table()
        scale = max(np.abs(hl).max(), np.abs(hg).max())
        assert np.abs(dl - hl).max() <= 1e-11 * scale, (g, e, v, b, np.abs(dl - hl).max())
        assert np.abs(dg - hg).max() <= 1e-11 * scale, (g, e, v, b, np.abs(dg - hg).max())


def test_batch_tables_outlive_their_neighbours(ctx):
    """The models of one kb_models_set_flatband call share one device allocation: closing
    some of them leaves the others' tables intact, with their maxima set (the batched
    maximum kernel), and a table uploaded later replaces a slice in place."""
    models = capi.flatband_models(ctx, CASES, 10.0, 2001)
    for i in (0, 3, 5):
        models[i].close()
    for i in (1, 2, 4, 6, 7):
        g, e, v, b = CASES[i]
        _, hl, hg = g0_tables.flatband(g, e, v, b, 10.0, 2001)
        dl, dg = models[i].table()
        scale = max(np.abs(hl).max(), np.abs(hg).max())
        assert np.abs(dl - hl).max() <= 1e-11 * scale and np.abs(dg - hg).max() <= 1e-11 * scale
    _, hl, hg = g0_tables.flatband(1.0, 0.1, 0.2, 30.0, 10.0, 2001)
    models[2].set_table(0, 0, 0, hl, hg)
    dl, dg = models[2].table()
    np.testing.assert_array_equal(dl, hl)
    np.testing.assert_array_equal(dg, hg)
    chain = [(capi.WARPER_PLASMA_UV, 10.0, 0.0), (capi.WARPER_EXPONENTIAL, 10.0, 1.0)]
    r = capi.integrate(ctx, [dict(model=models[7], rng=ctx.sobol(3), chain=chain, A=(10.0, 0, 0), B=(10.0, 0, 1),
                                  order=3, n_points=4096)])[0]
    assert r[1] == 4096 and np.isfinite(r[0])
    for i in (1, 2, 4, 6, 7):
        models[i].close()


def test_gpu_builder_known_answers(ctx, keldy_tests):
    # keldy's model_flatband_test.cpp:154-220 values (tol as in keldy)
    for case in keldy_tests["flatband_kat"]:
        p = case["params"]
        beta = math.inf if p["beta"] < 0 else p["beta"]
        npts = int(p["nr_time_points_gf"])
        npts += 1 - npts % 2
        m, = capi.flatband_models(ctx, [(p["Gamma"], p["eps_d"], p["bias_V"], beta)], p["time_max"], npts)
        gl, _ = m.table()
        t = g0_tables.time_mesh(p["time_max"], npts)
        for v in case["values"]:
            i = int(np.argmin(np.abs(t - v["t"])))
            assert abs(gl[i] - complex(v["re"], v["im"])) < v["tol"]


def test_gpu_built_model_integrates_like_uploaded(ctx):
    _, le, gr = g0_tables.flatband(1.0, 0.5, 1.0, 100.0, 10.0, 4001)
    up = ctx.model(10.0, le, gr)
    built, = capi.flatband_models(ctx, [(1.0, 0.5, 1.0, 100.0)], 10.0, 4001)
    chain = [(capi.WARPER_PLASMA_UV, 10.0, 0.0), (capi.WARPER_EXPONENTIAL, 10.0, 1.0)]
    rng = ctx.sobol(5)
    items = [dict(model=m, rng=rng, chain=chain, A=(10.0, 0, 0, 0, 0), B=(10.0, 0, 1, 0, 0), order=5,
                  n_points=20000) for m in (up, built)]
    (a, na, da, _), (b, nb, db, _) = capi.integrate(ctx, items)
    assert (na, da) == (nb, db)
    assert abs(a - b) <= 1e-9 * abs(a)


def test_builder_errors(ctx):
    with pytest.raises(capi.KbError):
        capi.flatband_models(ctx, [(1.0, 0.0, 0.0, 10.0)], 10.0, 2000)  # even mesh
    with pytest.raises(capi.KbError):
        capi.flatband_models(ctx, [(0.0, 0.0, 0.0, 10.0)], 10.0, 2001)  # Gamma = 0


# ------------------------------------------------------------------ semicircular bath
SEMI_CASES = [  # (Gamma, eps_d, V, beta, D)
    (1.0, 0.0, 0.0, 50.0, 2.0), (0.5, 0.3, 0.5, 20.0, 2.0), (1.0, -0.4, 3.0, 10.0, 1.0), (1.0, 0.2, 0.6, math.inf, 2.0),
]


@pytest.mark.parametrize("case", SEMI_CASES)
def test_gpu_semicircle_equals_host_builder(ctx, case):
    """The band quadrature's Fourier sums on the GPU (kb_model_set_fourier) against the same
    sums on the host (g0_tables.semicircle): every block within 1e-11 of the table maximum,
    with the dot-lead blocks and their mirror."""
    g, e, v, b, d = case
    time_max, npts = 10.0, 2001
    m = capi.semicircle_model(ctx, g, e, v, b, d, time_max, npts, dot_lead=True)
    t, hl, hg, l10, g10, l01, g01 = g0_tables.semicircle(g, e, v, b, d, time_max, npts, dot_lead=True)
    for (o1, o2), (wl, wg) in {(0, 0): (hl, hg), (1, 0): (l10, g10), (0, 1): (l01, g01)}.items():
        dl, dg = m.table(0, o1, o2)
        scale = max(np.abs(wl).max(), np.abs(wg).max())
        assert np.abs(dl - wl).max() <= 1e-11 * scale, (case, o1, o2, np.abs(dl - wl).max())
        assert np.abs(dg - wg).max() <= 1e-11 * scale, (case, o1, o2, np.abs(dg - wg).max())
    mid = npts // 2
    dl, _ = m.table()
    assert np.abs(dl[:mid] + np.conj(dl[::-1][:mid])).max() == 0.0  # g(-t) = -conj(g(t)) exactly


def test_gpu_semicircle_known_answers(keldy_tests):
    """keldy's model_semicircle_test.cpp:30-86 values (tolerance as keldy's) through
    G0Model, whose semicircular tables are now summed on the GPU."""
    from keldy_b200 import impurity_oneband as io
    case = keldy_tests["semicircle_kat"][1]
    p = dict(case["params"])
    p["nr_time_points_gf"] = 2001
    g = io.G0Model(p, True)
    t = g0_tables.time_mesh(p["time_max"], 2001)
    blocks = {(0, 0): g.get_table(0, 0, 0)[0], (0, 1): g.get_table(0, 0, 1)[0], (1, 0): g.get_table(0, 1, 0)[0]}
    for v in case["values"]:
        i = int(np.argmin(np.abs(t - v["t"])))
        assert abs(blocks[(v["o1"], v["o2"])][i] - complex(v["re"], v["im"])) < v["tol"]
    np.testing.assert_array_equal(g.g0_lesser, blocks[(0, 0)])
    # spin down reads the spin-up blocks
    np.testing.assert_array_equal(g.get_table(1, 1, 0)[0], blocks[(1, 0)])


def test_gpu_semicircle_model_integrates(ctx):
    """A charge integral on a GPU-built semicircular model equals the one on the same tables
    uploaded from the host (same table bytes up to the builder's 1e-11: sums within 1e-9)."""
    g, e, v, b, d = SEMI_CASES[1]
    m_dev = capi.semicircle_model(ctx, g, e, v, b, d, 10.0, 4001)
    _, hl, hg = g0_tables.semicircle(g, e, v, b, d, 10.0, 4001)
    m_host = ctx.model(10.0, hl, hg)
    chain = [(capi.WARPER_PLASMA_UV, 5.0, 0.0), (capi.WARPER_EXPONENTIAL, 5.0, 1.0)]
    items = [dict(model=m, rng=ctx.sobol(4), chain=chain, A=(5.0, 0, 0, 0, 0), B=(5.0, 0, 1, 0, 0), order=4,
                  n_points=1 << 14) for m in (m_dev, m_host)]
    (s1, n1, d1, _), (s2, n2, d2, _) = capi.integrate(ctx, items)
    assert (n1, d1) == (n2, d2) and abs(s1 - s2) <= 1e-9 * abs(s2)


def test_fourier_builder_errors(ctx):
    m = capi.Model(ctx, 10.0, None, None, npts=2000)
    w = np.array([0.0, 1.0])
    c = np.array([1.0 + 0j, 0.5j])
    with pytest.raises(capi.KbError, match="odd number"):
        m.set_fourier(0, 0, w, c, c, capi.FT_SYMMETRIC)
    m2 = capi.Model(ctx, 10.0, None, None, npts=2001)
    with pytest.raises(capi.KbError, match="off-diagonal"):
        m2.set_fourier(0, 0, w, c, c, capi.FT_MIRROR)
    with pytest.raises(capi.KbError, match="finite"):
        m2.set_fourier(0, 0, np.array([np.nan, 1.0]), c, c, 0)
    # a single node: g(t) = c e^{-i w t} exactly
    m2.set_fourier(1, 0, np.array([0.7]), np.array([0.3 - 0.2j]), np.array([1j]), capi.FT_MIRROR)
    t = g0_tables.time_mesh(10.0, 2001)
    l10, g10 = m2.table(0, 1, 0)
    np.testing.assert_allclose(l10, (0.3 - 0.2j) * np.exp(-0.7j * t), rtol=1e-13, atol=1e-15)
    l01, _ = m2.table(0, 0, 1)
    np.testing.assert_array_equal(l01, -np.conj(l10[::-1]))
