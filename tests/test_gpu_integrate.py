"""integrator::run on the GPU (Sobol -> warper chain -> integrand -> sum), through the C
ABI, against keldy's integrator (golden.npz), the CPU oracle and keldy's Horvatic-Zlatic
known answer."""
import numpy as np
import pytest

from keldy_b200 import capi
from keldy_b200.g0_tables import flatband_analytic
from tests.golden.make_golden import EXTERNALS

pytestmark = pytest.mark.gpu

CHARGE = (EXTERNALS[0][1], EXTERNALS[0][2])
PLASMA_EXP = [(capi.WARPER_PLASMA_UV, 10.0, 0.0), (capi.WARPER_EXPONENTIAL, 10.0, 1.0)]
UNIFORM = [(capi.WARPER_UNIFORM, 10.0, 0.0)]


def _item(model, rng, chain, order, n, k_first=1, A=CHARGE[0], B=CHARGE[1], cutoff=0.0):
    return dict(model=model, rng=rng, chain=chain, A=A, B=B, cutoff=cutoff, order=order, k_first=k_first,
                n_points=n)


@pytest.mark.parametrize("algo", [capi.ALGO_AUTO, capi.ALGO_DIRECT])
def test_integrate_vs_keldy(ctx, oracle, golden, algo):
    le, gr = golden["table_beta20_lesser"], golden["table_beta20_greater"]
    gm = ctx.model(10.0, le, gr)
    om = oracle.model(10.0, le, gr)
    for n in (1, 2, 3, 4):
        rng = ctx.sobol(n)
        for cname, chain in (("plasma_exponential", PLASMA_EXP), ("uniform", UNIFORM)):
            (s, npts, ndom, nfb), = capi.integrate(ctx, [_item(gm, rng, chain, n, 4096)], algo)
            g = golden[f"integrate_{cname}_n{n}"]
            _, _, _, sc = oracle.integrate(om, CHARGE[0], CHARGE[1], chain, n, 4096)
            assert (npts, ndom) == (int(g[2]), int(g[3]))
            assert abs(s - complex(g[0], g[1])) <= 1e-12 * sc


def test_integrate_higher_orders_vs_oracle(ctx, oracle, golden):
    le, gr = golden["table_beta20_lesser"], golden["table_beta20_greater"]
    gm = ctx.model(10.0, le, gr)
    om = oracle.model(10.0, le, gr)
    for n, npts in ((5, 1024), (6, 512), (7, 256), (8, 128), (9, 64), (10, 24)):
        rng = ctx.sobol(n)
        (s, np_, nd, _), = capi.integrate(ctx, [_item(gm, rng, PLASMA_EXP, n, npts)])
        w, onp, ond, sc = oracle.integrate(om, CHARGE[0], CHARGE[1], PLASMA_EXP, n, npts)
        assert (np_, nd) == (onp, ond)
        assert abs(s - w) <= 1e-12 * sc, (n, abs(s - w) / sc)


def test_kept_g_across_path_passes(ctx, oracle, golden):
    """Orders 10-13 walk their first n - 8 levels in 2^(n-8) passes from one G per point,
    built once and kept at the end of a shared-memory frontier buffer. Their sums equal
    the oracle's, and bit for bit those of the no-alloc entry point (same kernel, its
    scratch in the library's static array)."""
    le, gr = golden["table_beta20_lesser"], golden["table_beta20_greater"]
    gm = ctx.model(10.0, le, gr)
    om = oracle.model(10.0, le, gr)
    for n, npts in ((10, 6), (11, 4), (12, 3), (13, 2)):
        item = _item(gm, ctx.sobol(n), PLASMA_EXP, n, npts)
        (s, np_, nd, _), = capi.integrate(ctx, [item])
        w, onp, ond, sc = oracle.integrate(om, CHARGE[0], CHARGE[1], PLASMA_EXP, n, npts)
        assert (np_, nd) == (onp, ond)
        assert abs(s - w) <= 1e-12 * sc, (n, abs(s - w) / sc)
        (s2, np2, nd2, _), = capi.integrate_noalloc(ctx, [item])
        assert (s2, np2, nd2) == (s, np_, nd), n


def test_batched_items_equal_separate_calls(ctx, golden):
    le, gr = golden["table_beta20_lesser"], golden["table_beta20_greater"]
    gm = ctx.model(10.0, le, gr)
    rngs = {n: ctx.sobol(n) for n in range(1, 8)}
    shifted = ctx.sobol(5, 31, True, True, 17)
    items = [_item(gm, rngs[n], PLASMA_EXP, n, 3000 + 17 * n, k_first=1 + 5 * n) for n in range(1, 8)]
    items.append(_item(gm, shifted, UNIFORM, 5, 2000))
    items.append(_item(gm, rngs[3], PLASMA_EXP, 3, 0))
    batched = capi.integrate(ctx, items)
    for it, b in zip(items, batched):
        assert capi.integrate(ctx, [it])[0] == b
    # deterministic: the same call twice gives identical sums
    assert capi.integrate(ctx, items) == batched


def test_integrate_equals_sum_of_point_values(ctx, golden):
    le, gr = golden["table_T0_lesser"], golden["table_T0_greater"]
    gm = ctx.model(10.0, le, gr)
    n, N = 4, 777
    rng = ctx.sobol(n, 31, True, False, 3)
    (s, npts, ndom, _), = capi.integrate(ctx, [_item(gm, rng, PLASMA_EXP, n, N, k_first=10)])
    li = rng.points(10, N)
    v, jac, dom = gm.evaluate_warped(CHARGE[0], CHARGE[1], PLASMA_EXP, li)
    assert npts == N and ndom == dom.sum()
    assert abs(s - v.sum()) <= 1e-13 * np.abs(v).sum()


def test_integrate_errors(ctx, golden):
    gm = ctx.model(10.0, golden["table_T0_lesser"], golden["table_T0_greater"])
    rng = ctx.sobol(3, 12)
    with pytest.raises(capi.KbError) as e:
        capi.integrate(ctx, [_item(gm, rng, UNIFORM, 3, 5000)])
    assert e.value.code == capi.KB_E_EXHAUSTED
    with pytest.raises(capi.KbError):
        capi.integrate(ctx, [_item(gm, ctx.sobol(2), UNIFORM, 3, 10)])  # fewer Sobol dimensions than the order
    with pytest.raises(capi.KbError) as e:  # warper reaching outside the g0 window
        capi.integrate(ctx, [_item(gm, ctx.sobol(2), [(capi.WARPER_UNIFORM, 25.0, 0.0)], 2, 100)])
    assert e.value.code == capi.KB_E_RANGE


def test_integrate_pivot_guard(ctx, oracle):
    t = np.linspace(-10, 10, 2001)
    le = 1j * t * np.exp(-t * t / 8) + 0.2 * np.sin(t)
    gr = -np.conj(le[::-1])
    gm = ctx.model(10.0, le, gr)
    om = oracle.model(10.0, le, gr)
    for n in (3, 5):
        (s, npts, nd, nfb), = capi.integrate(ctx, [_item(gm, ctx.sobol(n), PLASMA_EXP, n, 300)])
        w, _, ond, sc = oracle.integrate(om, CHARGE[0], CHARGE[1], PLASMA_EXP, n, 300)
        assert nfb > 0 and nd == ond
        assert abs(s - w) <= 1e-12 * sc


@pytest.mark.parametrize("run", [0, 1])
def test_horvatic_zlatic_series(ctx, keldy_tests, run):
    """keldy's known answer (compute_obs_test.cpp:93-181): charge series of the flat-band
    dot at T = 0 to order 6."""
    p = keldy_tests["hz_params"]
    cfg = p["runs"][run]
    hz = keldy_tests["hz_charge_series"]
    _, le, gr = flatband_analytic(p["Gamma"], p["time_max"], p["nr_time_points_gf"])
    gm = ctx.model(p["time_max"], le, gr)
    t = p["t"]
    kind = capi.WARPER_INVERSE_SQUARE if cfg["warper"] == "inverse_square" else capi.WARPER_EXPONENTIAL
    chain = [(capi.WARPER_PLASMA_UV, t, 0.0), (kind, t, cfg["w"])]
    items = [_item(gm, ctx.sobol(n), chain, n, cfg["n_points"], A=(t, 0, 0), B=(t, 0, 1)) for n in range(1, 7)]
    res = capi.integrate(ctx, items)
    i_n = [1, 1j, -1, -1j]
    for n, (s, npts, _, _) in zip(range(1, 7), res):
        q = -1j * i_n[n % 4] * s / npts
        tol = cfg["rtol"][0] if n < 5 else cfg["rtol"][1]
        assert abs(q - hz[n]) <= tol * abs(hz[n]), (n, q, hz[n])


def test_flat_band_orders_1_4_full_size_vs_oracle(ctx, oracle):
    """Orders 1..4 with 2^16 Sobol points each on the flat-band dot at beta = 50, t = 10,
    g0 on 10,001 points (10,000 raised to odd), with the product-1D 1/t ("identity on
    [0, t]") warper and with the plasma + exponential chain, against the CPU oracle."""
    from keldy_b200.g0_tables import flatband
    _, le, gr = flatband(1.0, 0.0, 0.0, 50.0, 10.0, 10001)
    gm = ctx.model(10.0, le, gr)
    om = oracle.model(10.0, le, gr)
    for chain in (UNIFORM, PLASMA_EXP):
        for n in (1, 2, 3, 4):
            (s, npts, nd, _), = capi.integrate(ctx, [_item(gm, ctx.sobol(n), chain, n, 1 << 16)])
            w, onp, ond, sc = oracle.integrate(om, CHARGE[0], CHARGE[1], chain, n, 1 << 16)
            assert (npts, nd) == (onp, ond)
            assert abs(s - w) <= 1e-12 * sc, (n, abs(s - w) / sc)


def test_biased_dot_high_orders_vs_oracle(ctx, oracle):
    """The biased dot (V = 1, eps_d = 0.5, beta = 100, t_max = 50, 100,001 mesh points, GPU
    builder), charge at t = 50, orders 6..12: integrate against the oracle on the same
    table and Sobol points."""
    gm, = capi.flatband_models(ctx, [(1.0, 0.5, 1.0, 100.0)], 50.0, 100001)
    le, gr = gm.table()
    om = oracle.model(50.0, le, gr)
    chain = [(capi.WARPER_PLASMA_UV, 50.0, 0.0), (capi.WARPER_EXPONENTIAL, 50.0, 1.0)]
    A, B = (50.0, 0, 0, 0, 0), (50.0, 0, 1, 0, 0)
    for n, npts in ((6, 256), (8, 64), (10, 12), (12, 3)):
        (s, np_, nd, _), = capi.integrate(ctx, [_item(gm, ctx.sobol(n), chain, n, npts, A=A, B=B)])
        w, onp, ond, sc = oracle.integrate(om, A, B, chain, n, npts)
        assert (np_, nd) == (onp, ond)
        assert abs(s - w) <= 1e-12 * sc, (n, abs(s - w) / sc)


def test_model_sweep_batched_equals_separate(ctx):
    """Many models with their own GPU-built tables and uneven orders in one launch give the
    same sums as one call per model."""
    params = [(1.0, e, v, b) for b in (10.0, 200.0) for v in (0.0, 1.3) for e in (-1.0, 0.2, 0.9)]
    models = capi.flatband_models(ctx, params, 20.0, 20001)
    chain = [(capi.WARPER_PLASMA_UV, 20.0, 0.0), (capi.WARPER_EXPONENTIAL, 20.0, 1.0)]
    rngs = {n: ctx.sobol(n) for n in range(2, 11)}
    items = [_item(m, rngs[2 + i % 9], chain, 2 + i % 9, 1500 - 60 * (i % 9), A=(20.0, 0, 0, 0, 0),
                   B=(20.0, 0, 1, 0, 0)) for i, m in enumerate(models)]
    batched = capi.integrate(ctx, items)
    for it, b in zip(items, batched):
        assert capi.integrate(ctx, [it])[0] == b


def test_contexts_on_two_devices(oracle, golden):
    """A context on each of two devices in one process: each sets the kernels' shared-memory
    limits on its own device when it is created, so the tree kernel (over the 48 KB
    default) launches on both. Skipped with fewer than two GPUs."""
    import torch
    if torch.cuda.device_count() < 2:
        pytest.skip("needs two GPUs")
    le, gr = golden["table_beta20_lesser"], golden["table_beta20_greater"]
    om = oracle.model(10.0, le, gr)
    w, onp, ond, sc = oracle.integrate(om, CHARGE[0], CHARGE[1], PLASMA_EXP, 8, 256)
    for dev in (0, 1):
        c = capi.Context(dev)
        gm = c.model(10.0, le, gr)
        (s, npts, nd, _), = capi.integrate(c, [_item(gm, c.sobol(8), PLASMA_EXP, 8, 256)])
        assert (npts, nd) == (onp, ond)
        assert abs(s - w) <= 1e-12 * sc, dev
