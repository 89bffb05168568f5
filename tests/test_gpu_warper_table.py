"""Tabulated product warpers (warper_product_1d_simple_interp_nearest_t,
warper_product_1d_interp_nearest_t) and make_warper_from_proj on the GPU: maps against the
oracle restatement (oracle/warper_table_oracle.py), keldy's interp-warper tests
(test/c++/warpers/product_1d_simple_interp_test.cpp), and a projection warper in the
chain: the same estimate as without it."""
import math

import numpy as np
import pytest

from keldy_b200 import capi, impurity_oneband as io, rqmc, warpers
from keldy_b200.g0_tables import flatband
from oracle import warper_table_oracle as wt

pytestmark = pytest.mark.gpu


def _random_tables(nt, rng):
    out = []
    for _ in range(nt):
        n = int(rng.integers(3, 40))
        u = np.concatenate([[0.0], np.cumsum(rng.random(n - 1) + 0.05)])
        f1 = rng.random(n) + 0.1
        out.append((u, f1))
    return out


@pytest.mark.parametrize("ndims", [1, 4])
def test_maps_vs_oracle(ctx, ndims):
    rng = np.random.default_rng(ndims)
    tabs = _random_tables(ndims, rng)
    tw = capi.WarperTable(ctx, tabs)
    li = rng.random((300, 4))
    u, jac = ctx.warp([tw.entry()], li)
    ou, ojac = wt.map_reverse([wt.table(a, b) for a, b in tabs], li)
    assert np.abs(u - ou).max() <= 1e-13 * np.abs(ou).max()
    assert np.abs(jac / ojac - 1).max() <= 1e-13
    back, fj = ctx.warp([tw.entry()], u, capi.FORWARD)
    np.testing.assert_allclose(back, li, atol=1e-12)
    np.testing.assert_allclose(fj * jac, 1.0, rtol=1e-12)


def test_keldy_interp_nearest_tests():
    """product_1d_simple_interp_test.cpp:14-52: f1 = 1 on [0, 1.5] (from a function or from
    points) maps l to u = 1.5 (1 - l) with Jacobian 1.5 per coordinate; f1 = exp(-u / 2)
    gives keldy's closed form l(u) within 1e-9 at 1000 points."""
    t_max = 1.5
    for w in (warpers.WarperProduct1dSimpleInterpNearestT(lambda u: 1.0, t_max, 8),
              warpers.WarperProduct1dSimpleInterpNearestT([0.0, 0.5, 0.75, 1.0, t_max], [1.0] * 5)):
        li = [0.3, 0.7, 0.05]
        u, jac = w.map_reverse(li)
        assert np.allclose(u, [t_max * (1 - l) for l in li], atol=1e-10)
        assert abs(jac - t_max ** 3) < 1e-10
        assert np.allclose(w.map_forward(u)[0], li, atol=1e-10)
    w = warpers.WarperProduct1dSimpleInterpNearestT(lambda u: math.exp(-u / 2.0), 5.0, 1000)
    for x in (0.0, 0.7, 2.5, 4.99, 5.0):
        l = w.map_forward([x])[0][0]
        want = (math.exp(-2.5) - math.exp(-x / 2.0)) / math.expm1(-2.5)
        assert abs(l - want) < 1e-6
    with pytest.raises(RuntimeError, match="flat zero"):
        warpers.WarperProduct1dSimpleInterpNearestT([0.0, 1.0, 2.0], [0.0, 0.0, 0.0])
    with pytest.raises(RuntimeError, match=">= 3"):
        warpers.WarperProduct1dSimpleInterpNearestT([0.0, 1.0], [1.0, 1.0])
    prod = warpers.WarperProduct1dInterpNearestT()
    prod.emplace_back(warpers.WarperProduct1dSimpleInterpNearestT(lambda u: 1.0, 2.0, 5))
    prod.emplace_back(warpers.WarperProduct1dSimpleInterpNearestT(lambda u: 1.0, 3.0, 5))
    u, jac = prod.map_reverse([0.5, 0.5])
    assert np.allclose(u, [1.0, 1.5]) and abs(jac - 6.0) < 1e-12


def _flat_model(ctx, order=4):
    """Flat band at t = 20; the g0 window is order * t, as keldy's projection example
    (test/python/projection_test.py:20-29), since without keep_u_hypercube the plasma
    warper's vertex times reach beyond [0, t]."""
    _, le, gr = flatband(1.0, 0.0, 0.0, 50.0, 20.0 * order, 8001)
    return ctx.model(20.0 * order, le, gr)


def test_projection_warper_vs_oracle(ctx):
    gm = _flat_model(ctx, 3)
    A, B = (20.0, 0, 0, 0, 0), (20.0, 0, 1, 0, 0)
    chain = [(capi.WARPER_PLASMA_UV, 20.0, 0.0), (capi.WARPER_INVERSE, 20.0, 1.2)]
    order, nbins, nsamples, sigma = 3, 100, 5000, 0.1
    tw = capi.WarperTable.from_projection(ctx, gm, A, B, chain, order, nbins, nsamples, sigma, keep_u_hypercube=False)
    li = ctx.sobol(order).points(1, nsamples)
    vals = np.abs(gm.evaluate_warped(A, B, chain, li, keep_u_hypercube=False)[0])
    tabs = [wt.table(u, f1) for u, f1 in wt.projection(li, vals, nbins, sigma)]
    x = np.random.default_rng(3).random((200, order))
    u, jac = ctx.warp([tw.entry()], x)
    ou, ojac = wt.map_reverse(tabs, x)
    assert np.abs(u - ou).max() <= 1e-9 and np.abs(jac / ojac - 1).max() <= 1e-9


def test_projection_warper_in_the_chain_keeps_the_estimate(ctx):
    gm = _flat_model(ctx)
    A, B = (20.0, 0, 0, 0, 0), (20.0, 0, 1, 0, 0)
    chain = [(capi.WARPER_PLASMA_UV, 20.0, 0.0), (capi.WARPER_INVERSE, 20.0, 1.2)]
    order = 4
    tw = capi.WarperTable.from_projection(ctx, gm, A, B, chain, order, 200, 1 << 14, 0.1)
    mp, ep, _ = rqmc.estimate(ctx, gm, A, B, chain, order, 1 << 14, 16)
    ml, el, _ = rqmc.estimate(ctx, gm, A, B, chain + [tw.entry()], order, 1 << 14, 16)
    assert abs(ml - mp) <= 4 * math.hypot(ep, el), (ml, mp, ep, el)


def test_make_warper_from_proj_api():
    params = {"beta": -1.0, "bias_V": 0.0, "eps_d": 0.0, "Gamma": 1.0, "alpha": 0.0, "half_bandwidth": 2.0,
              "bath_type": "flatband", "time_max": 60.0, "nr_time_points_gf": 10001, "ft_method": "analytic"}
    model = io.G0Model(params, False)
    computer = io.ComputeChargeQDirect(model, 20.0, 3, 1e-15)
    train = warpers.WarperTrainT()
    train.emplace_back(warpers.WarperPlasmaUvT(20.0))
    train.emplace_back(warpers.make_product_1d_simple_inverse(20.0, 1.2))
    computer.warper = train
    proj = warpers.make_warper_from_proj(computer, 3, 500, 5000, 0.1, False)
    train.emplace_back(proj)
    computer.warper = train
    computer.run(4096)
    assert computer.reduce_nr_points_run() == 4096 and np.isfinite(computer.reduce_result())
