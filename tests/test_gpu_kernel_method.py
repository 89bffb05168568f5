"""keldy's kernel method (integrand_g_kernel, compute_gf_kernel; wick_kernel.cpp:42-138,
compute_obs.hpp:105-117) on the GPU: point values and binned integration against the
oracle (pinned to keldy's closed forms in test_kernel_method_oracle.py), and keldy's
order-2 value test (compute_obs_kernel_test.cpp:12-60)."""
import numpy as np
import pytest

from keldy_b200 import capi, impurity_oneband as io, warpers

pytestmark = pytest.mark.gpu

X = (7.0, 0, 0, 0, 0)
PLASMA_EXP = [(capi.WARPER_PLASMA_UV, 10.0, 0.0), (capi.WARPER_EXPONENTIAL, 10.0, 1.0)]


@pytest.mark.parametrize("n", [1, 2, 3, 5, 7])
def test_point_values_vs_oracle(ctx, oracle, golden, n):
    le, gr = golden["table_beta20_lesser"], golden["table_beta20_greater"]
    gm = ctx.model(10.0, le, gr, 0.3)
    om = oracle.model(10.0, le, gr, 0.3)
    t = np.random.default_rng(n).random((12, n)) * 10.0
    t[1, 0] = -0.5               # out of the domain
    if n >= 2:
        t[2, 1] = t[2, 0]        # equal vertex times
    t[3, 0] = X[0]               # a vertex at the fixed point's time
    got, dom = gm.integrand_kernel(X, t)
    want, odom, sc = oracle.integrand_kernel(om, X, t)
    assert np.array_equal(dom, odom)
    for p in range(len(t)):
        assert np.abs(got[p] - want[p]).max() <= 1e-12 * max(sc[p], 1e-300), (p, np.abs(got[p] - want[p]).max(), sc[p])


@pytest.mark.parametrize("n", [1, 2, 4])
def test_binned_integration_vs_oracle(ctx, oracle, golden, n):
    le, gr = golden["table_beta20_lesser"], golden["table_beta20_greater"]
    gm = ctx.model(10.0, le, gr)
    om = oracle.model(10.0, le, gr)
    npts = 1024
    item = dict(model=gm, rng=ctx.sobol(n), chain=PLASMA_EXP, A=X, order=n, k_first=1, n_points=npts)
    s, npt, nd, bins, counts, dropped = capi.integrate_kernel(ctx, [item], 8, 0.0, 10.0)[0]
    ws, onp, ond, sc, obins, ocounts, odropped = oracle.integrate_kernel(om, X, PLASMA_EXP, n, npts, 8, 0.0, 10.0)
    assert (npt, nd) == (onp, ond)
    assert np.array_equal(counts, ocounts) and dropped == odropped
    assert np.abs(bins - obins).max() <= 1e-12 * sc
    assert abs(s - ws) <= 1e-12 * sc
    assert abs(bins.sum() - s) <= 1e-12 * sc  # nothing dropped on [0, t]


def test_keldy_order_2_kernel_values(keldy_tests):
    """compute_obs_kernel_test.cpp:12-60: semicircular bath at zero temperature, alpha = 0.5,
    G(t) bins of the order-2 kernel method against keldy's stored result (keldy's tolerance
    1e-6, its own QMC accuracy 2e-8). keldy integrated 1e6 points through an interpolated
    hybrid warper; here 2^22 Sobol points through plasma_uv + the 1/(v + 1) product warper
    (the same integral; g0 decays as 1/t at zero temperature, so a 1/v^3 warper would
    undersample the early time bins). The lesser column is the conjugate of the greater one."""
    k = keldy_tests["kernel_kat"]
    p = dict(k["params"])
    p["nr_time_points_gf"] = int(p["nr_time_points_gf"])
    model = io.G0Model(p, False)
    comp = io.ComputeGfKernel(model, k["t_max"], k["order"], k["nr_bins"])
    comp.warper.emplace_back(warpers.WarperPlasmaUvT(k["t_max"]))
    comp.warper.emplace_back(warpers.make_product_1d_simple_inverse(k["t_max"], 1.0))
    comp.run(1 << 22)
    res = comp.reduce_result()
    data = io.binner_data(res) / res.get_bin_size()
    want = np.array([[complex(*c) for c in row] for row in k["expected"]])
    assert np.abs(data[:, 0] - np.conj(data[:, 1])).max() < 1e-12
    assert np.abs(data - want).max() < k["tol"], np.abs(data - want).max()


def test_kernel_method_errors(ctx, golden):
    gm = ctx.model(10.0, golden["table_beta20_lesser"], golden["table_beta20_greater"])
    item = dict(model=gm, rng=ctx.sobol(11), chain=PLASMA_EXP, A=X, order=11, k_first=1, n_points=10)
    with pytest.raises(capi.KbError, match="orders 1..10"):
        capi.integrate_kernel(ctx, [item], 8, 0.0, 10.0)
    with pytest.raises(capi.KbError, match="wrong order"):
        capi.integrate_kernel(ctx, [dict(item, order=2, rng=ctx.sobol(2))], 8, 3.0, 1.0)


@pytest.mark.parametrize("n", [8, 9, 10])
def test_point_values_high_orders_vs_oracle(ctx, oracle, golden, n):
    """Orders 8-10 (the tree form walks the first n - 7 levels of orders 9 and 10 one path
    at a time)."""
    le, gr = golden["table_beta20_lesser"], golden["table_beta20_greater"]
    gm = ctx.model(10.0, le, gr, 0.3)
    om = oracle.model(10.0, le, gr, 0.3)
    t = np.random.default_rng(50 + n).random((3, n)) * 10.0
    got, dom = gm.integrand_kernel(X, t)
    want, odom, sc = oracle.integrand_kernel(om, X, t)
    assert np.array_equal(dom, odom)
    for p in range(len(t)):
        assert np.abs(got[p] - want[p]).max() <= 1e-12 * max(sc[p], 1e-300), (p, np.abs(got[p] - want[p]).max(), sc[p])


def test_spin_asymmetric_and_guarded_points(ctx, oracle, golden):
    """Points that leave the tree form take keldy's pivoted-LU path: a model whose spin-down
    tables differ (det(s2) is then not the tree's), and a table that vanishes at t = 0 (every
    diagonal pivot below the guard)."""
    le, gr = golden["table_beta20_lesser"], golden["table_beta20_greater"]
    rng = np.random.default_rng(4)
    t = rng.random((6, 4)) * 10.0
    # different spin-down tables
    ld, gd = 0.7 * le, 1.3 * gr
    gm = ctx.model(10.0, le, gr, 0.0, lesser_down=ld, greater_down=gd)
    om = oracle.model(10.0, le, gr, 0.0, lesser_down=ld, greater_down=gd)
    got, _ = gm.integrand_kernel(X, t)
    want, _, sc = oracle.integrand_kernel(om, X, t)
    for p in range(len(t)):
        assert np.abs(got[p] - want[p]).max() <= 1e-12 * sc[p]
    # a table zero at t = 0
    mid = len(le) // 2
    lz, gz = le.copy(), gr.copy()
    lz[mid] = 0.0
    gz[mid] = 0.0
    gm = ctx.model(10.0, lz, gz)
    om = oracle.model(10.0, lz, gz)
    got, _ = gm.integrand_kernel(X, t)
    want, _, sc = oracle.integrand_kernel(om, X, t)
    for p in range(len(t)):
        assert np.abs(got[p] - want[p]).max() <= 1e-12 * max(sc[p], 1e-300)


def _omega_values(oracle, om, times, omega):
    """integrand_g_kernel_single_omega restated on the oracle's per-(vertex, index) terms
    (wick_kernel_single_omega.cpp:126-135): sum_i e^{i omega t_i} (term_i0 + term_i1)."""
    vals, dom, sc = oracle.integrand_kernel(om, X_OMEGA, times)
    ph = np.exp(1j * omega * np.atleast_2d(times))
    return (vals.sum(axis=2) * ph).sum(axis=1), dom, sc


X_OMEGA = (5.0, 0, 0, 0, 0)


def test_single_omega_point_values_vs_oracle(ctx, oracle):
    """keldy's wick_kernel_single_omega_test.cpp setting (flat band, beta = 1, Gamma = 1,
    t_max = 10, 1,000 -> 1,001 points, X = (5, up, forward), omega = 1, times {2, 0} and
    {4.9, 4.8}), plus random points at orders 1..6, through keldy's Python name."""
    from keldy_b200.g0_tables import flatband
    _, le, gr = flatband(1.0, 0.0, 0.0, 1.0, 10.0, 1001)
    model = io.G0Model.from_tables(10.0, le, gr)
    om = oracle.model(10.0, le, gr)
    integ = io.IntegrandGKernelSingleOmega(io.G0KeldyshContourT(model), io.GfIndexT(5.0, 0, 0), 1.0)
    rng = np.random.default_rng(5)
    cases = [np.array([[2.0, 0.0], [4.9, 4.8]])] + [rng.random((6, n)) * 10.0 for n in range(1, 7)]
    for t in cases:
        want, dom, sc = _omega_values(oracle, om, t, 1.0)
        for p in range(len(t)):
            v, d = integ(list(t[p]))
            assert d == dom[p]
            assert abs(v - want[p]) <= 1e-12 * max(sc[p], 1e-300), (t[p], v, want[p])


@pytest.mark.parametrize("n,omega", [(1, 1.0), (2, -0.7), (4, 2.5), (6, 1.0)])
def test_single_omega_integration_vs_oracle(ctx, oracle, golden, n, omega):
    """integrator<dcomplex, integrand_g_kernel_single_omega>::run: Sobol points through the
    chain, each point's Fourier-weighted kernel terms times its Jacobian, summed."""
    le, gr = golden["table_beta20_lesser"], golden["table_beta20_greater"]
    gm = ctx.model(10.0, le, gr)
    om = oracle.model(10.0, le, gr)
    npts = 512
    item = dict(model=gm, rng=ctx.sobol(n), chain=PLASMA_EXP, A=X_OMEGA, order=n, k_first=1, n_points=npts)
    s, npt, nd = capi.integrate_kernel_single_omega(ctx, [item], omega)[0]
    li = oracle.sobol_points(n, 0, npts)
    u, jac = oracle.warp(PLASMA_EXP, li)
    f, dom, sc = _omega_values(oracle, om, u, omega)
    assert (npt, nd) == (npts, int(dom.sum()))
    assert abs(s - (f * jac).sum()) <= 1e-12 * (sc * np.abs(jac)).sum()


def test_single_omega_compute_class(ctx, oracle, golden):
    """ComputeGfKernelSingleOmega (compute_obs.hpp:119-133): run() twice continues the Sobol
    sequence, and reduce_result() is the mean over all points, equal to one integration."""
    le, gr = golden["table_beta20_lesser"], golden["table_beta20_greater"]
    model = io.G0Model.from_tables(10.0, le, gr)
    comp = io.ComputeGfKernelSingleOmega(model, 7.0, 0.8, 3)
    comp.warper.emplace_back(warpers.WarperPlasmaUvT(7.0))
    comp.run(300)
    comp.run(212)
    gm = ctx.model(10.0, le, gr)
    chain = [(capi.WARPER_PLASMA_UV, 7.0, 0.0)]
    s, npt, nd = capi.integrate_kernel_single_omega(ctx, [dict(model=gm, rng=ctx.sobol(3), chain=chain,
                                                               A=(7.0, 0, 0, 0, 0), order=3, k_first=1,
                                                               n_points=512)], 0.8)[0]
    assert comp.reduce_nr_points_run() == 512 and comp.reduce_nr_points_in_domain() == nd
    assert abs(comp.reduce_result() - s / 512) <= 1e-12 * abs(s / 512) + 1e-15
