"""The Wick-determinant integrand on the GPU (Schur-complement tree and keldy's
per-configuration LU), through the C ABI, against keldy's integrand (golden.npz) and the
CPU oracle. Tolerance: |gpu - keldy| <= 1e-12 * sum_a |det up det down| (the alternating
sum cancels, so the error scale is the sum of the magnitudes of its terms)."""
import numpy as np
import pytest

from keldy_b200 import capi
from tests.golden.make_golden import EXTERNALS

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _check(got, want, scale, tol=TOL):
    err = np.abs(got - want)
    bound = tol * np.maximum(scale, 1e-300) + 1e-300
    assert np.all(err <= bound), (err / np.maximum(scale, 1e-300)).max()


@pytest.mark.parametrize("algo", [capi.ALGO_TREE, capi.ALGO_DIRECT])
def test_integrand_vs_keldy(ctx, oracle, golden, algo):
    for tname in ("T0", "beta20"):
        le, gr = golden[f"table_{tname}_lesser"], golden[f"table_{tname}_greater"]
        for alpha in (0.0, 0.8):
            gm = ctx.model(10.0, le, gr, alpha)
            om = oracle.model(10.0, le, gr, alpha)
            for ename, A, B in EXTERNALS:
                for n in range(0, 7):
                    key = f"integrand_{tname}_a{alpha}_{ename}_n{n}"
                    t = golden[key + "_t"]
                    v, d = gm.integrand(A, B, t, algo=algo, order=n)
                    _, _, sc = oracle.integrand(om, A, B, t)
                    np.testing.assert_array_equal(d, golden[key + "_d"])
                    _check(v, golden[key + "_v"], sc)


@pytest.mark.parametrize("n", [7, 8, 9, 10, 11, 12])
def test_integrand_high_orders_vs_oracle(ctx, oracle, golden, n):
    le, gr = golden["table_beta20_lesser"], golden["table_beta20_greater"]
    gm = ctx.model(10.0, le, gr, 0.3)
    om = oracle.model(10.0, le, gr, 0.3)
    rng = np.random.default_rng(100 + n)
    count = 6 if n <= 10 else 2
    t = rng.random((count, n)) * 10.0
    t[0] = np.sort(t[0])[::-1]
    A, B = EXTERNALS[0][1], EXTERNALS[0][2]
    want, dw, sc = oracle.integrand(om, A, B, t)
    for algo in (capi.ALGO_TREE, capi.ALGO_AUTO) + ((capi.ALGO_DIRECT,) if n <= 9 else ()):
        v, d, gsc = gm.integrand(A, B, t, algo=algo, want_scale=True)
        np.testing.assert_array_equal(d, dw)
        _check(v, want, sc)
        np.testing.assert_allclose(gsc, sc, rtol=1e-9)


def test_no_det_vs_keldy(ctx, golden):
    for tname in ("T0", "beta20"):
        gm = ctx.model(10.0, golden[f"table_{tname}_lesser"], golden[f"table_{tname}_greater"], 0.8)
        for ename, A, B in EXTERNALS:
            for n in (1, 2):
                key = f"integrand_{tname}_a0.8_{ename}_n{n}"
                v, _ = gm.integrand_no_det(A, B, golden[key + "_t"])
                np.testing.assert_allclose(v, golden[key + "_nodet"], rtol=1e-13, atol=1e-16)


def test_cutoff_domain_spins(ctx, oracle, golden):
    le, gr = golden["table_beta20_lesser"], golden["table_beta20_greater"]
    gm = ctx.model(10.0, le, gr)
    A, B = (5.0, 0, 0, 0, 0), (5.0, 0, 0, 0, 0)
    small = abs(gm.integrand(A, B, np.array([[2.0, 0.0]]))[0][0])
    for algo in (capi.ALGO_TREE, capi.ALGO_DIRECT):
        v, d = gm.integrand(A, B, np.array([[2.0, 0.0], [4.9, 4.8]]), cutoff=small * 1.0001, algo=algo)
        assert v[0] == 0 and v[1] != 0 and list(d) == [1, 1]
        v, d = gm.integrand(A, B, np.array([[1.0, -1.0]]), algo=algo)
        assert v[0] == 0 and d[0] == 0
        v, d = gm.integrand(A, (5.0, 1, 0, 0, 0), np.array([[2.0, 1.0]]), algo=algo)
        assert v[0] == 0 and d[0] == 0
    # keep_u_hypercube = false: negative times are evaluated (inside the g0 window)
    om = oracle.model(10.0, le, gr)
    t = np.array([[1.0, -2.0, 3.0]])
    v, d = gm.integrand(A, B, t, keep_u_hypercube=False)
    w, dw, sc = oracle.integrand(om, A, B, t, keep_u_hypercube=False)
    assert d[0] == 1 and dw[0] == 1
    _check(v, w, sc)


def test_external_time_checks(ctx, golden):
    gm = ctx.model(10.0, golden["table_T0_lesser"], golden["table_T0_greater"])
    with pytest.raises(capi.KbError):  # "An external point has negative time."
        gm.integrand((-1.0, 0, 0), (1.0, 0, 1), np.array([[1.0]]))
    with pytest.raises(capi.KbError):  # "An external point is out of g0 time window."
        gm.integrand((11.0, 0, 0), (1.0, 0, 1), np.array([[1.0]]))
    with pytest.raises(capi.KbError) as e:  # g0 evaluated outside the window
        gm.integrand((10.0, 0, 0), (10.0, 0, 1), np.array([[-5.0, 6.0]]), keep_u_hypercube=False)
    assert e.value.code == capi.KB_E_RANGE


def test_spin_asymmetric_model(ctx, oracle, golden):
    """Different spin-down tables: det(s2) is not the tree's pivot product, so AUTO runs
    keldy's per-configuration LU, and the tree refuses."""
    le, gr = golden["table_beta20_lesser"], golden["table_beta20_greater"]
    ld, gd = golden["table_T0_lesser"], golden["table_T0_greater"]
    gm = ctx.model(10.0, le, gr, 0.0, ld, gd)
    om = oracle.model(10.0, le, gr, 0.0, ld, gd)
    t = np.random.default_rng(5).random((10, 4)) * 10
    for A, B in [((10.0, 0, 0), (10.0, 0, 1)), ((6.0, 1, 1), (3.0, 1, 0))]:
        v, d = gm.integrand(A, B, t)
        w, dw, sc = oracle.integrand(om, A, B, t)
        _check(v, w, sc)
    with pytest.raises(capi.KbError):
        gm.integrand((10.0, 0, 0), (10.0, 0, 1), t, algo=capi.ALGO_TREE)


def test_dot_lead_orbitals(ctx, oracle, golden):
    """External points on orbital 1 (keldy's current observable, compute_obs.hpp:67-80)
    read the (1,0) / (0,1) blocks of the g0 tables."""
    le, gr = golden["table_beta20_lesser"], golden["table_beta20_greater"]
    le10, gr10 = 0.3 * le[::-1].conj(), 0.7 * gr
    gm = ctx.model(10.0, le, gr, 0.0, blocks={(0, 1, 0): (le10, gr10), (0, 0, 1): (-le10.conj(), -gr10.conj())})
    om = oracle.model(10.0, le, gr)
    import ctypes
    keep = []
    for (o1, o2), (a, b) in {(1, 0): (le10, gr10), (0, 1): (-le10.conj(), -gr10.conj())}.items():
        for k, arr in ((0, a), (1, b)):
            x = np.ascontiguousarray(arr, dtype=np.complex128).view(np.float64)
            keep.append(x)
            om.tab[(0 * 2 + o1) * 4 + o2 * 2 + k] = x.ctypes.data
            om.tab[(1 * 2 + o1) * 4 + o2 * 2 + k] = x.ctypes.data
    om._keep += keep
    t = np.random.default_rng(9).random((12, 3)) * 10
    A, B = (8.0, 0, 0, 0, 1), (8.0, 0, 1, 0, 0)
    v, d = gm.integrand(A, B, t)
    w, dw, sc = oracle.integrand(om, A, B, t)
    _check(v, w, sc)


def test_pivot_guard_falls_back_to_lu(ctx, oracle):
    """A table that vanishes at t = 0 makes every diagonal pivot ~0: the tree hands all
    points to the pivoted LU, and the values still equal keldy's."""
    t = np.linspace(-10, 10, 2001)
    le = 1j * t * np.exp(-t * t / 8) + 0.2 * np.sin(t)
    gr = -np.conj(le[::-1])
    gm = ctx.model(10.0, le, gr)
    om = oracle.model(10.0, le, gr)
    x = np.random.default_rng(2).random((20, 5)) * 10
    A, B = (10.0, 0, 0), (10.0, 0, 1)
    v, d = gm.integrand(A, B, x)
    w, dw, sc = oracle.integrand(om, A, B, x)
    _check(v, w, sc)


# ------------------------------------------------------------------ cubic g0 interpolation
def test_cubic_interpolation_vs_oracle(ctx, oracle, golden):
    """The cubic-interpolation option (an extension with no keldy counterpart) against the
    oracle's: g0 lookups bit-exact across the window (ends included), the integrand of
    orders 1-8 on both algorithms and the fused integration within the usual tolerances."""
    le, gr = golden["table_beta20_lesser"], golden["table_beta20_greater"]
    gm = ctx.model(10.0, le, gr, 0.3)
    gm.set_interpolation(3)
    om = oracle.model(10.0, le, gr, 0.3, interp=3)
    x = np.concatenate([np.random.default_rng(5).uniform(-10, 10, 300), [-10.0, -9.999, 9.999, 10.0, 0.0]])
    a = [(v, 0, 0, 0, 0) for v in x]
    b = [(0.0, 0, 1, 0, 0)] * len(x)
    got = gm.g0(a, b)
    want = np.array([oracle.g0(om, p, q) for p, q in zip(a, b)])
    np.testing.assert_array_equal(got, want)
    lin = ctx.model(10.0, le, gr, 0.3)
    assert np.abs(lin.g0(a, b) - got).max() > 0  # the option changes the values
    rng = np.random.default_rng(9)
    A, B = EXTERNALS[0][1], EXTERNALS[0][2]
    for n in range(1, 9):
        t = rng.random((8, n)) * 10.0
        want, dw, sc = oracle.integrand(om, A, B, t)
        for algo in (capi.ALGO_TREE, capi.ALGO_DIRECT):
            v, d = gm.integrand(A, B, t, algo=algo)
            np.testing.assert_array_equal(d, dw)
            _check(v, want, sc)
    chain = [(capi.WARPER_PLASMA_UV, 10.0, 0.0), (capi.WARPER_EXPONENTIAL, 10.0, 1.0)]
    for n in (2, 4, 6):
        s_o, np_o, nd_o, scale = oracle.integrate(om, A, B, chain, n, 4096)
        (s_g, np_g, nd_g, _), = capi.integrate(ctx, [dict(model=gm, rng=ctx.sobol(n), chain=chain, A=A, B=B,
                                                          order=n, n_points=4096)])
        assert (np_g, nd_g) == (np_o, nd_o) and abs(s_g - s_o) <= 1e-12 * scale


def test_cubic_interpolation_high_orders_vs_oracle(ctx, oracle, golden):
    """Cubic interpolation at the orders whose G is built once for several path passes
    (kept at the end of a shared-memory frontier buffer): evaluations and the fused
    integration against the oracle."""
    le, gr = golden["table_beta20_lesser"], golden["table_beta20_greater"]
    gm = ctx.model(10.0, le, gr, 0.3)
    gm.set_interpolation(3)
    om = oracle.model(10.0, le, gr, 0.3, interp=3)
    A, B = EXTERNALS[0][1], EXTERNALS[0][2]
    rng = np.random.default_rng(77)
    chain = [(capi.WARPER_PLASMA_UV, 10.0, 0.0), (capi.WARPER_EXPONENTIAL, 10.0, 1.0)]
    for n in (10, 11, 12):
        t = rng.random((2, n)) * 10.0
        want, dw, sc = oracle.integrand(om, A, B, t)
        v, d = gm.integrand(A, B, t, algo=capi.ALGO_TREE)
        np.testing.assert_array_equal(d, dw)
        _check(v, want, sc)
        s_o, np_o, nd_o, scale = oracle.integrate(om, A, B, chain, n, 3)
        (s_g, np_g, nd_g, _), = capi.integrate(ctx, [dict(model=gm, rng=ctx.sobol(n), chain=chain, A=A, B=B,
                                                          order=n, n_points=3)])
        assert (np_g, nd_g) == (np_o, nd_o) and abs(s_g - s_o) <= 1e-12 * scale, n


@pytest.mark.parametrize("n", [13, 14, 15, 16])
def test_integrand_maximum_orders_vs_oracle(ctx, oracle, golden, n):
    """The largest orders (up to the library's 16): the tree walks its first n - 8 levels one
    path at a time; one point each against the oracle's 2^n LU pairs."""
    le, gr = golden["table_beta20_lesser"], golden["table_beta20_greater"]
    gm = ctx.model(10.0, le, gr, 0.3)
    om = oracle.model(10.0, le, gr, 0.3)
    t = np.random.default_rng(300 + n).random((1, n)) * 10.0
    A, B = EXTERNALS[0][1], EXTERNALS[0][2]
    want, dw, sc = oracle.integrand(om, A, B, t)
    for algo in (capi.ALGO_TREE, capi.ALGO_AUTO):
        v, d = gm.integrand(A, B, t, algo=algo)
        np.testing.assert_array_equal(d, dw)
        _check(v, want, sc)


def test_empty_and_ragged_inputs(ctx, golden):
    """No points: empty results, no launch error; a work list mixing empty items and orders
    of uneven cost sums each item as it would alone; order 17 is refused."""
    gm = ctx.model(10.0, golden["table_beta20_lesser"], golden["table_beta20_greater"])
    A, B = EXTERNALS[0][1], EXTERNALS[0][2]
    v, d = gm.integrand(A, B, np.zeros((0, 3)))
    assert v.shape == (0,) and d.shape == (0,)
    chain = [(capi.WARPER_PLASMA_UV, 10.0, 0.0), (capi.WARPER_EXPONENTIAL, 10.0, 1.0)]
    items = [dict(model=gm, rng=ctx.sobol(n), chain=chain, A=A, B=B, order=n, n_points=p)
             for n, p in ((3, 0), (7, 333), (1, 5), (5, 0), (2, 1000))]
    together = capi.integrate(ctx, items)
    for it, res in zip(items, together):
        alone = capi.integrate(ctx, [it])[0]
        assert res[:3] == alone[:3]
        if it["n_points"] == 0:
            assert res[0] == 0 and res[1] == 0
    with pytest.raises(capi.KbError):
        capi.integrate(ctx, [dict(items[1], order=17, rng=ctx.sobol(17))])
