"""The CPU oracle against keldy's own outputs (golden.npz, made by keldy's compiled
sources) and against the known answers of keldy's test suite."""
import numpy as np
import pytest

from oracle.pyoracle import W_PLASMA_UV, W_EXPONENTIAL, W_INVERSE_SQUARE, W_UNIFORM
from tests.golden.make_golden import CHAINS, EXTERNALS, SOBOL_CASES, SOBOL_COUNT


def test_sobol_bit_exact(oracle, golden):
    for i, (dim, seed, sh, sc, ss) in enumerate(SOBOL_CASES):
        got = oracle.sobol_points(dim, seed, SOBOL_COUNT, bool(sh), bool(sc), ss)
        assert np.array_equal(got, golden[f"sobol_{i}"]), (dim, seed, sh, sc, ss)


def test_sobol_first_points(oracle):
    # digitalseq_b2g's first points (sobol(3, 0): k = 1, 2, 3)
    p = oracle.sobol_points(3, 0, 3)
    assert np.array_equal(p, [[0.5, 0.5, 0.5], [0.75, 0.25, 0.25], [0.25, 0.75, 0.75]])


def test_sobol_seed_is_offset(oracle):
    a = oracle.sobol_points(6, 0, 200)
    b = oracle.sobol_points(6, 150, 50)
    assert np.array_equal(a[150:], b)


@pytest.mark.parametrize("name", sorted(CHAINS))
def test_warpers(oracle, golden, name):
    chain = CHAINS[name]
    u, j = oracle.warp(chain, golden[f"warp_{name}_li"], "reverse")
    assert np.array_equal(u, golden[f"warp_{name}_ui"])
    assert np.array_equal(j, golden[f"warp_{name}_jr"])
    l, jf = oracle.warp(chain, golden[f"warp_{name}_fin"], "forward")
    assert np.array_equal(l, golden[f"warp_{name}_fout"])
    assert np.array_equal(jf, golden[f"warp_{name}_jf"])


def test_plasma_vectors(oracle, keldy_tests):
    for v in keldy_tests["plasma_vectors"]:
        chain = [(W_PLASMA_UV, v["t_max"], 0.0)]
        vi, _ = oracle.warp(chain, np.array([v["ui"]]), "forward")
        np.testing.assert_allclose(vi[0], v["vi"], rtol=0, atol=1e-15)
        ui, _ = oracle.warp(chain, vi, "reverse")
        np.testing.assert_array_equal(ui[0], sorted(v["ui"], reverse=True))


def _models(oracle, golden):
    for tname in ("T0", "beta20"):
        for alpha in (0.0, 0.8):
            m = oracle.model(10.0, golden[f"table_{tname}_lesser"], golden[f"table_{tname}_greater"], alpha)
            yield tname, alpha, m


def test_integrand_matches_keldy(oracle, golden):
    """Restated integrand vs keldy's wick_direct.cpp: equal within 1e-13 of the
    sum of |det up * det down| (the alternating sum cancels)."""
    for tname, alpha, m in _models(oracle, golden):
        for ename, A, B in EXTERNALS:
            for n in range(0, 7):
                key = f"integrand_{tname}_a{alpha}_{ename}_n{n}"
                t = golden[key + "_t"]
                v, d, sc = oracle.integrand(m, A, B, t)
                np.testing.assert_array_equal(d, golden[key + "_d"])
                err = np.abs(v - golden[key + "_v"])
                assert np.all(err <= 1e-13 * np.maximum(sc, 1e-300) + 1e-300), (key, err.max())


def test_no_det_matches_keldy(oracle, golden):
    for tname, alpha, m in _models(oracle, golden):
        for ename, A, B in EXTERNALS:
            for n in range(0, 3):
                key = f"integrand_{tname}_a{alpha}_{ename}_n{n}"
                v, d = oracle.integrand(m, A, B, golden[key + "_t"], no_det=True)[:2]
                np.testing.assert_allclose(v, golden[key + "_nodet"], rtol=1e-14, atol=1e-17)


def test_det_equals_closed_form_orders_1_2(oracle, golden):
    # keldy's wick_direct_test.cpp:61-175: the determinant path equals the written-out
    # connected Wick sums at orders 1 and 2. eval_no_det hard-codes spin-up vertices for
    # the external line (wick_direct.cpp:188-216), so it applies to spin-up externals.
    for tname, alpha, m in _models(oracle, golden):
        for ename, A, B in EXTERNALS:
            if A[1] != 0:
                continue
            for n in (1, 2):
                t = golden[f"integrand_{tname}_a{alpha}_{ename}_n{n}_t"]
                v, _, sc = oracle.integrand(m, A, B, t)
                w, _, _ = oracle.integrand(m, A, B, t, no_det=True)
                assert np.all(np.abs(v - w) <= 1e-14 * sc + 1e-17)


def test_cutoff_and_domain(oracle, golden):
    m = oracle.model(10.0, golden["table_beta20_lesser"], golden["table_beta20_greater"])
    A, B = (5.0, 0, 0, 0, 0), (5.0, 0, 0, 0, 0)
    v, d, _ = oracle.integrand(m, A, B, np.array([[2.0, 1.0], [1.0, -1.0]]))
    assert list(d) == [1, 0] and v[1] == 0
    small = np.abs(oracle.integrand(m, A, B, np.array([[2.0, 0.0]]))[0][0])
    v2, _, _ = oracle.integrand(m, A, B, np.array([[2.0, 0.0]]), cutoff=small * 1.0001)
    assert v2[0] == 0
    # spins differ: zero and out of domain
    v3, d3, _ = oracle.integrand(m, A, (5.0, 1, 0, 0, 0), np.array([[2.0, 1.0]]))
    assert v3[0] == 0 and d3[0] == 0


def test_integrate_matches_keldy(oracle, golden):
    m = oracle.model(10.0, golden["table_beta20_lesser"], golden["table_beta20_greater"])
    A, B = EXTERNALS[0][1], EXTERNALS[0][2]
    for n in (1, 2, 3, 4):
        for cname in ("plasma_exponential", "uniform"):
            chain = [(W_PLASMA_UV, 10.0, 0.0), (W_EXPONENTIAL, 10.0, 1.0)] if cname == "plasma_exponential" \
                else [(W_UNIFORM, 10.0, 0.0)]
            s, npts, ndom, sc = oracle.integrate(m, A, B, chain, n, 4096)
            g = golden[f"integrate_{cname}_n{n}"]
            assert (npts, ndom) == (int(g[2]), int(g[3]))
            assert abs(s - complex(g[0], g[1])) <= 1e-13 * sc


def test_horvatic_zlatic_series(oracle, keldy_tests):
    """keldy's statistical known-answer test (compute_obs_test.cpp:93-136): charge
    series of the flat-band dot at T = 0 to order 6, 10^4 Sobol points."""
    from keldy_b200.g0_tables import flatband_analytic
    p = keldy_tests["hz_params"]
    hz = keldy_tests["hz_charge_series"]
    _, le, gr = flatband_analytic(p["Gamma"], p["time_max"], p["nr_time_points_gf"])
    m = oracle.model(p["time_max"], le, gr)
    t = p["t"]
    A, B = (t, 0, 0, 0, 0), (t, 0, 1, 0, 0)
    i_n = [1, 1j, -1, -1j]
    for order in range(1, 7):
        chain = [(W_PLASMA_UV, t, 0.0), (W_INVERSE_SQUARE, t, 1.0)]
        s, npts, _, _ = oracle.integrate(m, A, B, chain, order, 10000)
        q = -1j * i_n[order % 4] * s / npts
        tol = 1e-3 if order < 5 else 1e-2
        assert abs(q - hz[order]) <= tol * abs(hz[order]), (order, q, hz[order])
