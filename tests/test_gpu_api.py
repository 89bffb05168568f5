"""keldy's Python interface (common, warpers, impurity_oneband names) running on the GPU:
the same calls a keldy user makes, checked against keldy's outputs, the oracle and
keldy's known answers."""
import math

import numpy as np
import pytest

from keldy_b200 import common, impurity_oneband as io, warpers
from tests.golden.make_golden import EXTERNALS

pytestmark = pytest.mark.gpu


def test_sobol(oracle):
    s = common.Sobol(3, 0)
    assert s() == [0.5, 0.5, 0.5] and s() == [0.75, 0.25, 0.25]
    s = common.Sobol(6, 0)
    want = oracle.sobol_points(6, 0, 200)
    got = np.array([s() for _ in range(100)] + list(s.points(100)))
    assert np.array_equal(got, want)
    s.seed(1000)
    assert np.array_equal(np.array(s()), oracle.sobol_points(6, 1000, 1)[0])
    s.discard(9)
    assert np.array_equal(np.array(s()), oracle.sobol_points(6, 1010, 1)[0])
    s = common.Sobol(5, 7, True, True, 3)
    assert np.array_equal(s.points(50), oracle.sobol_points(5, 7, 50, True, True, 3))
    s = common.Sobol(2, (1 << 10) - 2, 10)
    s()
    s()  # k = 2^10: the last point
    with pytest.raises(RuntimeError, match="More sample points"):
        s()


def test_warpers(oracle, keldy_tests):
    for v in keldy_tests["plasma_vectors"]:
        w = warpers.WarperPlasmaUvT(v["t_max"])
        np.testing.assert_allclose(w.li_from_ui(v["ui"]), v["vi"], atol=1e-15)
        np.testing.assert_allclose(warpers.vi_from_ui(v["t_max"], v["ui"]), v["vi"], atol=1e-15)
        assert w.ui_from_li(w.li_from_ui(v["ui"])) == sorted(v["ui"], reverse=True)
        assert w.jacobian_reverse(v["vi"]) == 1.0
    train = warpers.WarperTrainT()
    assert train.size() == 0 and train.map_reverse([0.3, 0.1]) == ([0.3, 0.1], 1.0)
    train.emplace_back(warpers.WarperPlasmaUvT(10.0))
    train.emplace_back(warpers.make_product_1d_simple_exponential(10.0, 1.5))
    x = [0.2, 0.7, 0.4]
    ui, jac = train.map_reverse(x)
    uo, jo = oracle.warp([(1, 10.0, 0.0), (2, 10.0, 1.5)], np.array([x]))
    np.testing.assert_allclose(ui, uo[0], rtol=1e-13)
    assert abs(jac / jo[0] - 1) < 1e-13
    ui1, j1 = train.map_reverse(x, 1, 0)
    assert ui1 == warpers.WarperPlasmaUvT(10.0).ui_from_li(x) and j1 == 1.0
    p = warpers.make_product_1d_simple_inverse_power(3, 10.0, 1.5)
    assert abs(p.jacobian_forward([2.0, 4.0]) / p.jacobian_forward([3.0, 4.0]) - ((3 + 1.5) / (2 + 1.5)) ** 3) < 1e-14


def _model(golden, alpha=0.0):
    return io.G0Model.from_tables(10.0, golden["table_beta20_lesser"], golden["table_beta20_greater"], alpha)


def test_g0_contour_and_integrand(oracle, golden):
    g0k = io.G0KeldyshContourT(_model(golden, 0.8))
    om = oracle.model(10.0, golden["table_beta20_lesser"], golden["table_beta20_greater"], 0.8)
    a, b = io.GfIndexT(3.0, 0, 0, 1), io.GfIndexT(1.5, 0, 1, 0)
    assert g0k(a, b) == oracle.g0(om, (3.0, 0, 0, 1, 0), (1.5, 0, 1, 0, 0))
    assert g0k(a, a, False) == oracle.g0(om, (3.0, 0, 0, 1, 0), (3.0, 0, 0, 1, 0), False)
    assert g0k.get_time_max() == 10.0
    for ename, A, B in EXTERNALS:
        f = io.IntegrandGDirect(g0k, io.GfIndexT(*A[:3]), io.GfIndexT(*B[:3]), 0.0)
        key = f"integrand_beta20_a0.8_{ename}_n4"
        t = golden[key + "_t"]
        _, _, sc = oracle.integrand(om, A, B, t)
        for i in range(len(t)):
            v, d = f(list(t[i]))
            assert d == golden[key + "_d"][i] and abs(v - golden[key + "_v"][i]) <= 1e-12 * sc[i] + 1e-300
        vb, db = f.evaluate_batch(t)
        assert np.all(np.abs(vb - golden[key + "_v"]) <= 1e-12 * sc + 1e-300)
        k2 = f"integrand_beta20_a0.8_{ename}_n2"
        nd = [f.eval_no_det(list(x))[0] for x in golden[k2 + "_t"]]
        np.testing.assert_allclose(nd, golden[k2 + "_nodet"], rtol=1e-13, atol=1e-16)
    with pytest.raises(RuntimeError, match="negative time"):
        io.IntegrandGDirect(g0k, io.GfIndexT(-1.0, 0, 0), io.GfIndexT(1.0, 0, 1), 0.0)


def test_charge_series_through_compute_charge_q_direct(keldy_tests):
    """keldy's compute_obs_test.cpp:93-136, written as a keldy user writes it."""
    p = keldy_tests["hz_params"]
    hz = keldy_tests["hz_charge_series"]
    params = {"beta": -1.0, "bias_V": 0.0, "eps_d": 0.0, "Gamma": 1.0, "time_max": 30.0,
              "nr_time_points_gf": 10001, "alpha": 0.0, "bath_type": "flatband", "ft_method": "analytic"}
    model = io.G0Model(params, False)
    t = p["t"]
    i_n = [1, 1j, -1, -1j]
    for order in range(1, 7):
        computer = io.ComputeChargeQDirect(model, t, order, 0.0)
        computer.warper.emplace_back(warpers.WarperPlasmaUvT(t))
        computer.warper.emplace_back(warpers.make_product_1d_simple_inverse_square(t, 1.0))
        computer.run(5000)
        computer.run(5000)
        assert computer.reduce_nr_points_run() == 10000
        q = -1j * i_n[order % 4] * computer.reduce_result()
        tol = 1e-3 if order < 5 else 1e-2
        assert abs(q - hz[order]) <= tol * abs(hz[order]), (order, q, hz[order])


def test_current_known_answer(keldy_tests):
    """keldy's compute_obs_test.cpp:183-206: order-1 current through a semicircular bath
    at zero temperature, dot-lead blocks of the g0 tables."""
    c = keldy_tests["current_kat"]
    p = dict(c["params"])
    p["nr_time_points_gf"] = int(p["nr_time_points_gf"])
    computer = io.ComputeCurrentJDirect(p, c["t_max"], 1, 0.0)
    computer.warper.emplace_back(warpers.WarperPlasmaUvT(c["t_max"]))
    computer.warper.emplace_back(warpers.make_product_1d_simple_inverse_square(c["t_max"], c["w_scale"]))
    computer.run(c["n_points"])
    value = -2 * (1j * computer.reduce_result()).real
    assert abs(value - c["value"]) < c["tol"], value


def test_integrator_rng_and_single_points(oracle, golden):
    model = _model(golden)
    om = oracle.model(10.0, golden["table_beta20_lesser"], golden["table_beta20_greater"])
    comp = io.ComputeChargeQDirect(model, 10.0, 3, 0.0)
    comp.warper.emplace_back(warpers.WarperPlasmaUvT(10.0))
    comp.warper.emplace_back(warpers.make_product_1d_simple_exponential(10.0, 1.0))
    chain = [(1, 10.0, 0.0), (2, 10.0, 1.0)]
    li = [0.3, 0.6, 0.2]
    v, d = comp.evaluate_warped_integrand(li)
    w, _, dw, sc = oracle.evaluate_warped(om, EXTERNALS[0][1], EXTERNALS[0][2], chain, np.array([li]))
    assert d == dw[0] and abs(v - w[0]) <= 1e-12 * sc[0]
    comp.reset_rng("sobol", 0, True, True, 9)
    comp.run(2000)
    s, npts, ndom, sc = oracle.integrate(om, EXTERNALS[0][1], EXTERNALS[0][2], chain, 3, 2000, do_shift=True,
                                         do_scramble=True, seed_shift=9)
    assert comp.reduce_nr_points_run() == npts and comp.reduce_nr_points_in_domain() == ndom
    assert abs(comp.reduce_result() * npts - s) <= 1e-12 * sc
    with pytest.raises(RuntimeError, match="no device form"):
        comp.reset_rng("mt19937_64", 0)
    with pytest.raises(RuntimeError, match="Dimension"):
        io.ComputeChargeQDirect(model, 10.0, 0, 0.0)
    assert comp.get_warper().size() == 2
