"""The kernel-method oracle (oracle/keldy_oracle.c: or_integrand_kernel) against the
closed forms of keldy's own tests (test/c++/impurity_oneband/wick_kernel_test.cpp:26-107):
order 1 and order 2, per (vertex, Keldysh index) as keldy compares them."""
import numpy as np
import pytest

from keldy_b200.g0_tables import flatband

UP, DOWN, FWD, BWD = 0, 1, 0, 1


@pytest.fixture(scope="module")
def model(oracle):
    _, le, gr = flatband(1.0, 0.2, 0.3, 20.0, 10.0, 4001)
    return oracle.model(10.0, le, gr, 0.0)


def _g(oracle, model, a, b):
    """g0_keldysh_contour_t(a, b) with internal = true: a, b = (time, spin, k_idx[, timesplit])."""
    return oracle.g0(model, tuple(a) + (0,) * (5 - len(a)), tuple(b) + (0,) * (5 - len(b)), True)


def test_order_1(oracle, model):
    X = (5.0, UP, FWD)
    u = 2.0
    g = lambda a, b: _g(oracle, model, a, b)
    want = {FWD: -g((u, UP, FWD), X) * g((u, DOWN, FWD), (u, DOWN, BWD)),
            BWD: g((u, UP, BWD), X) * g((u, DOWN, FWD), (u, DOWN, BWD))}
    vals, dom, _ = oracle.integrand_kernel(model, X + (0, 0), [[u]])
    assert dom[0] == 1
    for k in (FWD, BWD):
        assert abs(vals[0, 0, k] - want[k]) < 1e-15


def test_order_2(oracle, model):
    X = (5.0, UP, FWD)
    u, v = 2.0, 4.0
    g = lambda a, b: _g(oracle, model, a, b)

    def det_down(a, b):
        return (g((u, DOWN, FWD), (u, DOWN, BWD)) * g((v, DOWN, FWD), (v, DOWN, BWD))
                - g((v, DOWN, b), (u, DOWN, a)) * g((u, DOWN, a), (v, DOWN, b)))

    def det_prod_u(a, b):
        sign = 1 if a == b else -1
        return sign * (g((u, UP, a), (v, UP, b)) * g((v, UP, b), X) * det_down(a, b)
                       + g((v, UP, FWD), (v, UP, BWD)) * g((u, UP, a), X) * g((v, DOWN, b), (u, DOWN, a))
                       * g((u, DOWN, a), (v, DOWN, b)))

    def det_prod_v(a, b):
        sign = 1 if a == b else -1
        return -sign * (-g((v, UP, b), (u, UP, a)) * g((u, UP, a), X) * det_down(a, b)
                        - g((u, UP, FWD), (u, UP, BWD)) * g((v, UP, b), X) * g((v, DOWN, b), (u, DOWN, a))
                        * g((u, DOWN, a), (v, DOWN, b)))

    vals, dom, _ = oracle.integrand_kernel(model, X + (0, 0), [[u, v]])
    for k in (FWD, BWD):
        assert abs(vals[0, 0, k] - (det_prod_u(k, FWD) + det_prod_u(k, BWD))) < 1e-15
        assert abs(vals[0, 1, k] - (det_prod_v(FWD, k) + det_prod_v(BWD, k))) < 1e-15


def test_negative_time_is_out_of_domain(oracle, model):
    vals, dom, _ = oracle.integrand_kernel(model, (5.0, UP, FWD, 0, 0), [[2.0, -1.0]])
    assert dom[0] == 0 and np.all(vals == 0)
