"""Host g0 table builder against keldy's model known answers and its analytic formula."""
import math

import numpy as np
import pytest

from keldy_b200 import g0_tables


def _at(t, g, x):
    i = int(np.argmin(np.abs(t - x)))
    assert abs(t[i] - x) < 1e-12
    return g[i]


def test_flatband_zero_temperature_equals_keldy_analytic():
    t, a_l, a_g = g0_tables.flatband_analytic(1.0, 20.0, 4001)
    _, b_l, b_g = g0_tables.flatband(1.0, 0.0, 0.0, math.inf, 20.0, 4001)
    assert np.abs(a_l - b_l).max() < 1e-12 and np.abs(a_g - b_g).max() < 1e-12


def test_flatband_asymmetric_known_answers(keldy_tests):
    # model_flatband_test.cpp:154-220 ("value from Marjan analytic formula", tol 1e-7)
    for case in keldy_tests["flatband_kat"]:
        p = case["params"]
        beta = math.inf if p["beta"] < 0 else p["beta"]
        t, gl, gg = g0_tables.flatband(p["Gamma"], p["eps_d"], p["bias_V"], beta, p["time_max"],
                                       int(p["nr_time_points_gf"]))
        for v in case["values"]:
            assert abs(_at(t, gl, v["t"]) - complex(v["re"], v["im"])) < v["tol"]


def test_semicircle_known_answers(keldy_tests):
    # model_semicircle_test.cpp:30-86 (values from another code; keldy's tolerance 1e-3)
    p = keldy_tests["semicircle_kat"][1]["params"]
    t, gl, gg, l10, g10, l01, g01 = g0_tables.semicircle(p["Gamma"], p["eps_d"], p["bias_V"], p["beta"],
                                                         p["half_bandwidth"], p["time_max"], 2001, dot_lead=True)
    blocks = {(0, 0): gl, (0, 1): l01, (1, 0): l10}
    for v in keldy_tests["semicircle_kat"][1]["values"]:
        assert abs(_at(t, blocks[(v["o1"], v["o2"])], v["t"]) - complex(v["re"], v["im"])) < v["tol"]
    # t <-> -t symmetry checked by keldy at 1e-8
    i = int(np.argmin(np.abs(t - 1.0)))
    j = len(t) - 1 - i
    assert abs(gl[i] + np.conj(gl[j])) < 1e-12 and abs(l01[i] + np.conj(l10[j])) < 1e-12


@pytest.mark.parametrize("args", [(1.0, 0.3, 0.4, 20.0), (1.5, -1.0, 2.0, 10.0), (0.7, 0.0, 0.0, 200.0)])
def test_flatband_structure(args):
    gamma, eps, V, beta = args
    t, gl, gg = g0_tables.flatband(gamma, eps, V, beta, 10.0, 2001)
    mid = len(t) // 2
    # g^<(0) = i n, g^>(0) = -i (1 - n) with 0 < n < 1, anti-hermitian in time
    n = gl[mid].imag
    assert 0 < n < 1 and abs(gl[mid].real) < 1e-14 and abs(gg[mid] + 1j * (1 - n)) < 1e-12
    assert np.abs(gl + np.conj(gl[::-1])).max() < 1e-14
    # the retarded function is causal: g^R(t) = g^>(t) - g^<(t) = -i e^{-i eps t - gamma t} for t > 0
    tp = t[mid + 1:]
    gr = gg[mid + 1:] - gl[mid + 1:]
    assert np.abs(gr - (-1j) * np.exp(-1j * eps * tp - gamma * tp)).max() < 1e-10
