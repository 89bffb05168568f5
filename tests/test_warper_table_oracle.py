"""The tabulated-warper oracle (oracle/warper_table_oracle.py) against the closed forms
of keldy's own tests (test/c++/warpers/product_1d_simple_interp_test.cpp:14-75) and the
smoothing against a direct weighted fit."""
import math

import numpy as np

from oracle import warper_table_oracle as wt


def test_constant_f1_is_linear():
    t_max = 1.5
    for u in (np.linspace(0, t_max, 8), np.array([0.0, 0.5, 0.75, 1.0, t_max])):
        t = wt.table(u, np.ones(len(u)))
        for l in (0.0, 0.2, 0.5, 0.999, 1.0):
            uu, jac = wt.reverse(t, l)
            assert abs((t_max - uu) / t_max - l) < 1e-10 and abs(jac - t_max) < 1e-10
            ll, f = wt.forward(t, uu)
            assert abs(ll - l) < 1e-10 and abs(f * t_max - 1) < 1e-10


def test_exponential_f1():
    t_max = 5.0
    u = np.array([i / 999 * t_max for i in range(1000)])
    u[-1] = t_max
    t = wt.table(u, np.exp(-u / 2))
    for x in np.linspace(0, t_max, 37):
        l, _ = wt.forward(t, x)
        want = (math.exp(-t_max / 2) - math.exp(-x / 2)) / math.expm1(-t_max / 2)
        assert abs(l - want) < 1e-6


def test_kernel_smoothing_recovers_an_exponential():
    y = np.exp(-0.03 * np.arange(200))
    assert np.allclose(wt.kernel_smoothing(y, 5.0), y, rtol=1e-12)
    y2 = y.copy()
    y2[50] = 0.0  # a dead point is left out of every fit
    assert np.allclose(wt.kernel_smoothing(y2, 5.0), y, rtol=1e-12)
