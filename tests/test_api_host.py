"""keldy's Python names on keldy_b200: the host-side logic (no GPU needed)."""
import math

import pytest

from keldy_b200 import common, impurity_oneband as io, warpers  # noqa: F401


def test_compare_3way_truth_table():
    # k_countour_pt.cpp:8-116
    C = common.ContourPtT
    for t in (-1.0, 0.0, 1.0):
        for s in (-1, 0, 1):
            for k in (0, 1):
                assert common.compare_3way(C(t, k, s), C(t, k, s)) == 0
    for t0 in (-2.0, 0.0, 2.0):
        for t1 in (-2.0, 0.0, 2.0):
            assert common.compare_3way(C(t0, 0, 1), C(t1, 1, -1)) < 0
            assert common.compare_3way(C(t1, 1, -1), C(t0, 0, 1)) > 0
    assert common.compare_3way(C(1.0, 0, 0), C(2.0, 0, 0)) < 0
    assert common.compare_3way(C(2.0, 1, 0), C(1.0, 1, 0)) < 0
    assert common.compare_3way(C(0.5, 0, 0), C(0.5, 0, 1)) < 0
    assert common.compare_3way(C(0.5, 1, 1), C(0.5, 1, 0)) < 0
    assert C(1.0, 0, 0) == C(1.0, 0, 0) and not (C(1.0, 0, 0) == C(1.0, 1, 0))


def test_model_param_t_defaults_and_keys():
    p = io.model_param_t()
    assert p["bath_type"] == "semicircle" and p["nr_time_points_gf"] == 1000 and p["ft_method"] == "fft"
    assert io.model_param_t({"beta": 5.0}, Gamma=2.0)["Gamma"] == 2.0
    with pytest.raises(KeyError):
        io.model_param_t({"betta": 1.0})


def test_g0_model_parameter_errors():
    # keldy's g0_model constructor errors (model.cpp:113-173, 428-436) come before any table
    with pytest.raises(RuntimeError, match="singular"):
        io.G0Model({"bath_type": "flatband"}, True)
    with pytest.raises(RuntimeError, match="Analytic flatband"):
        io.G0Model({"bath_type": "flatband", "ft_method": "analytic", "beta": 10.0})
    with pytest.raises(RuntimeError, match="only works for flatband"):
        io.G0Model({"bath_type": "semicircle", "ft_method": "analytic"})
    with pytest.raises(RuntimeError, match="bath_type not defined"):
        io.G0Model({"bath_type": "cubic"})
    with pytest.raises(RuntimeError, match="is not defined"):
        io.G0Model({"ft_method": "laplace"})


def test_product_warper_from_functions_has_no_device_form():
    with pytest.raises(RuntimeError, match="no device form"):
        warpers.WarperProduct1dSimpleT(lambda u: 1.0, lambda u: u, lambda l: l, 1.0)
