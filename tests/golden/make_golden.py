"""Generates tests/golden/golden.npz and tests/golden/keldy_tests.json.

Run in a checkout that has keldy's sources (KELDY_SRC, default: a checkout named
`reference` beside the repository) and a built oracle/_ref (``make -C oracle``):

    python tests/golden/make_golden.py

* golden.npz: outputs of keldy's own code (digitalseq_b2g.hpp, the warper headers and
  wick_direct.cpp, compiled by oracle/Makefile) on seeded inputs: Sobol points, warper
  chains, tabulated (interp-nearest) warpers, integrand values (two g0 tables, several external-point pairs, orders 0-6),
  eval_no_det values and the integrator's sums.
* keldy_tests.json: known answers read from keldy's test files: the Horvatic-Zlatic
  charge series and its parameters and the order-1 current
  (test/c++/impurity_oneband/compute_obs_test.cpp), the order-2 kernel-method G(t) bins
  (compute_obs_kernel_test.cpp), the projection warper's values
  (test/c++/warpers/projection_test.cpp), the plasma-warper vectors
  (test/c++/warpers/warper_plasma_uv_test.cpp), and g0 values of the semicircular and
  flat-band models (model_semicircle_test.cpp, model_flatband_test.cpp).

    python tests/golden/make_golden.py --json-only   # rewrite keldy_tests.json only
"""
from __future__ import annotations

import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.pyoracle import (Reference, W_EXPONENTIAL, W_IDENTITY, W_INVERSE, W_INVERSE_POWER,  # noqa: E402
                             W_INVERSE_SQUARE, W_PLASMA_UV, W_UNIFORM)
from keldy_b200.g0_tables import flatband, flatband_analytic  # noqa: E402

KELDY_SRC = os.environ.get("KELDY_SRC", os.path.join(os.path.dirname(ROOT), "reference"))

SOBOL_CASES = [  # (dim, seed, do_shift, do_scramble, seed_shift)
    (1, 0, 0, 0, 0), (3, 0, 0, 0, 0), (8, 0, 0, 0, 0), (12, 0, 0, 0, 0), (8, 1000, 0, 0, 0),
    (8, 0, 1, 0, 1), (8, 0, 0, 1, 2), (10, 0, 1, 1, 3), (16, 77, 1, 1, -4), (40, 0, 1, 1, 5),
]
SOBOL_COUNT = 96

CHAINS = {
    "plasma": [(W_PLASMA_UV, 20.0, 0.0)],
    "exponential": [(W_EXPONENTIAL, 20.0, 1.0)],
    "plasma_exponential": [(W_PLASMA_UV, 20.0, 0.0), (W_EXPONENTIAL, 20.0, 1.0)],
    "plasma_inverse_square": [(W_PLASMA_UV, 20.0, 0.0), (W_INVERSE_SQUARE, 20.0, 1.0)],
    "inverse": [(W_INVERSE, 10.0, 1.5)],
    "inverse_power3": [(W_INVERSE_POWER, 10.0, 1.5, 3)],
    "uniform": [(W_UNIFORM, 10.0, 0.0)],
    "identity": [(W_IDENTITY, 0.0, 0.0)],
    "inverse_exponential": [(W_INVERSE, 10.0, 1.0), (W_EXPONENTIAL, 1.0, 1.0)],
}

# (name, A, B): gf_index tuples (time, spin, k_idx, timesplit, orbital)
EXTERNALS = [
    ("charge", (10.0, 0, 0, 0, 0), (10.0, 0, 1, 0, 0)),
    ("ab", (4.0, 0, 0, 0, 0), (5.0, 0, 0, 0, 0)),
    ("down_bwd", (7.5, 1, 1, 0, 0), (2.0, 1, 0, 0, 0)),
]


def keldy_test_values():
    src = open(os.path.join(KELDY_SRC, "test/c++/impurity_oneband/compute_obs_test.cpp")).read()
    m = re.search(r"HZ_charge_series = \{([^}]*)\}", src)
    hz = [float(x) for x in m.group(1).replace("\n", " ").split(",")]
    pl = open(os.path.join(KELDY_SRC, "test/c++/warpers/warper_plasma_uv_test.cpp")).read()
    vecs = []
    for block in re.findall(r"TEST\(ViUiMaps, \w+\).*?\n}\n", pl, re.S):
        t_max = float(re.search(r"t_max = ([\d.]+)", block).group(1))
        ui = [float(x) for x in re.search(r"ui_times = \{([^}]*)\}", block).group(1).split(",")]
        vi = [float(x) for x in re.search(r"vi_result = \{([^}]*)\}", block).group(1).split(",")]
        vecs.append({"t_max": t_max, "ui": ui, "vi": vi})
    def params_of(block, names=None):
        out = {}
        for k, v in re.findall(r"params\.(\w+) = ([^;]+);", block):
            v = v.strip()
            out[k] = v.strip('"') if v.startswith('"') else (names[v] if names and v in names else float(v))
        return out

    def test_block(text, name):
        return re.search(r"TEST\(" + name + r"\).*?\n}\n", text, re.S).group(0)

    cur = test_block(src, r"ComputeObs, ValueCurrent1")
    current = {"params": params_of(cur),
               "t_max": float(re.search(r"double t_max = ([\d.]+);", cur).group(1)),
               "w_scale": float(re.search(r"make_product_1d_simple_inverse_square\(t_max, ([\d.]+)\)", cur).group(1)),
               "n_points": int(float(re.search(r"computer\.run\(([\de.]+)\)", cur).group(1))),
               "value": float(re.search(r"EXPECT_NEAR\([^,]+, ([\d.e-]+), ([\d.e-]+)\)", cur).group(1)),
               "tol": float(re.search(r"EXPECT_NEAR\([^,]+, ([\d.e-]+), ([\d.e-]+)\)", cur).group(2))}
    sc = open(os.path.join(KELDY_SRC, "test/c++/impurity_oneband/model_semicircle_test.cpp")).read()
    semi = []
    for name in ("g0_model, Semicirc_fft", "g0_model, Semicirc_contour"):
        blk = test_block(sc, name)
        vals = re.findall(r"EXPECT_COMPLEX_NEAR\(([-\d.e]+) \+ ([-\d.e]+)i, g0\.g0_lesser\[up\]\(([\d.]+)\)\((\d), (\d)\), "
                          r"([\d.e-]+)\)", blk)
        semi.append({"params": params_of(blk), "values": [
            {"re": float(a), "im": float(b), "t": float(t), "o1": int(i), "o2": int(j), "tol": float(tol)}
            for a, b, t, i, j, tol in vals]})
    fb = open(os.path.join(KELDY_SRC, "test/c++/impurity_oneband/model_flatband_test.cpp")).read()
    flat = []
    for name in ("g0_model, Flatband_asym_1", "g0_model, Flatband_asym_2"):
        blk = test_block(fb, name)
        first = blk.split("g0_model g0_ctr")[0]
        vals = re.findall(r"EXPECT_COMPLEX_NEAR\(([-\d.e]+) \+ ([-\d.e]+)i, g0_ctr\.g0_lesser\[up\]\(([\d.]+)\)\(0, 0\), "
                          r"([\d.e-]+)\)", blk)
        p = params_of(first)
        p.update(params_of(blk.split("g0_model g0_fft")[1]))  # the contour run's parameters
        flat.append({"params": p, "values": [{"re": float(a), "im": float(b), "t": float(t), "tol": float(tol)}
                                             for a, b, t, tol in vals]})
    # the same tests' fft runs (first part of Flatband_asym_1/2, Flatband_3) and Flatband_sym
    flat_fft = []
    for name in ("g0_model, Flatband_asym_1", "g0_model, Flatband_asym_2", "g0_model, Flatband_3"):
        blk = test_block(fb, name)
        first = blk.split("g0_model g0_ctr")[0] if "g0_model g0_ctr" in blk else blk
        first = first.split("params.bath_type = \"flatband\";\n  params.ft_method = \"contour\"")[0]
        vals = re.findall(r"EXPECT_COMPLEX_NEAR\(([-\d.e]+) \+ ([-\d.e]+)i, g0(?:_fft)?\.g0_lesser\[up\]\(([\d.]+)\)"
                          r"\(0, 0\), ([\d.e-]+)\)", first)
        sym = re.findall(r"EXPECT_COMPLEX_NEAR\(g0_fft\.g0_(lesser|greater)\[up\]\(([\d.]+)\)\(0, 0\), "
                         r"-std::conj\(g0_fft\.g0_\w+\[up\]\(-[\d.]+\)\(0, 0\)\), ([\d.e-]+)\)", first)
        flat_fft.append({"test": name.split(", ")[1], "params": params_of(blk.split("g0_model g0_fft")[0]),
                         "values": [{"re": float(a), "im": float(b), "t": float(t), "tol": float(tol)}
                                    for a, b, t, tol in vals],
                         "symmetry": [{"function": f, "t": float(t), "tol": float(tol)} for f, t, tol in sym]})
    sb = test_block(fb, "g0_model, Flatband_sym")
    grid = re.search(r"for \(size_t i = 0; i <= (\d+); \+\+i\) \{\s*time = ([-\d.]+) \+ i \* ([\d.]+);", sb)
    flat_sym = {"params": params_of(sb), "n_times": int(grid.group(1)) + 1, "t0": float(grid.group(2)),
                "dt": float(grid.group(3)),
                "tol": float(re.search(r"g0\.g0_lesser\[up\]\(time\)\(0, 0\), ([\d.e-]+)\)", sb).group(1))}
    kt = open(os.path.join(KELDY_SRC, "test/c++/impurity_oneband/compute_obs_kernel_test.cpp")).read()
    kb = test_block(kt, r"ComputeObs, ValueKernel")
    kvals = re.findall(r"\{([-\d.e]+) ([+-]) ([\d.e-]+)i, ([-\d.e]+) ([+-]) ([\d.e-]+)i\}", kb)
    ktmax = float(re.search(r"double const tmax = ([\d.]+);", kb).group(1))
    kernel = {"params": params_of(kb, {"tmax": ktmax}),
              "t_max": ktmax,
              "order": int(re.search(r"compute_gf_kernel computer\(g0, tmax, (\d+), nr_bins\)", kb).group(1)),
              "nr_bins": int(re.search(r"int const nr_bins = (\d+);", kb).group(1)),
              "n_points": int(float(re.search(r"computer\.run\(([\de.]+)\)", kb).group(1))),
              "tol": float(re.search(r"EXPECT_LT\(max_element\(abs\(result - expected_result\)\), ([\de.-]+)\)",
                                     kb).group(1)),
              "expected": [[[float(a), float(b + c)], [float(d), float(e + f)]] for a, b, c, d, e, f in kvals]}
    pt = open(os.path.join(KELDY_SRC, "test/c++/warpers/projection_test.cpp")).read()
    pb = test_block(pt, r"ProjectionWarper, Values")
    pargs = re.search(r"warper_projection_t\(warped_integrand, (\d+), int\(([\de.]+)\), int\(([\de.]+)\), "
                      r"([\d.]+), (true|false)\)", pb)
    projection = {
        "t_max": float(re.search(r"double const tmax = ([\d.]+);", pb).group(1)),
        "tol": float(re.search(r"double const tol = ([\de.-]+);", pb).group(1)),
        "interp_points": int(re.search(r"warper = \{cst, tmax, (\d+)\}", pb).group(1)),
        "order": int(pargs.group(1)), "num_bins": int(float(pargs.group(2))),
        "nr_samples": int(float(pargs.group(3))), "sigma": float(pargs.group(4)),
        "optimize_sigma": pargs.group(5) == "true",
        "values": [{"method": m, "x": float(x), "value": float(v)} for m, x, v in
                   re.findall(r"EXPECT_NEAR\(proj_warper\.(\w+)\(\{([\d.]+)\}\)(?:\[0\])?, ([\d.]+), tol\)", pb)],
    }
    return {
        "source": "keldy test/c++/impurity_oneband/compute_obs_test.cpp:93-206, "
                  "test/c++/impurity_oneband/compute_obs_kernel_test.cpp:12-60, "
                  "test/c++/warpers/warper_plasma_uv_test.cpp:15-43, "
                  "test/c++/impurity_oneband/model_semicircle_test.cpp:30-86, "
                  "test/c++/impurity_oneband/model_flatband_test.cpp:60-269, "
                  "test/c++/warpers/projection_test.cpp:70-103",
        "current_kat": current,
        "semicircle_kat": semi,
        "flatband_kat": flat,
        "flatband_fft_kat": flat_fft,
        "flatband_sym_kat": flat_sym,
        "hz_charge_series": hz,
        "hz_params": {"beta": "inf", "bias_V": 0.0, "eps_d": 0.0, "Gamma": 1.0, "time_max": 30.0,
                      "nr_time_points_gf": 10001, "alpha": 0.0, "bath_type": "flatband", "ft_method": "analytic",
                      "t": 20.0, "orders": [1, 6],
                      "runs": [{"warper": "inverse_square", "w": 1.0, "n_points": 10000, "rtol": [1e-3, 1e-2]},
                               {"warper": "exponential", "w": 2.0, "n_points": 50000, "rtol": [1e-2, 1e-2]}]},
        "plasma_vectors": vecs,
        "kernel_kat": kernel,
        "projection_kat": projection,
    }


def main():
    if "--json-only" in sys.argv:
        values = keldy_test_values()
        with open(os.path.join(HERE, "keldy_tests.json"), "w") as f:
            json.dump(values, f, indent=1)
        return
    ref = Reference()
    rng = np.random.default_rng(20240601)
    out = {}
    # Sobol
    for i, (dim, seed, sh, sc, ss) in enumerate(SOBOL_CASES):
        out[f"sobol_{i}"] = ref.sobol_points(dim, seed, SOBOL_COUNT, bool(sh), bool(sc), ss)
    out["sobol_cases"] = np.array(SOBOL_CASES, dtype=np.int64)
    # warpers
    for name, chain in CHAINS.items():
        x = rng.random((64, 6))
        u, j = ref.warp(chain, x, "reverse")
        out[f"warp_{name}_li"] = x
        out[f"warp_{name}_ui"] = u
        out[f"warp_{name}_jr"] = j
        y = np.abs(u) + 0.05 if name not in ("identity",) else x
        y = np.minimum(y, 9.5)
        lf, jf = ref.warp(chain, y, "forward")
        out[f"warp_{name}_fin"] = y
        out[f"warp_{name}_fout"] = lf
        out[f"warp_{name}_jf"] = jf
    # g0 tables: zero-temperature analytic and finite beta, t in [-10, 10]
    _, l0, g0 = flatband_analytic(1.0, 10.0, 2001)
    _, l1, g1 = flatband(1.0, 0.3, 0.4, 20.0, 10.0, 2001)
    out["table_T0_lesser"], out["table_T0_greater"] = l0, g0
    out["table_beta20_lesser"], out["table_beta20_greater"] = l1, g1
    for tname, (le, gr) in {"T0": (l0, g0), "beta20": (l1, g1)}.items():
        for alpha in (0.0, 0.8):
            model = ref.model(10.0, le, gr, alpha)
            for ename, A, B in EXTERNALS:
                for n in range(0, 7):
                    t = rng.random((24, n)) * 10.0
                    if n >= 2:
                        t[0, 1] = t[0, 0]            # equal vertex times
                        t[1, 0] = -0.5               # out of the domain
                        t[2, :] = np.sort(t[2, :])[::-1]
                    if n >= 1:
                        t[3, 0] = A[0]               # vertex at an external time
                    key = f"integrand_{tname}_a{alpha}_{ename}_n{n}"
                    vals, dom = ref.integrand(model, A, B, t)
                    out[key + "_t"] = t
                    out[key + "_v"] = vals
                    out[key + "_d"] = dom
                    if n <= 2:
                        nv, nd = ref.integrand(model, A, B, t, no_det=True)
                        out[key + "_nodet"] = nv
    # integrator sums (keldy's loop, sobol_unshifted seed 0)
    model = ref.model(10.0, l1, g1, 0.0)
    for n in (1, 2, 3, 4):
        for cname in ("plasma_exponential", "uniform"):
            chain = [(W_PLASMA_UV, 10.0, 0.0), (W_EXPONENTIAL, 10.0, 1.0)] if cname == "plasma_exponential" \
                else [(W_UNIFORM, 10.0, 0.0)]
            s, npts, ndom = ref.integrate(model, EXTERNALS[0][1], EXTERNALS[0][2], chain, n, 4096)
            out[f"integrate_{cname}_n{n}"] = np.array([s.real, s.imag, npts, ndom])
    # tabulated warpers (warper_product_1d_simple_interp_nearest_t): random positive f1,
    # f1 with a zero tail (the inverse's cut), keldy's f1 = exp(-u/2) on 1000 points
    tables = []
    for k in range(3):
        n = int(rng.integers(5, 40))
        u = np.concatenate([[0.0], np.cumsum(rng.random(n - 1) + 0.05)])
        f1 = rng.random(n) + 0.1
        if k == 1:
            f1[-4:] = 0.0
        tables.append((u, f1))
    u = np.array([i / 999 * 5.0 for i in range(1000)])
    u[-1] = 5.0
    tables.append((u, np.exp(-u / 2.0)))
    for k, (u, f1) in enumerate(tables):
        x = rng.random((48, 3))
        x[0] = [0.0, 1.0, 0.5]
        ur, jr = ref.interp_nearest(u, f1, x, "reverse")
        y = np.clip(ur, u[0], u[-1])
        lf, jf = ref.interp_nearest(u, f1, y, "forward")
        for key, val in (("u", u), ("f1", f1), ("li", x), ("ui", ur), ("jr", jr), ("fin", y), ("fout", lf),
                         ("jf", jf)):
            out[f"interp_{k}_{key}"] = val
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **out)
    with open(os.path.join(HERE, "keldy_tests.json"), "w") as f:
        json.dump(keldy_test_values(), f, indent=1)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    main()
