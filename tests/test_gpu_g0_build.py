"""g0 tables built on the GPU (kb_models_set_flatband) against the host builder
(g0_tables.flatband) and keldy's flat-band known answers."""
import math

import numpy as np
import pytest

from keldy_b200 import capi, g0_tables

pytestmark = pytest.mark.gpu

CASES = [  # (Gamma, eps_d, V, beta)
    (1.0, 0.0, 0.0, 50.0), (1.0, 0.5, 1.0, 100.0), (1.0, 0.3, 0.4, 20.0), (1.5, -1.0, 2.0, 10.0),
    (0.7, 0.0, 0.0, 200.0), (1.0, 0.0, 0.0, math.inf), (1.0, -0.5, 1.0, math.inf), (1.0, 0.25, 0.5, 10.0),
]


@pytest.mark.parametrize("time_max,npts", [(10.0, 2001), (20.0, 4001), (50.0, 10001)])
def test_gpu_builder_equals_host_builder(ctx, time_max, npts):
    models = capi.flatband_models(ctx, CASES, time_max, npts)
    for m, (g, e, v, b) in zip(models, CASES):
        _, hl, hg = g0_tables.flatband(g, e, v, b, time_max, npts)
        dl, dg = m.table()
        scale = max(np.abs(hl).max(), np.abs(hg).max())
        assert np.abs(dl - hl).max() <= 1e-11 * scale, (g, e, v, b, np.abs(dl - hl).max())
        assert np.abs(dg - hg).max() <= 1e-11 * scale, (g, e, v, b, np.abs(dg - hg).max())


def test_gpu_builder_known_answers(ctx, keldy_tests):
    # keldy's model_flatband_test.cpp:154-220 values (tol as in keldy)
    for case in keldy_tests["flatband_kat"]:
        p = case["params"]
        beta = math.inf if p["beta"] < 0 else p["beta"]
        npts = int(p["nr_time_points_gf"])
        npts += 1 - npts % 2
        m, = capi.flatband_models(ctx, [(p["Gamma"], p["eps_d"], p["bias_V"], beta)], p["time_max"], npts)
        gl, _ = m.table()
        t = g0_tables.time_mesh(p["time_max"], npts)
        for v in case["values"]:
            i = int(np.argmin(np.abs(t - v["t"])))
            assert abs(gl[i] - complex(v["re"], v["im"])) < v["tol"]


def test_gpu_built_model_integrates_like_uploaded(ctx):
    _, le, gr = g0_tables.flatband(1.0, 0.5, 1.0, 100.0, 10.0, 4001)
    up = ctx.model(10.0, le, gr)
    built, = capi.flatband_models(ctx, [(1.0, 0.5, 1.0, 100.0)], 10.0, 4001)
    chain = [(capi.WARPER_PLASMA_UV, 10.0, 0.0), (capi.WARPER_EXPONENTIAL, 10.0, 1.0)]
    rng = ctx.sobol(5)
    items = [dict(model=m, rng=rng, chain=chain, A=(10.0, 0, 0, 0, 0), B=(10.0, 0, 1, 0, 0), order=5,
                  n_points=20000) for m in (up, built)]
    (a, na, da, _), (b, nb, db, _) = capi.integrate(ctx, items)
    assert (na, da) == (nb, db)
    assert abs(a - b) <= 1e-9 * abs(a)


def test_builder_errors(ctx):
    with pytest.raises(capi.KbError):
        capi.flatband_models(ctx, [(1.0, 0.0, 0.0, 10.0)], 10.0, 2000)  # even mesh
    with pytest.raises(capi.KbError):
        capi.flatband_models(ctx, [(0.0, 0.0, 0.0, 10.0)], 10.0, 2001)  # Gamma = 0
