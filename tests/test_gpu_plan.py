"""Plans (one CUDA-graph launch per run of a fixed batch) and the launch-shape autotuner."""
import os

import numpy as np
import pytest

from keldy_b200 import autotune, capi
from keldy_b200.g0_tables import flatband

pytestmark = pytest.mark.gpu

CHAIN = [(capi.WARPER_PLASMA_UV, 20.0, 0.0), (capi.WARPER_EXPONENTIAL, 20.0, 1.0)]


@pytest.fixture(scope="module")
def model(ctx):
    _, le, gr = flatband(1.0, 0.0, 0.0, 50.0, 20.0, 40001)
    return ctx.model(20.0, le, gr)


def _items(ctx, model):
    return [dict(model=model, rng=ctx.sobol(n), chain=CHAIN, A=(20.0, 0, 0), B=(20.0, 0, 1), order=n, k_first=1 + n,
                 n_points=5000 + 77 * n) for n in range(1, 11)]


def test_plan_equals_integrate_and_replays(ctx, model):
    items = _items(ctx, model)
    want = capi.integrate(ctx, items)
    plan = capi.Plan(ctx, items)
    assert plan.run() == want
    assert plan.run() == want  # graph replay
    # advance one item's Sobol block without rebuilding the plan
    plan.set_k_first(3, 1 + 100000)
    got = plan.run()
    again = capi.integrate(ctx, [dict(items[3], k_first=1 + 100000)])
    assert got[3] == again[0] and got[:3] == want[:3]
    with pytest.raises(capi.KbError):
        plan.set_k_first(0, (1 << 31) - 10)  # past the end of the generator
    plan.close()


def _scale(it):
    li = it["rng"].points(it["k_first"], it["n_points"])
    v, _, _ = it["model"].evaluate_warped(it["A"], it["B"], it["chain"], li)
    return np.abs(v).sum()


def test_launch_shape_keeps_results(ctx, model):
    items = _items(ctx, model)[4:7]
    base = capi.integrate(ctx, items)
    scale = [_scale(it) for it in items]
    ctx.set_launch(-1, 32, 1)
    try:
        other = capi.integrate(ctx, items)
    finally:
        ctx.set_launch(-1, 128, 2)
    for (a, n, d, _), (b, m, e, _), sc in zip(base, other, scale):
        assert (n, d) == (m, e) and abs(a - b) <= 1e-12 * sc


def test_autotune_small(ctx, tmp_path):
    os.environ["KELDY_B200_CACHE"] = str(tmp_path)
    table = autotune.tune(ctx, orders=(2, 8), chunks=(64, 128), ctas=(1, 2), repeats=1, points=4096)
    assert set(table) == {2, 8}
    for v in table.values():
        assert v["chunk_points"] in (64, 128) and v["ctas_per_sm"] in (1, 2) and v["ms"] > 0
    autotune.apply(ctx, table)
    assert ctx.get_launch(8)[0] == table[8]["chunk_points"]
    ctx.set_launch(-1, 128, 2)
