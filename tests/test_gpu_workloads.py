"""The measured workloads against the CPU checkers, so that every number the bench reports
is computed on a configuration whose sums are known to be keldy's.

* The order-8 throughput workload (flat-band dot at beta = 50, t = 20, g0 on 40,001
  points, chain [plasma_uv(20), exponential(20, 1)]) against keldy's own integrand
  compiled into oracle/_ref and against the C restatement, at the Sobol index the
  bench's first timed step starts from.
* Models of the 256-model sweep at the grid's beta, V and eps_d extremes, integrated
  inside the batched 256-item plan, against the C restatement on the tables the GPU
  built.
* Orders 10 and 12, point by point, on the biased dot (V = 1, eps_d = 0.5, beta = 100,
  t = 50) and on the sweep grid's corners: the tree's diagonal pivots with their guard
  give keldy's values at every point.

Tolerance (the integrand's alternating sum cancels): |gpu - cpu| <= 1e-12 * sum|f J|.
"""
import numpy as np
import pytest

import bench
from keldy_b200 import capi
from oracle.pyoracle import Reference, W_EXPONENTIAL, W_PLASMA_UV, reference_available

pytestmark = pytest.mark.gpu

CHAIN_20 = [(capi.WARPER_PLASMA_UV, 20.0, 0.0), (capi.WARPER_EXPONENTIAL, 20.0, 1.0)]
ORACLE_CHAIN_20 = [(W_PLASMA_UV, 20.0, 0.0), (W_EXPONENTIAL, 20.0, 1.0)]
A20, B20 = (20.0, 0, 0, 0, 0), (20.0, 0, 1, 0, 0)


def _bench_model(ctx, oracle):
    from keldy_b200.g0_tables import flatband
    _, le, gr = flatband(bench.GAMMA, bench.EPS_D, bench.BIAS, bench.BETA, bench.T_MAX, bench.NPTS)
    return le, gr, ctx.model(bench.T_MAX, le, gr), oracle.model(bench.T_MAX, le, gr)


@pytest.mark.parametrize("warmup", [0, 5])
def test_bench_workload_vs_keldy(ctx, oracle, warmup):
    """16,384 points of the bench's order-8 step from k_first = 1 + W * 2^20 (the first timed
    step after W warm-up steps on one GPU)."""
    assert (bench.T_MAX, bench.NPTS, bench.BETA) == (20.0, 40001, 50.0)
    le, gr, gm, om = _bench_model(ctx, oracle)
    n_pts, order = 1 << 14, 8
    k_first = 1 + warmup * (1 << 20)
    item = dict(model=gm, rng=ctx.sobol(order), chain=CHAIN_20, A=A20, B=B20, order=order, k_first=k_first,
                n_points=n_pts)
    (s, npts, nd, nfb), = capi.integrate(ctx, [item])
    w, onp, ond, sc = oracle.integrate(om, A20, B20, ORACLE_CHAIN_20, order, n_pts, seed=k_first - 1)
    assert (npts, nd) == (onp, ond) and nfb == 0
    assert abs(s - w) <= 1e-12 * sc, abs(s - w) / sc
    # the same sums through the plan the bench replays
    plan = capi.Plan(ctx, [item])
    (sp, npp, ndp, _), = plan.run()
    plan.close()
    assert (sp, npp, ndp) == (s, npts, nd)
    if reference_available():
        ref = Reference()
        rm = ref.model(bench.T_MAX, le, gr)
        r, rnp, rnd = ref.integrate(rm, A20, B20, ORACLE_CHAIN_20, order, n_pts, seed=k_first - 1, mode=1,
                                    threads=4)
        assert (rnp, rnd) == (npts, nd)
        assert abs(s - r) <= 1e-12 * sc, abs(s - r) / sc


# the sweep's grid (bench.measure_sweep): beta outer, V middle, eps_d inner, truncated to 256
SWEEP_PARAMS = [(1.0, e, v, b) for b in (10.0, 50.0, 200.0) for v in np.linspace(0.0, 2.0, 8)
                for e in np.linspace(-1.0, 1.0, 11)][:256]
# beta 10 / V 0 / eps_d -1; beta 10 / V 2 / eps_d 1; beta 200 / V 0 / eps_d 1; beta 200 / V 2 / eps_d -0.6
SWEEP_CHECKED = (0, 87, 186, 255)


def test_sweep_models_vs_oracle(ctx, oracle):
    """All 256 sweep models in one plan (2^10 points each, model i at order 2 + i % 9); the
    models at the grid's extremes against the oracle on the GPU-built tables."""
    models = capi.flatband_models(ctx, SWEEP_PARAMS, 20.0, 20001)
    rngs = {n: ctx.sobol(n) for n in range(2, 11)}
    n_pts = 1 << 10
    items = [dict(model=m, rng=rngs[2 + i % 9], chain=CHAIN_20, A=A20, B=B20, order=2 + i % 9, k_first=1,
                  n_points=n_pts) for i, m in enumerate(models)]
    plan = capi.Plan(ctx, items)
    res = plan.run()
    plan.close()
    assert len(res) == 256
    seen = set()
    for i in SWEEP_CHECKED:
        g, e, v, b = SWEEP_PARAMS[i]
        seen.add((b, v))
        le, gr = models[i].table()
        om = oracle.model(20.0, le, gr)
        w, onp, ond, sc = oracle.integrate(om, A20, B20, ORACLE_CHAIN_20, 2 + i % 9, n_pts)
        s, npts, nd, _ = res[i]
        assert (npts, nd) == (onp, ond), i
        assert abs(s - w) <= 1e-12 * sc, (i, abs(s - w) / sc)
    assert {10.0, 200.0} <= {b for b, _ in seen} and {0.0, 2.0} <= {v for _, v in seen}


# (Gamma, eps_d, V, beta): the biased dot and the corners of the sweep's grid
GUARD_MODELS = [(1.0, 0.5, 1.0, 100.0), (1.0, -1.0, 0.0, 10.0), (1.0, 1.0, 2.0, 200.0), (1.0, -1.0, 2.0, 200.0)]


@pytest.mark.parametrize("order,n_pts", [(10, 256), (12, 256)])
def test_high_order_pivot_guard_vs_oracle(ctx, oracle, order, n_pts):
    """Point values at orders 10 and 12 on the biased dot (t = 50, 100,001 points) and on the
    sweep grid's corners (t = 20, 20,001 points). The tree pivots on the diagonal and hands
    points with a pivot below 1e-8 max|g0| to keldy's partially pivoted LU; every point,
    guarded or not, equals the oracle, and the integration's sum (tree points plus the
    guarded points it counts as fallback) equals the sum of the point values."""
    for g, e, v, b in GUARD_MODELS:
        t = 50.0 if (e, v, b) == (0.5, 1.0, 100.0) else 20.0
        gm, = capi.flatband_models(ctx, [(g, e, v, b)], t, 100001 if t == 50.0 else 20001)
        le, gr = gm.table()
        om = oracle.model(t, le, gr)
        chain = [(capi.WARPER_PLASMA_UV, t, 0.0), (capi.WARPER_EXPONENTIAL, t, 1.0)]
        ochain = [(W_PLASMA_UV, t, 0.0), (W_EXPONENTIAL, t, 1.0)]
        A, B = (t, 0, 0, 0, 0), (t, 0, 1, 0, 0)
        rng = ctx.sobol(order)
        (s, npts, nd, nfb), = capi.integrate(ctx, [dict(model=gm, rng=rng, chain=chain, A=A, B=B, order=order,
                                                        k_first=1, n_points=n_pts)])
        w, onp, ond, sc = oracle.integrate(om, A, B, ochain, order, n_pts)
        assert (npts, nd) == (onp, ond) and 0 <= nfb <= nd
        assert abs(s - w) <= 1e-12 * sc, (g, e, v, b, abs(s - w) / sc)
        li = rng.points(1, n_pts)
        val, jac, dom = gm.evaluate_warped(A, B, chain, li)
        ov, ojac, odom, osc = oracle.evaluate_warped(om, A, B, ochain, li)
        assert np.array_equal(dom, odom)
        assert np.all(np.abs(val - ov) <= 1e-12 * osc), (g, e, v, b)
        assert abs(val.sum() - s) <= 1e-12 * osc.sum()
