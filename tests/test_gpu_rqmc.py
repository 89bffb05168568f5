"""Randomised QMC error bars (R random digital shifts in one batched launch)."""
import numpy as np
import pytest

from keldy_b200 import capi, rqmc
from keldy_b200.g0_tables import flatband

pytestmark = pytest.mark.gpu


def test_replicas_and_unbiasedness(ctx):
    _, le, gr = flatband(1.0, 0.0, 0.0, 50.0, 20.0, 40001)
    m = ctx.model(20.0, le, gr)
    chain = [(capi.WARPER_PLASMA_UV, 20.0, 0.0), (capi.WARPER_EXPONENTIAL, 20.0, 1.0)]
    A, B = (20.0, 0, 0), (20.0, 0, 1)
    mean, err, means = rqmc.estimate(ctx, m, A, B, chain, 4, 1 << 14, replicas=8)
    # each replica equals a separate integrate call with that shifted generator
    for r in (0, 5):
        (s, n, _, _), = capi.integrate(ctx, [dict(model=m, rng=ctx.sobol(4, 31, True, False, 1 + r), chain=chain,
                                                  A=A, B=B, order=4, k_first=1, n_points=1 << 14)])
        assert s / n == means[r]
    # the shifted estimates agree with a long unshifted run within their error bar
    (s, n, _, _), = capi.integrate(ctx, [dict(model=m, rng=ctx.sobol(4), chain=chain, A=A, B=B, order=4,
                                              k_first=1, n_points=1 << 22)])
    assert abs(mean - s / n) < 5 * err + 1e-12
    res = rqmc.time_to_relative_error(ctx, m, A, B, chain, 2, target=1e-3, replicas=8, start_points=1 << 10)
    assert res["reached"] and res["rel"] <= 1e-3
