"""The learned autoregressive spline flow on the GPU (kb_flow_create_kind(KB_FLOW_AR_SPLINE)):
its maps and the gradient of its training kernel against the CPU restatement
(oracle/ar_spline_flow_oracle.py, whose gradient is checked against finite differences),
its reduction to the separable spline flow, integration with the map applied in line, and
training warm-started from the separable flow."""
import math

import numpy as np
import pytest

from keldy_b200 import capi, learned
from keldy_b200.g0_tables import flatband
from oracle import ar_spline_flow_oracle as ar
from oracle import spline_flow_oracle as so

pytestmark = pytest.mark.gpu

PLASMA_EXP = [(capi.WARPER_PLASMA_UV, 10.0, 0.0), (capi.WARPER_EXPONENTIAL, 10.0, 1.0)]
CHARGE = ((10.0, 0, 0, 0, 0), (10.0, 0, 1, 0, 0))


def _params(n, seed, scale=0.3):
    p = ar.identity(n) + scale * np.random.default_rng(seed).normal(size=ar.n_params(n))
    return p.astype(np.float32)


def test_identity_and_roundtrip(ctx):
    fl = ctx.flow(4, kind=capi.FLOW_AR_SPLINE)
    assert fl.n_params == ar.n_params(4)
    z = np.random.default_rng(0).random((500, 4))
    x, jac = fl.sample(z)
    np.testing.assert_allclose(x, z, atol=1e-14)
    np.testing.assert_allclose(jac, 1.0, atol=1e-13)
    p = _params(4, 1)
    fl.set_params(p)
    np.testing.assert_array_equal(fl.params(), p)


@pytest.mark.parametrize("n", [1, 4, 8])
def test_maps_vs_oracle(ctx, n):
    fl = ctx.flow(n, kind=capi.FLOW_AR_SPLINE)
    p = _params(n, 10 + n)
    fl.set_params(p)
    pd = p.astype(np.float64)
    x = np.random.default_rng(n).random((800, n))
    z, logq = fl.density(x)
    zo, lqo = ar.forward(pd, x)
    assert np.abs(z - zo).max() < 1e-12 and np.abs(logq - lqo).max() < 1e-10
    xs, jac = fl.sample(z)
    xo, jo = ar.inverse(pd, z)
    assert np.abs(xs - xo).max() < 1e-11 and np.abs(xs - x).max() < 1e-10
    np.testing.assert_allclose(jac, jo, rtol=1e-9)


def test_separable_parameters_give_the_separable_flow(ctx):
    n = 5
    sep = (so.identity_params(n) + 0.4 * np.random.default_rng(3).normal(size=(n, so.PER_DIM))).astype(np.float32)
    fs = ctx.flow(n, kind=capi.FLOW_SPLINE)
    fs.set_params(sep)
    fa = ctx.flow(n, kind=capi.FLOW_AR_SPLINE)
    fa.set_params(learned.ar_from_separable(sep))
    z = np.random.default_rng(4).random((600, n))
    xs, js = fs.sample(z)
    xa, ja = fa.sample(z)
    np.testing.assert_array_equal(xs, xa)
    np.testing.assert_array_equal(js, ja)


def test_gradient_vs_oracle(ctx):
    """The training kernel's loss and gradient (per-sample derivatives chained to the
    conditioners, summed per CTA by a product in shared memory, then over CTAs) against the
    oracle on fp32-representable samples; 1,000 samples = 8 tiles, the last one partial."""
    n = 4
    fl = ctx.flow(n, kind=capi.FLOW_AR_SPLINE)
    p = _params(n, 7)
    fl.set_params(p)
    rng = np.random.default_rng(9)
    x = rng.random((1000, n)).astype(np.float32).astype(np.float64)
    w = (rng.random(1000) + 0.05).astype(np.float32).astype(np.float64)
    loss, g = fl.gradient(x, w)
    pd = p.astype(np.float64)
    lo = ar.loss(pd, x, w)
    assert abs(loss - lo) <= 1e-10 * abs(lo)
    go = ar.gradient(pd, x, w)
    assert np.abs(np.ravel(g) - go).max() <= 1e-6 * np.abs(go).max()


def _model(ctx):
    _, le, gr = flatband(1.0, 0.0, 0.0, 50.0, 10.0, 4001)
    return ctx.model(10.0, le, gr)


@pytest.mark.parametrize("n", [3, 8])
def test_inline_map_equals_map_kernel(ctx, n):
    """Work items with the flow are mapped in line by the integrand kernel: the sum equals
    f J over the points that the flow's own map kernel gives for the same Sobol indices,
    through kb_integrate and through a plan."""
    gm = _model(ctx)
    fl = ctx.flow(n, kind=capi.FLOW_AR_SPLINE)
    fl.set_params(_params(n, 31, 0.2))
    npts, k0 = 3000, 5
    rng = ctx.sobol(n)
    x, jac = fl.sample_sobol(rng, k0, npts)
    f = gm.evaluate_warped(CHARGE[0], CHARGE[1], PLASMA_EXP, x)[0] * jac
    item = dict(model=gm, rng=rng, chain=PLASMA_EXP, A=CHARGE[0], B=CHARGE[1], order=n, k_first=k0, n_points=npts,
                flow=fl)
    s, npt, nd, nfb = capi.integrate(ctx, [item])[0]
    assert npt == npts and nfb == 0
    assert abs(s - f.sum()) <= 1e-12 * np.abs(f).sum(), (s, f.sum())
    plan = capi.Plan(ctx, [item])
    assert plan.run()[0] == (s, npt, nd, nfb)
    plan.close()


def test_training_improves_on_the_separable_flow(ctx):
    """Warm-started from the separable spline flow and trained at order 4, the
    autoregressive flow's loss is no worse than the separable flow's, it lowers the
    per-point variance of f J against the plain chain, and its RQMC estimate agrees with the
    plain one within 4 combined standard errors."""
    gm = _model(ctx)
    order = 4
    sep, _, lsep = learned.fit(ctx, gm, CHARGE[0], CHARGE[1], PLASMA_EXP, order, 1 << 16, seed=3,
                               kind=capi.FLOW_SPLINE)
    fl, _, lar = learned.fit(ctx, gm, CHARGE[0], CHARGE[1], PLASMA_EXP, order, 1 << 16, seed=3,
                             kind=capi.FLOW_AR_SPLINE)
    assert math.isfinite(lar) and lar <= lsep + 0.02, (lar, lsep)
    assert learned.variance_gain(ctx, gm, CHARGE[0], CHARGE[1], PLASMA_EXP, fl) > 1.2
    c = learned.compare(ctx, gm, CHARGE[0], CHARGE[1], PLASMA_EXP, order, fl, 1 << 14, 16)
    assert c["diff_sigma"] <= 4.0, c
