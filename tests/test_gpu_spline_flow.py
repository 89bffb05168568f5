"""The learned separable spline flow on the GPU (kb_flow_create_kind(KB_FLOW_SPLINE)): its
maps and the gradient of its training kernel against the CPU restatement
(oracle/spline_flow_oracle.py, whose gradient is checked against finite differences),
training, and integration through it: unbiased against the plain warper chain, with a
smaller per-point variance than the chain alone."""
import math

import numpy as np
import pytest

from keldy_b200 import capi
from keldy_b200.g0_tables import flatband
from oracle import spline_flow_oracle as so

pytestmark = pytest.mark.gpu

PLASMA_EXP = [(capi.WARPER_PLASMA_UV, 10.0, 0.0), (capi.WARPER_EXPONENTIAL, 10.0, 1.0)]
CHARGE = ((10.0, 0, 0, 0, 0), (10.0, 0, 1, 0, 0))


def _params(n, seed):
    return (so.identity_params(n) + 0.5 * np.random.default_rng(seed).normal(size=(n, so.PER_DIM))).astype(np.float32)


def test_identity_and_roundtrip(ctx):
    fl = ctx.flow(3, kind=capi.FLOW_SPLINE)
    assert fl.n_params == 3 * so.PER_DIM
    z = np.random.default_rng(0).random((500, 3))
    x, jac = fl.sample(z)
    np.testing.assert_allclose(x, z, atol=1e-14)
    np.testing.assert_allclose(jac, 1.0, atol=1e-13)
    p = _params(3, 1)
    fl.set_params(p)
    np.testing.assert_array_equal(fl.params(), p)


@pytest.mark.parametrize("n", [1, 4, 8])
def test_maps_vs_oracle(ctx, n):
    fl = ctx.flow(n, kind=capi.FLOW_SPLINE)
    p = _params(n, 10 + n)
    fl.set_params(p)
    pd = p.astype(np.float64)
    x = np.random.default_rng(n).random((800, n))
    z, logq = fl.density(x)
    zo, lqo = so.forward(pd, x)
    assert np.abs(z - zo).max() < 1e-13 and np.abs(logq - lqo).max() < 1e-11
    xs, jac = fl.sample(z)
    xo, jo = so.inverse(pd, z)
    assert np.abs(xs - xo).max() < 1e-12 and np.abs(xs - x).max() < 1e-11
    np.testing.assert_allclose(jac, jo, rtol=1e-10)


def test_gradient_vs_oracle(ctx):
    """The training kernel's loss and gradient (fp64 sums of per-sample derivatives, chained
    to the parameters on the GPU) against the oracle on fp32-representable samples."""
    n = 5
    fl = ctx.flow(n, kind=capi.FLOW_SPLINE)
    p = _params(n, 7)
    fl.set_params(p)
    rng = np.random.default_rng(9)
    x = rng.random((5000, n)).astype(np.float32).astype(np.float64)
    w = (rng.random(5000) + 0.05).astype(np.float32).astype(np.float64)
    loss, g = fl.gradient(x, w)
    pd = p.astype(np.float64)
    assert abs(loss - so.loss(pd, x, w)) <= 1e-10 * abs(so.loss(pd, x, w))
    go = so.gradient(pd, x, w)
    assert np.abs(g - go).max() <= 1e-6 * np.abs(go).max()


def _model(ctx):
    _, le, gr = flatband(1.0, 0.0, 0.0, 50.0, 10.0, 4001)
    return ctx.model(10.0, le, gr)


def _replicas(ctx, gm, order, n_points, R, flow=None):
    items = [dict(model=gm, rng=ctx.sobol(order, 31, True, False, 100 + r), chain=PLASMA_EXP, A=CHARGE[0],
                  B=CHARGE[1], order=order, n_points=n_points, flow=flow) for r in range(R)]
    means = np.array([s / n for s, n, _, _ in capi.integrate(ctx, items)])
    return means.mean(), means.std(ddof=1) / math.sqrt(R)


def test_spline_flow_gain_and_unbiased(ctx):
    """Trained on |f J| of the plain chain at order 4, the spline flow lowers its loss, lowers
    the per-point variance of f J (same Sobol points, chain alone vs flow + chain), keeps
    the RQMC estimate within 4 combined standard errors of the plain one, and integrates
    through plans as through kb_integrate."""
    gm = _model(ctx)
    order = 4
    fl = ctx.flow(order, seed=2, kind=capi.FLOW_SPLINE)
    hist_loss = fl.fit(gm, CHARGE[0], CHARGE[1], PLASMA_EXP, ctx.sobol(order), 1 << 16, epochs=20, batch=8192,
                       lr=2e-2, lr_final=1e-3, seed=3)
    assert math.isfinite(hist_loss) and hist_loss < -0.05
    rng = ctx.sobol(order, 31, True, False, 77)
    z = rng.points(1, 1 << 14)
    plain = gm.evaluate_warped(CHARGE[0], CHARGE[1], PLASMA_EXP, z)[0]
    x, jac = fl.sample_sobol(rng, 1, 1 << 14)
    learned = gm.evaluate_warped(CHARGE[0], CHARGE[1], PLASMA_EXP, x)[0] * jac
    assert np.var(plain) / np.var(learned) > 1.2
    mp, ep = _replicas(ctx, gm, order, 1 << 14, 16)
    ml, el = _replicas(ctx, gm, order, 1 << 14, 16, fl)
    assert abs(ml - mp) <= 4.0 * math.hypot(ep, el), (ml, mp, ep, el)
    item = dict(model=gm, rng=ctx.sobol(order), chain=PLASMA_EXP, A=CHARGE[0], B=CHARGE[1], order=order,
                n_points=20000, flow=fl)
    plan = capi.Plan(ctx, [item])
    assert plan.run()[0] == capi.integrate(ctx, [item])[0]
    plan.close()


@pytest.mark.parametrize("n", [3, 8])
def test_inline_map_equals_map_kernel(ctx, n):
    """Work items with a spline flow are mapped in line by the integrand kernel (no mapped
    point buffer): the sum equals f J over the points that the flow's own map kernel gives
    for the same Sobol indices, and a parameter change takes effect at the next call and the
    next plan replay."""
    gm = _model(ctx)
    fl = ctx.flow(n, kind=capi.FLOW_SPLINE)
    npts, k0 = 3000, 5
    for seed in (31, 32):
        fl.set_params(_params(n, seed))
        rng = ctx.sobol(n)
        x, jac = fl.sample_sobol(rng, k0, npts)
        f = gm.evaluate_warped(CHARGE[0], CHARGE[1], PLASMA_EXP, x)[0] * jac
        item = dict(model=gm, rng=rng, chain=PLASMA_EXP, A=CHARGE[0], B=CHARGE[1], order=n, k_first=k0,
                    n_points=npts, flow=fl)
        s, npt, nd, nfb = capi.integrate(ctx, [item])[0]
        assert npt == npts and nfb == 0
        assert abs(s - f.sum()) <= 1e-12 * np.abs(f).sum(), (s, f.sum())
        if seed == 31:
            plan = capi.Plan(ctx, [item])
            assert plan.run()[0] == (s, npt, nd, nfb)
    assert plan.run()[0] == (s, npt, nd, nfb)  # replay after set_params: the new knots
    plan.close()


def test_mixed_batch_equals_separate(ctx):
    """One kb_integrate call over a plain item, a spline-flow item and a coupling-flow item
    gives each the sum of its own call."""
    gm = _model(ctx)
    sp = ctx.flow(4, kind=capi.FLOW_SPLINE)
    sp.set_params(_params(4, 3))
    cp = ctx.flow(5)
    base = dict(model=gm, chain=PLASMA_EXP, A=CHARGE[0], B=CHARGE[1], n_points=5000)
    items = [dict(base, rng=ctx.sobol(6), order=6), dict(base, rng=ctx.sobol(4), order=4, flow=sp),
             dict(base, rng=ctx.sobol(5), order=5, flow=cp)]
    together = capi.integrate(ctx, items)
    for it, r in zip(items, together):
        assert capi.integrate(ctx, [it])[0] == r
