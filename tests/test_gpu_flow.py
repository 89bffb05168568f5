"""The learned coupling-flow warper on the GPU (kb_flow_*): the tensor-core maps and the
gradient of the training kernel against the CPU oracle (oracle/flow_oracle.py, bf16
operands emulated), the exact inverse / Jacobian relations, training on a known
density, and integration through the flow: unbiased against the plain warper chain and
with a smaller per-point variance than the chain alone."""
import math

import numpy as np
import pytest

from keldy_b200 import capi
from keldy_b200.g0_tables import flatband
from oracle import flow_oracle as fo

pytestmark = pytest.mark.gpu

PLASMA_EXP = [(capi.WARPER_PLASMA_UV, 10.0, 0.0), (capi.WARPER_EXPONENTIAL, 10.0, 1.0)]
CHARGE = ((10.0, 0, 0, 0, 0), (10.0, 0, 1, 0, 0))


def _random_params(n, seed, scale=0.3):
    p = fo.init_params(n, seed)
    p[:, 2] = np.random.default_rng(seed).normal(0.0, scale, size=p[:, 2].shape).astype(np.float32)
    return p


def test_identity_at_creation(ctx):
    fl = ctx.flow(4, seed=3)
    z = np.random.default_rng(0).random((1000, 4))
    x, jac = fl.sample(z)
    np.testing.assert_allclose(x, z, atol=1e-13)
    np.testing.assert_allclose(jac, 1.0, atol=1e-13)
    p = fl.params()
    assert np.all(p[:, 2] == 0.0) and np.abs(p[:, :2]).max() <= math.sqrt(6 / 128)


def test_params_roundtrip(ctx):
    fl = ctx.flow(5)
    p = _random_params(5, 1)
    fl.set_params(p)
    np.testing.assert_array_equal(fl.params(), p)


@pytest.mark.parametrize("n", [2, 3, 5, 8])
def test_density_and_sample_vs_oracle(ctx, n):
    fl = ctx.flow(n)
    p = _random_params(n, 10 + n)
    fl.set_params(p)
    x = np.random.default_rng(n).random((700, n))
    z, logq = fl.density(x)
    zo, lqo = fo.forward(p, x, bf=True)
    dz, dl = np.abs(z - zo), np.abs(logq - lqo)
    assert np.median(dz) < 1e-5 and dz.max() < 5e-3, (np.median(dz), dz.max())
    assert np.median(dl) < 1e-4 and dl.max() < 2e-2, (np.median(dl), dl.max())
    xs, jac = fl.sample(z)
    xo, jo = fo.sample(p, z, bf=True)
    assert np.median(np.abs(xs - xo)) < 1e-5
    # the GPU's own maps are exact inverses with Jacobian 1/q
    np.testing.assert_allclose(xs, x, atol=1e-6)
    np.testing.assert_allclose(jac * np.exp(logq), 1.0, rtol=1e-6)


@pytest.mark.parametrize("n", [3, 6])
def test_gradient_vs_oracle(ctx, n):
    fl = ctx.flow(n)
    p = _random_params(n, 20 + n)
    fl.set_params(p)
    g = np.random.default_rng(n)
    x = g.random((600, n))  # five tiles, the last one partial
    w = g.random(600) * 2.0
    loss, grad = fl.gradient(x, w)
    lo, go = fo.loss_and_grad(p, x, w, bf=True)
    assert abs(loss - lo) <= 1e-4 * abs(lo) + 1e-6
    for l in range(fo.LAYERS):
        for m in range(3):
            ref = go[l, m]
            err = np.linalg.norm(grad[l, m] - ref) / max(np.linalg.norm(ref), 1e-12)
            assert err < 2e-2, (l, m, err)


def test_training_learns_a_density(ctx):
    """Weights g(x) = prod 3 x_d^2 (integral 1): after training, g(x(z)) J(z) at Sobol
    points has a much smaller variance than g(z)."""
    n = 3
    fl = ctx.flow(n, seed=5)
    rng = ctx.sobol(n)
    x = rng.points(1, 1 << 16)
    w = np.prod(3.0 * x * x, axis=1)
    hist = fl.train(x, w, epochs=12, batch=4096, lr=3e-3, lr_final=1e-4, seed=1)
    assert hist[-16:].mean() < hist[:4].mean() - 0.3
    z = ctx.sobol(n, 31, True, False, 9).points(1, 1 << 14)
    xs, jac = fl.sample(z)
    plain = np.prod(3.0 * z * z, axis=1)
    learned = np.prod(3.0 * xs * xs, axis=1) * jac
    assert abs(learned.mean() - 1.0) < 0.02
    assert learned.var() < 0.1 * plain.var(), (learned.var(), plain.var())


def _model(ctx):
    _, le, gr = flatband(1.0, 0.0, 0.0, 50.0, 10.0, 10001)
    return ctx.model(10.0, le, gr)


def test_identity_flow_integrates_like_plain(ctx):
    gm = _model(ctx)
    rng = ctx.sobol(4)
    fl = ctx.flow(4)
    base = dict(model=gm, rng=rng, chain=PLASMA_EXP, A=CHARGE[0], B=CHARGE[1], order=4, n_points=20000)
    (s0, n0, d0, _), (s1, n1, d1, _) = capi.integrate(ctx, [base, dict(base, flow=fl)])
    scale = np.abs(gm.evaluate_warped(CHARGE[0], CHARGE[1], PLASMA_EXP, rng.points(1, 20000))[0]).sum()
    assert (n0, d0) == (n1, d1)
    assert abs(s1 - s0) <= 1e-12 * scale


def test_plan_with_flow_equals_integrate(ctx):
    gm = _model(ctx)
    rng = ctx.sobol(5)
    fl = ctx.flow(5)
    fl.set_params(_random_params(5, 4, scale=0.05))
    item = dict(model=gm, rng=rng, chain=PLASMA_EXP, A=CHARGE[0], B=CHARGE[1], order=5, n_points=30000, flow=fl)
    direct = capi.integrate(ctx, [item])[0]
    plan = capi.Plan(ctx, [item])
    assert plan.run()[0] == direct
    plan.set_k_first(0, 30001)
    assert plan.run()[0] == capi.integrate(ctx, [dict(item, k_first=30001)])[0]
    plan.close()


def _replicas(ctx, gm, order, n_points, R, flow=None):
    items = []
    for r in range(R):
        items.append(dict(model=gm, rng=ctx.sobol(order, 31, True, False, 100 + r), chain=PLASMA_EXP, A=CHARGE[0],
                          B=CHARGE[1], order=order, n_points=n_points, flow=flow))
    means = np.array([s / n for s, n, _, _ in capi.integrate(ctx, items)])
    return means.mean(), means.std(ddof=1) / math.sqrt(R)


def test_learned_flow_gain_order4(ctx):
    """Trained on |f J| of the plain chain, the flow lowers the per-point variance of the
    estimator at least 3-fold (the same Sobol points through chain alone vs flow + chain)
    and keeps the RQMC estimate within the combined standard error of the plain one."""
    gm = _model(ctx)
    order = 4
    fl = ctx.flow(order, seed=2)
    loss = fl.fit(gm, CHARGE[0], CHARGE[1], PLASMA_EXP, ctx.sobol(order), 1 << 16, epochs=10, batch=4096, lr=2e-3,
                  lr_final=1e-4, seed=3)
    assert math.isfinite(loss) and loss < -0.1
    rng = ctx.sobol(order, 31, True, False, 77)
    z = rng.points(1, 1 << 14)
    plain = gm.evaluate_warped(CHARGE[0], CHARGE[1], PLASMA_EXP, z)[0]
    x, jac = fl.sample_sobol(rng, 1, 1 << 14)
    learned = gm.evaluate_warped(CHARGE[0], CHARGE[1], PLASMA_EXP, x)[0] * jac
    gain = np.var(plain) / np.var(learned)
    assert gain > 3.0, gain
    mp, ep = _replicas(ctx, gm, order, 1 << 14, 16)
    ml, el = _replicas(ctx, gm, order, 1 << 14, 16, fl)
    assert abs(ml - mp) <= 4.0 * math.hypot(ep, el), (ml, mp, ep, el)
