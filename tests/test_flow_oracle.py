"""The learned flow's CPU oracle (oracle/flow_oracle.py): its analytic gradient against
central finite differences, the sampling map as the inverse of the density map with
Jacobian 1/q, the coupling masks, and Adam. These pin the oracle that the GPU kernels
are compared with in test_gpu_flow.py."""
import numpy as np
import pytest

from oracle import flow_oracle as fo


def _params(n, seed):
    rng = np.random.default_rng(seed)
    p = fo.init_params(n, seed).astype(np.float64)
    p[:, 2] = rng.normal(0.0, 0.3, size=p[:, 2].shape)
    return p


@pytest.mark.parametrize("n", [2, 3, 5, 8])
def test_masks(n):
    seen = np.zeros(n, dtype=int)
    for l in range(fo.LAYERS):
        T = fo.transformed(n, l)
        assert 1 <= len(T) <= fo.SLOTS and len(T) < n
        seen[T] += 1
    assert (seen >= 2).all()


@pytest.mark.parametrize("n", [2, 5, 8])
def test_sample_inverts_density(n):
    p = _params(n, 7)
    x = np.random.default_rng(1).random((200, n))
    z, logq = fo.forward(p, x)
    assert ((z >= 0) & (z <= 1)).all()
    xb, jac = fo.sample(p, z)
    np.testing.assert_allclose(xb, x, atol=1e-12)
    np.testing.assert_allclose(jac * np.exp(logq), 1.0, rtol=1e-11)


def test_density_normalised():
    """q integrates to 1 over the cube (QMC estimate with 2^14 points, n = 2)."""
    p = _params(2, 3)
    g = np.random.default_rng(0)
    x = (np.arange(1 << 14)[:, None] + g.random((1 << 14, 2))) / (1 << 14)
    x[:, 1] = g.permutation(x[:, 1])
    _, logq = fo.forward(p, x)
    assert abs(np.exp(logq).mean() - 1.0) < 0.02


@pytest.mark.parametrize("n", [3, 5])
def test_gradient_vs_finite_differences(n):
    p = _params(n, 11)
    g = np.random.default_rng(2)
    x = g.random((48, n))
    w = g.random(48)
    _, grad = fo.loss_and_grad(p, x, w)
    worst = 0.0
    for _ in range(30):
        l, m = int(g.integers(fo.LAYERS)), int(g.integers(3))
        T = fo.transformed(n, l)
        o = int(g.integers(fo.BINS * len(T))) if m == 2 else int(g.integers(fo.WIDTH - 1))
        if m == 0:
            cond = [d for d in range(n) if d not in T]
            i = fo.BLOB * cond[int(g.integers(len(cond)))] + int(g.integers(fo.BLOB))
        else:
            i = int(g.integers(fo.WIDTH))
        h = 1e-6
        q = p.copy()
        q[l, m, o, i] += h
        lp, _ = fo.loss_and_grad(q, x, w)
        q[l, m, o, i] -= 2 * h
        lm, _ = fo.loss_and_grad(q, x, w)
        worst = max(worst, abs((lp - lm) / (2 * h) - grad[l, m, o, i]))
    assert worst < 1e-8


def test_bf16_rounding():
    a = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 1e-30, 65504.0])
    r = fo.bf16(a)
    assert r[0] == 1.0 and r[1] == 1.0  # halfway (1 + 2^-8) rounds to even
    assert r[2] == 1.0078125           # above halfway rounds up
    assert abs(r[3] + 3.140625) < 1e-12
    assert np.all(np.abs(r - a) <= np.abs(a) * 2.0 ** -8)


def test_adam_step():
    p = np.ones(4, dtype=np.float32)
    m = np.zeros(4, dtype=np.float32)
    v = np.zeros(4, dtype=np.float32)
    fo.adam_step(p, m, v, np.array([1.0, -1.0, 0.5, 0.0]), 1, 0.1)
    np.testing.assert_allclose(p, [0.9, 1.1, 0.9, 1.0], atol=1e-6)


def test_spline_flow_oracle_gradient_and_inverse():
    """The separable spline flow's CPU restatement: its hand-derived gradient equals central
    finite differences of its loss, and inverse(forward(x)) = x with consistent Jacobians."""
    from oracle import spline_flow_oracle as so
    rng = np.random.default_rng(3)
    dim = 3
    p = so.identity_params(dim) + 0.4 * rng.normal(size=(dim, so.PER_DIM))
    x = rng.random((400, dim))
    w = rng.random(400) + 0.1
    g = so.gradient(p, x, w)
    num = np.zeros_like(p)
    eps = 1e-6
    for idx in np.ndindex(*p.shape):
        pp, pm = p.copy(), p.copy()
        pp[idx] += eps
        pm[idx] -= eps
        num[idx] = (so.loss(pp, x, w) - so.loss(pm, x, w)) / (2 * eps)
    assert np.abs(g - num).max() < 1e-7 * max(1.0, np.abs(num).max())
    z, lq = so.forward(p, x)
    xb, jac = so.inverse(p, z)
    assert np.abs(xb - x).max() < 1e-12
    assert np.allclose(jac, np.exp(-lq), rtol=1e-10)
    xi, _ = so.forward(so.identity_params(dim), x)
    assert np.abs(xi - x).max() < 1e-15


def test_ar_spline_flow_oracle_gradient_and_inverse():
    """The autoregressive spline flow's CPU restatement: its analytic gradient equals central
    finite differences of its loss, inverse(forward(x)) = x with Jacobian 1/q, and with
    only the constant feature set it is the separable spline flow."""
    from oracle import ar_spline_flow_oracle as ar
    from oracle import spline_flow_oracle as so
    rng = np.random.default_rng(4)
    dim = 3
    p = ar.identity(dim) + 0.3 * rng.normal(size=ar.n_params(dim))
    x = rng.random((400, dim))
    w = rng.random(400) + 0.1
    g = ar.gradient(p, x, w)
    num = np.zeros_like(p)
    eps = 1e-6
    for i in range(len(p)):
        pp, pm = p.copy(), p.copy()
        pp[i] += eps
        pm[i] -= eps
        num[i] = (ar.loss(pp, x, w) - ar.loss(pm, x, w)) / (2 * eps)
    assert np.abs(g - num).max() < 1e-7 * max(1.0, np.abs(num).max())
    z, lq = ar.forward(p, x)
    xb, jac = ar.inverse(p, z)
    assert np.abs(xb - x).max() < 1e-12
    assert np.allclose(jac, np.exp(-lq), rtol=1e-10)
    sep = so.identity_params(dim) + 0.4 * rng.normal(size=(dim, so.PER_DIM))
    z1, l1 = so.forward(sep, x)
    z2, l2 = ar.forward(ar.from_separable(sep), x)
    assert np.array_equal(z1, z2) and np.array_equal(l1, l2)
    assert ar.n_params(8) == 49 * (8 + 3 * 28)
