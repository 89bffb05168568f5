"""CPU float64 statement of the learned coupling-flow warper (test infrastructure only).

keldy has no learned warper: this flow is an extension of its warper chain
(warpers/warpers.hpp:72-85 applies the chain last to first; the flow runs before the
first warper, mapping the Sobol point z to the chain's input li). This file is the
reference for the GPU kernels in keldy_b200/csrc/flow.cu; its analytic gradient is
checked against finite differences in tests/test_flow_oracle.py.

Architecture (shared with the kernels):
* dim n in [2, 8]; 6 coupling layers. Layer l transforms the dims T_l whose bit
  b = (l // 2) % ceil(log2 n) equals l % 2; the others condition it.
* Conditioner input: 128 features, 16 hat functions per dim (phi_j(x) = max(0, 1 -
  |16 x - j - 0.5|)) for conditioning dims; zero for transformed dims except feature
  16 * T_l[0], which is the constant 1 (the bias of the first layer).
* MLP: h1 = relu(W1 e), h2 = relu(W2 h1), logits = W3 h2, every W 128x128 ([out][in]).
  Hidden unit 127 is the constant 1 in h1 and h2 (it carries the biases of W2, W3).
* Output: per transformed dim (slot s = position in T_l), 32 logits -> bin
  probabilities p = (1 - eps) softmax + eps / 32; the normalising direction maps x to
  z = CDF_p(x) (piecewise linear) with density 32 p_bin; sampling inverts it.

With bf16=True, the weights and every GEMM operand (e, h1, h2 and, in the backward
pass, the logit gradient and the masked hidden gradients) are rounded to bf16 where the
kernels round them, so that the GPU can be compared at fp32-accumulation accuracy.
"""
from __future__ import annotations

import numpy as np

LAYERS = 6
WIDTH = 128
BLOB = 16
BINS = 32
SLOTS = 4
MAX_DIM = 8
EPS = 0.01
CONST_UNIT = 127


def bf16(a):
    """Round to the nearest bfloat16 (ties to even) via float32."""
    a32 = np.ascontiguousarray(np.asarray(a, dtype=np.float32))
    u = a32.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def nbits(n):
    return max(1, int(np.ceil(np.log2(n))))


def transformed(n, l):
    b = (l >> 1) % nbits(n)
    return [i for i in range(n) if ((i >> b) & 1) == (l & 1)]


def init_params(n, seed=0):
    """[layer][matrix][out][in] float32: W1, W2 uniform(+-sqrt(6/128)), W3 = 0."""
    rng = np.random.default_rng(seed)
    a = np.sqrt(6.0 / WIDTH)
    p = np.zeros((LAYERS, 3, WIDTH, WIDTH), dtype=np.float32)
    p[:, 0:2] = rng.uniform(-a, a, size=(LAYERS, 2, WIDTH, WIDTH)).astype(np.float32)
    return p


def encode(x, T, with_grad=False, f32=False):
    """Features [P,128] of the conditioning dims of x [P,n]; with_grad also returns the
    index/derivative pairs of the two non-zero hats per conditioning dim. f32: the
    coordinates are first rounded to float32 (as the kernels read them)."""
    P, n = x.shape
    E = np.zeros((P, WIDTH))
    E[:, BLOB * T[0]] = 1.0
    grads = []
    for i in range(n):
        if i in T:
            continue
        xi = x[:, i].astype(np.float32).astype(np.float64) if f32 else x[:, i]
        u = xi * BLOB - 0.5
        j0 = np.floor(u).astype(np.int64)
        f = u - j0
        rows = np.arange(P)
        for j, val, der in ((j0, 1.0 - f, -float(BLOB)), (j0 + 1, f, float(BLOB))):
            ok = (j >= 0) & (j < BLOB)
            E[rows[ok], BLOB * i + j[ok]] = val[ok]
            grads.append((i, np.where(ok, BLOB * i + j, 0), np.where(ok, der, 0.0)))
    return (E, grads) if with_grad else E


def _probs(logits):
    m = logits.max(axis=1, keepdims=True)
    e = np.exp(logits - m)
    s = e / e.sum(axis=1, keepdims=True)
    return s, (1.0 - EPS) * s + EPS / BINS


def conditioner(params_l, E, bf=False):
    """(h1, h2, logits) of one layer; params_l = [W1, W2, W3]."""
    W = [bf16(w) if bf else np.asarray(w, dtype=np.float64) for w in params_l]
    r = bf16 if bf else (lambda a: a)
    E = r(E)
    h1 = np.maximum(E @ W[0].T, 0.0)
    h1[:, CONST_UNIT] = 1.0
    h1 = r(h1)
    h2 = np.maximum(h1 @ W[1].T, 0.0)
    h2[:, CONST_UNIT] = 1.0
    h2 = r(h2)
    return E, h1, h2, h2 @ W[2].T


def forward(params, x, bf=False):
    """Normalising direction: z [P,n] and log q(x) [P]."""
    z = np.array(x, dtype=np.float64)
    n = z.shape[1]
    logq = np.zeros(z.shape[0])
    for l in range(LAYERS):
        T = transformed(n, l)
        _, _, _, logits = conditioner(params[l], encode(z, T, f32=bf), bf)
        for s, d in enumerate(T):
            _, p = _probs(logits[:, BINS * s:BINS * (s + 1)])
            u = z[:, d] * BINS
            b = np.clip(np.floor(u).astype(np.int64), 0, BINS - 1)
            frac = u - b
            cum = np.concatenate([np.zeros((p.shape[0], 1)), np.cumsum(p, axis=1)], axis=1)
            rows = np.arange(p.shape[0])
            z[:, d] = cum[rows, b] + frac * p[rows, b]
            logq += np.log(BINS * p[rows, b])
    return z, logq


def sample(params, z, bf=False):
    """Sampling direction: x [P,n] and the Jacobian dx/dz = 1/q(x) [P]."""
    x = np.array(z, dtype=np.float64)
    n = x.shape[1]
    jac = np.ones(x.shape[0])
    for l in reversed(range(LAYERS)):
        T = transformed(n, l)
        _, _, _, logits = conditioner(params[l], encode(x, T, f32=bf), bf)
        for s, d in enumerate(T):
            _, p = _probs(logits[:, BINS * s:BINS * (s + 1)])
            cum = np.concatenate([np.zeros((p.shape[0], 1)), np.cumsum(p, axis=1)], axis=1)
            b = np.clip((x[:, d:d + 1] >= cum[:, 1:]).sum(axis=1), 0, BINS - 1)
            rows = np.arange(p.shape[0])
            x[:, d] = np.clip((b + (x[:, d] - cum[rows, b]) / p[rows, b]) / BINS, 0.0, 1.0)
            jac /= BINS * p[rows, b]
    return x, jac


def loss_and_grad(params, x, w, bf=False):
    """loss = sum_p w_p (-log q(x_p)) / P and its gradient [layer][matrix][out][in]."""
    x = np.array(x, dtype=np.float64)
    P, n = x.shape
    w = np.asarray(w, dtype=np.float64)
    glq = -w / P
    r = bf16 if bf else (lambda a: a)
    xs = []
    z = x.copy()
    logq = np.zeros(P)
    for l in range(LAYERS):
        xs.append(z.copy())
        T = transformed(n, l)
        _, _, _, logits = conditioner(params[l], encode(z, T, f32=bf), bf)
        for s, d in enumerate(T):
            _, p = _probs(logits[:, BINS * s:BINS * (s + 1)])
            u = z[:, d] * BINS
            b = np.clip(np.floor(u).astype(np.int64), 0, BINS - 1)
            cum = np.concatenate([np.zeros((P, 1)), np.cumsum(p, axis=1)], axis=1)
            rows = np.arange(P)
            z[:, d] = cum[rows, b] + (u - b) * p[rows, b]
            logq += np.log(BINS * p[rows, b])
    loss = float(np.sum(w * -logq) / P)
    grad = np.zeros((LAYERS, 3, WIDTH, WIDTH))
    gx = np.zeros((P, n))
    rows = np.arange(P)
    for l in reversed(range(LAYERS)):
        xl = xs[l]
        T = transformed(n, l)
        E0, egr = encode(xl, T, with_grad=True, f32=bf)
        E, h1, h2, logits = conditioner(params[l], E0, bf)
        W = [bf16(m) if bf else np.asarray(m, dtype=np.float64) for m in params[l]]
        dlog = np.zeros((P, WIDTH))
        gnew = gx.copy()
        for s, d in enumerate(T):
            sm, p = _probs(logits[:, BINS * s:BINS * (s + 1)])
            u = xl[:, d] * BINS
            b = np.clip(np.floor(u).astype(np.int64), 0, BINS - 1)
            frac = u - b
            gz = gx[:, d]
            j = np.arange(BINS)[None, :]
            dp = gz[:, None] * ((j < b[:, None]) + (j == b[:, None]) * frac[:, None])
            dp[rows, b] += glq / p[rows, b]
            ds = (1.0 - EPS) * dp
            dlog[:, BINS * s:BINS * (s + 1)] = sm * (ds - (sm * ds).sum(axis=1, keepdims=True))
            gnew[:, d] = gz * BINS * p[rows, b]
        dlog = r(dlog)
        grad[l, 2] = dlog.T @ h2
        dh2 = dlog @ W[2]
        g2 = dh2 * (h2 > 0)
        g2[:, CONST_UNIT] = 0.0
        g2 = r(g2)
        grad[l, 1] = g2.T @ h1
        dh1 = g2 @ W[1]
        g1 = dh1 * (h1 > 0)
        g1[:, CONST_UNIT] = 0.0
        g1 = r(g1)
        grad[l, 0] = g1.T @ E
        if l > 0:
            dE = g1 @ W[0]
            for i, idx, der in egr:
                gnew[:, i] += dE[rows, idx] * der
        gx = gnew
    return loss, grad


def adam_step(params, m, v, grad, step, lr, beta1=0.9, beta2=0.999, eps=1e-8):
    """One Adam update (float32 state, as the kernel); step counts from 1."""
    m[:] = beta1 * m + (1 - beta1) * grad
    v[:] = beta2 * v + (1 - beta2) * grad * grad
    mh = m / (1 - beta1 ** step)
    vh = v / (1 - beta2 ** step)
    params[:] = params - lr * mh / (np.sqrt(vh) + eps)
