"""CPU restatement of the autoregressive spline flow (keldy_b200/csrc/flow_arspline.cu;
test infrastructure only). Dimension d is mapped by a monotone rational-quadratic spline
CDF (the separable spline flow's, oracle/spline_flow_oracle.py) whose 49 parameters are a
linear function of smooth features of the dimensions before it (a Knothe-Rosenblatt
triangular map): theta_d = A_d phi_d(x_0..x_{d-1}), phi_d = [1, P1(x_k), P2(x_k), P3(x_k)
for k < d] with P_m the Legendre polynomials on [0, 1]. A_d is [49][1 + 3 d]; the flat
parameter vector holds A_0, A_1, ... row-major. The negative log-likelihood's gradient is
restated analytically (per sample: d loss / d theta_d through softmax, cumulative sums and
softplus, then the outer product with phi_d) and checked against central finite
differences in tests/test_flow_oracle.py."""
from __future__ import annotations

import numpy as np

from .spline_flow_oracle import BINS, MIN_BIN, MIN_DERIV, PER_DIM, identity_params

NFEAT = 3  # Legendre polynomials of degree 1..3 per conditioning coordinate


def n_features(d):
    return 1 + NFEAT * d


def n_params(dim):
    return PER_DIM * sum(n_features(d) for d in range(dim))


def offsets(dim):
    off, o = [], 0
    for d in range(dim):
        off.append(o)
        o += PER_DIM * n_features(d)
    return off


def unpack(params, dim):
    """[A_0, A_1, ...] with A_d of shape [PER_DIM][1 + 3 d]."""
    params = np.asarray(params, dtype=np.float64).ravel()
    out = []
    for d, o in enumerate(offsets(dim)):
        f = n_features(d)
        out.append(params[o:o + PER_DIM * f].reshape(PER_DIM, f))
    return out


def from_separable(sep):
    """The autoregressive flow equal to a separable spline flow (sep [dim][PER_DIM]): its
    parameters in the constant feature, zero elsewhere."""
    sep = np.atleast_2d(sep)
    dim = sep.shape[0]
    flat = np.zeros(n_params(dim))
    for d, o in enumerate(offsets(dim)):
        f = n_features(d)
        A = np.zeros((PER_DIM, f))
        A[:, 0] = sep[d]
        flat[o:o + PER_DIM * f] = A.ravel()
    return flat


def identity(dim):
    return from_separable(identity_params(dim))


def features(xprev):
    """phi for rows of conditioning coordinates xprev [count][d] -> [count][1 + 3 d]."""
    xprev = np.atleast_2d(xprev)
    cols = [np.ones(xprev.shape[0])]
    for k in range(xprev.shape[1]):
        u = 2.0 * xprev[:, k] - 1.0
        cols += [u, 1.5 * u * u - 0.5, (2.5 * u * u - 1.5) * u]
    return np.stack(cols, axis=1)


def _softmax_rows(a):
    e = np.exp(a - a.max(axis=1, keepdims=True))
    return e / e.sum(axis=1, keepdims=True)


def knots_rows(theta):
    """Per row of theta [count][PER_DIM]: x, y, delta [count][BINS + 1]."""
    w = MIN_BIN + (1 - BINS * MIN_BIN) * _softmax_rows(theta[:, :BINS])
    h = MIN_BIN + (1 - BINS * MIN_BIN) * _softmax_rows(theta[:, BINS:2 * BINS])
    z = np.zeros((theta.shape[0], 1))
    x = np.concatenate([z, np.cumsum(w, axis=1)], axis=1)
    y = np.concatenate([z, np.cumsum(h, axis=1)], axis=1)
    x[:, -1] = y[:, -1] = 1.0
    d = MIN_DERIV + np.logaddexp(0.0, theta[:, 2 * BINS:])
    return x, y, d


def _bin_rows(e, v):
    j = (v[:, None] >= e[:, 1:BINS]).sum(axis=1)
    return np.clip(j, 0, BINS - 1)


def _take(a, j):
    return np.take_along_axis(a, j[:, None], axis=1)[:, 0]


def forward(params, x):
    """z = F(x) and log q(x); x [count][dim]."""
    x = np.atleast_2d(x)
    dim = x.shape[1]
    As = unpack(params, dim)
    z = np.empty_like(x)
    lq = np.zeros(x.shape[0])
    for d in range(dim):
        th = features(x[:, :d]) @ As[d].T
        kx, ky, kd = knots_rows(th)
        j = _bin_rows(kx, x[:, d])
        w = _take(kx, j + 1) - _take(kx, j)
        h = _take(ky, j + 1) - _take(ky, j)
        s = h / w
        xi = np.clip((x[:, d] - _take(kx, j)) / w, 0.0, 1.0)
        e = xi * (1 - xi)
        d0, d1 = _take(kd, j), _take(kd, j + 1)
        den = s + (d1 + d0 - 2 * s) * e
        z[:, d] = _take(ky, j) + h * (s * xi * xi + d0 * e) / den
        lq += np.log(s * s * (d1 * xi * xi + 2 * s * e + d0 * (1 - xi) ** 2) / den ** 2)
    return z, lq


def inverse(params, z):
    """x = F^{-1}(z) dimension by dimension and dx/dz = 1 / q(x)."""
    z = np.atleast_2d(z)
    dim = z.shape[1]
    As = unpack(params, dim)
    x = np.empty_like(z)
    for d in range(dim):
        th = features(x[:, :d]) @ As[d].T
        kx, ky, kd = knots_rows(th)
        j = _bin_rows(ky, z[:, d])
        w = _take(kx, j + 1) - _take(kx, j)
        h = _take(ky, j + 1) - _take(ky, j)
        s = h / w
        d0, d1 = _take(kd, j), _take(kd, j + 1)
        t = z[:, d] - _take(ky, j)
        g = d1 + d0 - 2 * s
        a, b, c = h * (s - d0) + t * g, h * d0 - t * g, -s * t
        xi = np.clip(2 * c / (-b - np.sqrt(np.maximum(b * b - 4 * a * c, 0.0))), 0.0, 1.0)
        x[:, d] = np.clip(_take(kx, j) + xi * w, 0.0, 1.0)
    _, lq = forward(params, x)
    return x, np.exp(-lq)


def loss(params, x, w):
    """sum_i w_i (-log q(x_i)) / count."""
    return float(np.sum(-w * forward(params, x)[1]) / len(w))


def gradient(params, x, w):
    """d loss / d params (flat), by the chain the GPU kernels follow."""
    x = np.atleast_2d(x)
    dim = x.shape[1]
    As = unpack(params, dim)
    wn = w / len(w)
    grads = []
    cnt = x.shape[0]
    rows = np.arange(cnt)
    for d in range(dim):
        phi = features(x[:, :d])
        th = phi @ As[d].T
        kx, ky, kd = knots_rows(th)
        j = _bin_rows(kx, x[:, d])
        wj = _take(kx, j + 1) - _take(kx, j)
        h = _take(ky, j + 1) - _take(ky, j)
        s = h / wj
        xi = np.clip((x[:, d] - _take(kx, j)) / wj, 0.0, 1.0)
        e = xi * (1 - xi)
        d0, d1 = _take(kd, j), _take(kd, j + 1)
        N = d1 * xi * xi + 2 * s * e + d0 * (1 - xi) ** 2
        D = s + (d1 + d0 - 2 * s) * e
        ls = 2 / s + 2 * e / N - 2 * (1 - 2 * e) / D
        ld0 = (1 - xi) ** 2 / N - 2 * e / D
        ld1 = xi * xi / N - 2 * e / D
        lxi = (2 * d1 * xi + 2 * s * (1 - 2 * xi) - 2 * d0 * (1 - xi)) / N - 2 * (d1 + d0 - 2 * s) * (1 - 2 * xi) / D
        gh_j = -wn * ls / wj
        gw_j = -wn * (ls * (-s / wj) + lxi * (-xi / wj))
        gx_j = -wn * lxi * (-1 / wj)
        # widths: w_i enters bin j's width (i = j) and its left knot x_j (i < j)
        GW = np.zeros((cnt, BINS))
        GW[rows, j] += gw_j
        GW += np.where(np.arange(BINS)[None, :] < j[:, None], gx_j[:, None], 0.0)
        GH = np.zeros((cnt, BINS))
        GH[rows, j] = gh_j
        sa = _softmax_rows(th[:, :BINS])
        sb = _softmax_rows(th[:, BINS:2 * BINS])
        gth = np.zeros((cnt, PER_DIM))
        gth[:, :BINS] = (1 - BINS * MIN_BIN) * sa * (GW - (sa * GW).sum(axis=1, keepdims=True))
        gth[:, BINS:2 * BINS] = (1 - BINS * MIN_BIN) * sb * (GH - (sb * GH).sum(axis=1, keepdims=True))
        sig = 1 / (1 + np.exp(-th[:, 2 * BINS:]))
        gd = np.zeros((cnt, BINS + 1))
        gd[rows, j] = -wn * ld0
        gd[rows, j + 1] += -wn * ld1
        gth[:, 2 * BINS:] = gd * sig
        grads.append((gth.T @ phi).ravel())
    return np.concatenate(grads)
