"""CPU restatement of the separable spline flow (keldy_b200/csrc/flow_spline.cu; test
infrastructure only): per dimension a monotone rational-quadratic spline CDF on [0, 1]
(Durkan et al., "Neural Spline Flows", 2019), its inverse, the weighted negative
log-likelihood and its gradient with respect to the parameters, in numpy float64. The
gradient is checked against central finite differences in tests/test_flow_oracle.py."""
from __future__ import annotations

import numpy as np

BINS = 16
PER_DIM = 3 * BINS + 1
MIN_BIN = 1e-3
MIN_DERIV = 1e-3


def identity_params(dim):
    p = np.zeros((dim, PER_DIM))
    p[:, 2 * BINS:] = np.log(np.expm1(1.0 - MIN_DERIV))
    return p


def _softmax(a):
    e = np.exp(a - a.max())
    return e / e.sum()


def knots(p):
    """(x[17], y[17], delta[17]) of one dimension's parameters."""
    w = MIN_BIN + (1 - BINS * MIN_BIN) * _softmax(p[:BINS])
    h = MIN_BIN + (1 - BINS * MIN_BIN) * _softmax(p[BINS:2 * BINS])
    x = np.concatenate([[0.0], np.cumsum(w)])
    y = np.concatenate([[0.0], np.cumsum(h)])
    x[-1] = y[-1] = 1.0
    d = MIN_DERIV + np.logaddexp(0.0, p[2 * BINS:])
    return x, y, d


def _bin(kn, v):
    return np.clip(np.searchsorted(kn[1:BINS], v, side="right"), 0, BINS - 1)


def forward(p, x):
    """z = F(x) and log F'(x) per dimension; x [count][dim]."""
    x = np.atleast_2d(x)
    z = np.empty_like(x)
    lq = np.zeros(x.shape[0])
    for d in range(x.shape[1]):
        kx, ky, kd = knots(p[d])
        j = _bin(kx, x[:, d])
        w = kx[j + 1] - kx[j]
        h = ky[j + 1] - ky[j]
        s = h / w
        xi = np.clip((x[:, d] - kx[j]) / w, 0.0, 1.0)
        e = xi * (1 - xi)
        d0, d1 = kd[j], kd[j + 1]
        den = s + (d1 + d0 - 2 * s) * e
        z[:, d] = ky[j] + h * (s * xi * xi + d0 * e) / den
        lq += np.log(s * s * (d1 * xi * xi + 2 * s * e + d0 * (1 - xi) ** 2) / den ** 2)
    return z, lq


def inverse(p, z):
    """x = F^{-1}(z) and dx/dz = 1 / prod F'(x)."""
    z = np.atleast_2d(z)
    x = np.empty_like(z)
    for d in range(z.shape[1]):
        kx, ky, kd = knots(p[d])
        j = _bin(ky, z[:, d])
        w = kx[j + 1] - kx[j]
        h = ky[j + 1] - ky[j]
        s = h / w
        d0, d1 = kd[j], kd[j + 1]
        t = z[:, d] - ky[j]
        g = d1 + d0 - 2 * s
        a, b, c = h * (s - d0) + t * g, h * d0 - t * g, -s * t
        xi = np.clip(2 * c / (-b - np.sqrt(np.maximum(b * b - 4 * a * c, 0.0))), 0.0, 1.0)
        x[:, d] = np.clip(kx[j] + xi * w, 0.0, 1.0)
    _, lq = forward(p, x)
    return x, np.exp(-lq)


def loss(p, x, w):
    """sum_i w_i (-log q(x_i)) / count."""
    return float(np.sum(-w * forward(p, x)[1]) / len(w))


def gradient(p, x, w):
    """d loss / d p [dim][PER_DIM], by the same chain of derivatives as the GPU kernels."""
    x = np.atleast_2d(x)
    wn = w / len(w)
    grad = np.zeros_like(p, dtype=np.float64)
    for d in range(x.shape[1]):
        kx, ky, kd = knots(p[d])
        j = _bin(kx, x[:, d])
        wj = kx[j + 1] - kx[j]
        h = ky[j + 1] - ky[j]
        s = h / wj
        xi = np.clip((x[:, d] - kx[j]) / wj, 0.0, 1.0)
        e = xi * (1 - xi)
        d0, d1 = kd[j], kd[j + 1]
        N = d1 * xi * xi + 2 * s * e + d0 * (1 - xi) ** 2
        D = s + (d1 + d0 - 2 * s) * e
        ls = 2 / s + 2 * e / N - 2 * (1 - 2 * e) / D
        ld0 = (1 - xi) ** 2 / N - 2 * e / D
        ld1 = xi * xi / N - 2 * e / D
        lxi = (2 * d1 * xi + 2 * s * (1 - 2 * xi) - 2 * d0 * (1 - xi)) / N - 2 * (d1 + d0 - 2 * s) * (1 - 2 * xi) / D
        gw, gx, gh, gd = np.zeros(BINS), np.zeros(BINS), np.zeros(BINS), np.zeros(BINS + 1)
        np.add.at(gh, j, -wn * ls / wj)
        np.add.at(gw, j, -wn * (ls * (-s / wj) + lxi * (-xi / wj)))
        np.add.at(gx, j, -wn * lxi * (-1 / wj))
        np.add.at(gd, j, -wn * ld0)
        np.add.at(gd, j + 1, -wn * ld1)
        GW = gw + np.concatenate([np.cumsum(gx[::-1])[::-1][1:], [0.0]])  # + sum over knots to the right
        sa, sb = _softmax(p[d, :BINS]), _softmax(p[d, BINS:2 * BINS])
        grad[d, :BINS] = (1 - BINS * MIN_BIN) * sa * (GW - np.dot(sa, GW))
        grad[d, BINS:2 * BINS] = (1 - BINS * MIN_BIN) * sb * (gh - np.dot(sb, gh))
        grad[d, 2 * BINS:] = gd / (1 + np.exp(-p[d, 2 * BINS:]))
    return grad
