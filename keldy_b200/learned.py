"""The learned warper workflow: a flow per perturbation order, trained on the GPU on
|integrand| samples of the plain method, judged against the plain warper chain.

Three flow designs (kb_flow_*): coupling layers with tensor-core MLP conditioners
(csrc/flow.cu), a separable rational-quadratic spline per dimension (csrc/flow_spline.cu;
the one that pays under quasi-Monte Carlo) and its autoregressive extension
(csrc/flow_arspline.cu). The flow is a first stage before keldy's warper chain
(warpers.hpp:72-85); the plain chain alone is the method without it. Both are estimated
with randomised QMC (R random digital shifts of the Sobol sequence, qrng.hpp:77-109), so
their standard errors and their agreement are measured the same way.
"""
from __future__ import annotations

import math
import time

import numpy as np

from . import capi, rqmc

DEFAULT_TRAIN = dict(epochs=10, batch=8192, lr=2e-3, lr_final=1e-4)
# the separable spline flow has ~50 parameters per dimension: larger steps, more epochs
SPLINE_TRAIN = dict(epochs=20, batch=8192, lr=2e-2, lr_final=1e-3)
# the autoregressive spline flow after its separable warm start: a smaller first step
AR_TRAIN = dict(epochs=20, batch=8192, lr=5e-3, lr_final=2e-4)


def fit(ctx, model, A, B, chain, order, n_samples=1 << 18, seed=0, k_first=1, kind=capi.FLOW_COUPLING, **cfg):
    """Creates and trains a flow (kind FLOW_COUPLING, FLOW_SPLINE or FLOW_AR_SPLINE) of
    dimension `order` on n_samples plain-method points. The autoregressive spline flow is
    warm-started from a separable spline flow trained first (its parameters in the constant
    feature), then trained as a whole. Returns (flow, seconds, final loss)."""
    c = dict(DEFAULT_TRAIN if kind == capi.FLOW_COUPLING else SPLINE_TRAIN, **cfg)
    c.setdefault("seed", seed)
    flow = ctx.flow(order, seed=seed, kind=kind)
    ctx.synchronize()
    t0 = time.perf_counter()
    if kind == capi.FLOW_AR_SPLINE:
        sep = ctx.flow(order, seed=seed, kind=capi.FLOW_SPLINE)
        sep.fit(model, A, B, chain, ctx.sobol(order), n_samples, k_first=k_first, **c)
        flow.set_params(ar_from_separable(sep.params()))
        sep.close()
        c = dict(c, **AR_TRAIN)
        c.update(cfg)
    loss = flow.fit(model, A, B, chain, ctx.sobol(order), n_samples, k_first=k_first, **c)
    ctx.synchronize()
    return flow, time.perf_counter() - t0, loss


def ar_from_separable(sep):
    """Parameters of the autoregressive spline flow equal to a separable spline flow's
    (sep [dim][49]): each dimension's in its constant feature, the other weights zero."""
    sep = np.atleast_2d(np.asarray(sep, dtype=np.float32))
    dim = sep.shape[0]
    out = []
    for d in range(dim):
        a = np.zeros((49, 1 + 3 * d), dtype=np.float32)
        a[:, 0] = sep[d]
        out.append(a.ravel())
    return np.concatenate(out)


def variance_gain(ctx, model, A, B, chain, flow, n_points=1 << 15, seed_shift=977):
    """Per-point variance of f J through the chain alone over that through flow + chain, on
    the same shifted Sobol points (the plain Monte Carlo gain of the flow)."""
    rng = ctx.sobol(flow.dim, 31, True, False, seed_shift)
    z = rng.points(1, n_points)
    plain = model.evaluate_warped(A, B, chain, z)[0]
    x, jac = flow.sample_sobol(rng, 1, n_points)
    learned = model.evaluate_warped(A, B, chain, x)[0] * jac
    return float(np.var(plain) / np.var(learned))


def compare(ctx, model, A, B, chain, order, flow, n_points, replicas=16, seed_shift0=1):
    """Plain and learned RQMC estimates at n_points per replica: dict with mean, stderr,
    seconds (wall, one batched call each) and the difference in combined standard errors."""
    out = {}
    for name, f in (("plain", None), ("learned", flow)):
        rngs = [ctx.sobol(order, 31, True, False, seed_shift0 + r) for r in range(replicas)]
        rqmc.estimate(ctx, model, A, B, chain, order, min(n_points, 1 << 10), replicas, rngs=rngs, flow=f)
        ctx.synchronize()
        t0 = time.perf_counter()
        mean, err, _ = rqmc.estimate(ctx, model, A, B, chain, order, n_points, replicas, rngs=rngs, flow=f)
        dt = time.perf_counter() - t0
        out[name] = dict(mean=complex(mean), stderr=float(err), rel=float(err / abs(mean)), seconds=dt)
    p, l = out["plain"], out["learned"]
    out["diff_sigma"] = abs(l["mean"] - p["mean"]) / math.hypot(p["stderr"], l["stderr"])
    out["stderr_ratio"] = p["stderr"] / l["stderr"]
    return out


def select(ctx, model, A, B, chain, order, flow, pilot_points=1 << 14, replicas=16):
    """The plain estimator judges the flow: returns the flow when its RQMC standard error on
    a pilot run is below the plain chain's, else None (use the plain chain)."""
    c = compare(ctx, model, A, B, chain, order, flow, pilot_points, replicas, seed_shift0=10_001)
    return (flow if c["learned"]["stderr"] < c["plain"]["stderr"] else None), c
