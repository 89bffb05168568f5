"""Randomised quasi-Monte Carlo error bars on the GPU.

R independent random digital shifts of the same Sobol sequence (keldy's
sobol(dim, seed, do_shift=true, do_scramble, rng_seed_shift = 1..R), qrng.hpp:77-109)
give R unbiased estimates of the integral; their mean is the estimate and their
standard deviation / sqrt(R) its standard error. All replicas of all orders run in one
kb_integrate call (one batched launch).
"""
from __future__ import annotations

import math
import time

import numpy as np

from . import capi


def estimate(ctx, model, A, B, chain, order, n_points, replicas=16, seed_shift0=1, scramble=False, k_first=1,
             cutoff=0.0, algo=capi.ALGO_AUTO, rngs=None, flow=None):
    """Mean, standard error and per-replica means of int f(warp(x)) J dx over [0,1]^order.
    rngs: optional list of `replicas` prebuilt shifted generators (reused across calls).
    flow: optional learned flow applied before the chain."""
    if rngs is None:
        rngs = [ctx.sobol(order, 31, True, scramble, seed_shift0 + r) for r in range(replicas)]
    items = [dict(model=model, rng=g, chain=chain, A=A, B=B, cutoff=cutoff, order=order, k_first=k_first,
                  n_points=n_points, flow=flow) for g in rngs]
    res = capi.integrate(ctx, items, algo)
    means = np.array([s / n for s, n, _, _ in res])
    mean = means.mean()
    r = len(means)
    err = math.sqrt((np.abs(means - mean) ** 2).sum() / (r - 1) / r) if r > 1 else float("nan")
    return mean, err, means


def time_to_relative_error(ctx, model, A, B, chain, order, target=1e-3, replicas=16, start_points=1 << 12,
                           max_points=1 << 24, seed_shift0=1, scramble=False, flow=None):
    """Doubles the points per replica until stderr / |mean| <= target (or max_points is
    reached). Returns dict(mean, stderr, rel, points_per_replica, evaluations, seconds):
    `seconds` is the wall time of the run that met the target (the GPU work needed at
    that size, excluding the smaller probing runs)."""
    rngs = [ctx.sobol(order, 31, True, scramble, seed_shift0 + r) for r in range(replicas)]
    n = start_points
    while True:
        ctx.synchronize()
        t0 = time.perf_counter()
        mean, err, _ = estimate(ctx, model, A, B, chain, order, n, replicas, rngs=rngs, flow=flow)
        dt = time.perf_counter() - t0
        rel = err / abs(mean) if mean != 0 else float("inf")
        if rel <= target or n >= max_points:
            return dict(mean=mean, stderr=err, rel=rel, points_per_replica=n, evaluations=n * replicas, seconds=dt,
                        reached=rel <= target)
        n *= 2


def time_to_relative_error_ladders(ctx, model, A, B, chain, order, target=1e-3, ladders=8, replicas=16,
                                   start_points=1 << 8, max_points=1 << 22, seed_shift0=1, scramble=False, flow=None):
    """time_to_relative_error repeated over `ladders` independent ladders (disjoint blocks of
    random digital shifts), each on a sqrt(2) grid of points per replica (start_points *
    2^(k/2), rounded). Per ladder: the points per replica and the wall time of the run that
    first met stderr / |mean| <= target. Returns the medians and interquartile ranges over the
    ladders, and the per-ladder values."""
    grid, k = [], 0
    while True:
        n = int(round(start_points * 2.0 ** (k / 2.0)))
        grid.append(min(n, max_points))
        if n >= max_points:
            break
        k += 1
    secs, pts, reached = [], [], []
    for lad in range(ladders):
        rngs = [ctx.sobol(order, 31, True, scramble, seed_shift0 + lad * replicas + r) for r in range(replicas)]
        estimate(ctx, model, A, B, chain, order, grid[0], replicas, rngs=rngs, flow=flow)  # warm-up
        for n in grid:
            ctx.synchronize()
            t0 = time.perf_counter()
            mean, err, _ = estimate(ctx, model, A, B, chain, order, n, replicas, rngs=rngs, flow=flow)
            dt = time.perf_counter() - t0
            rel = err / abs(mean) if mean != 0 else float("inf")
            if rel <= target or n == grid[-1]:
                secs.append(dt)
                pts.append(n)
                reached.append(rel <= target)
                break
    q = lambda a, p: float(np.percentile(np.asarray(a, dtype=float), p))  # noqa: E731
    return dict(seconds_median=q(secs, 50), seconds_iqr=[q(secs, 25), q(secs, 75)],
                points_median=q(pts, 50), points_iqr=[q(pts, 25), q(pts, 75)], seconds=secs, points=pts,
                all_reached=all(reached), ladders=ladders, replicas=replicas, target=target)
