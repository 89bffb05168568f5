"""Autotuner of the tree kernel's launch shape.

For each perturbation order it times a plan (one CUDA-graph launch) of a flat-band
workload over the candidate scheduling-chunk sizes and resident CTAs per SM, and keeps
the fastest. Results are cached per GPU model in ~/.cache/keldy_b200/ (or
$KELDY_B200_CACHE) and applied to a context with `apply`.
"""
from __future__ import annotations

import json
import os

from . import capi

CHUNKS = (32, 64, 128)
CTAS = (2, 4)
TIE = 0.01


def _points(order):
    """Points of a tuning run: 2^20 up to order 8 (over a dozen 128-point chunks per resident
    CTA of a B200's 592, so that the last partial wave does not favour small chunks);
    fewer at the costly high orders."""
    return {9: 1 << 18, 10: 1 << 17, 11: 1 << 16, 12: 1 << 15}.get(order, 1 << 20 if order <= 8 else 1 << 14)


def cache_path(ctx):
    import torch
    name = torch.cuda.get_device_name(0).replace(" ", "_") if torch.cuda.is_available() else "device"
    root = os.environ.get("KELDY_B200_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "keldy_b200"))
    return os.path.join(root, f"launch_{name}.json")


def tune(ctx, orders=range(1, 13), chunks=CHUNKS, ctas=CTAS, repeats=3, points=None):
    """{order: {"chunk_points", "ctas_per_sm", "ms"}} measured on this device. Shapes are
    tried from the largest chunk and CTA count down; a smaller one is kept only when it is
    faster by more than TIE (timing noise does not move the default)."""
    from .g0_tables import flatband
    _, le, gr = flatband(1.0, 0.0, 0.0, 50.0, 20.0, 40001)
    model = ctx.model(20.0, le, gr)
    chain = [(capi.WARPER_PLASMA_UV, 20.0, 0.0), (capi.WARPER_EXPONENTIAL, 20.0, 1.0)]
    saved = {n: ctx.get_launch(n) for n in range(0, 17)}
    ctx.set_timing(True)
    table = {}
    try:
        for n in orders:
            rng = ctx.sobol(n)
            npts = points or _points(n)
            best = None
            for c in sorted(chunks, reverse=True):
                for k in sorted(ctas, reverse=True):
                    ctx.set_launch(n, c, k)
                    plan = capi.Plan(ctx, [dict(model=model, rng=rng, chain=chain, A=(20.0, 0, 0), B=(20.0, 0, 1),
                                                order=n, k_first=1, n_points=npts)])
                    plan.run()  # first launch captures the graph
                    times = []
                    for _ in range(repeats):
                        plan.run()
                        times.append(ctx.last_timing()[0])
                    plan.close()
                    ms = min(times)
                    if best is None or ms < best[2] * (1.0 - TIE):
                        best = (c, k, ms)
            table[n] = {"chunk_points": best[0], "ctas_per_sm": best[1], "ms": best[2], "points": npts}
    finally:
        for n, (c, k) in saved.items():
            ctx.set_launch(n, c, k)
    return table


def apply(ctx, table):
    """Set the tuned chunk sizes, and the CTAs per SM of the most expensive tuned order."""
    if not table:
        return
    for n, v in table.items():
        ctx.set_launch(int(n), int(v["chunk_points"]), 0)
    heaviest = max(table, key=lambda n: int(n))
    ctx.set_launch(int(heaviest), int(table[heaviest]["chunk_points"]), int(table[heaviest]["ctas_per_sm"]))


def load_or_tune(ctx, orders=range(1, 13), retune=False):
    path = cache_path(ctx)
    if not retune and os.path.exists(path):
        with open(path) as f:
            table = {int(k): v for k, v in json.load(f).items()}
    else:
        table = tune(ctx, orders)
        os.makedirs(os.path.dirname(path), exist_ok=True)
        with open(path, "w") as f:
            json.dump(table, f, indent=1)
    apply(ctx, table)
    return table
