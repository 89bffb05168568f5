#!/usr/bin/env python
"""Throughput of the keldy QMC hot path on B200: integrand evaluations per second at
perturbation order 8.

Workload (the batched flat-band configuration): single-level dot, flat-band leads
Gamma = 1, eps_d = 0, V = 0, beta = 50; g0^<, g0^> tabulated on 40,001 points over
[-20, 20]; charge observable G^<_{up,up}(t, t) at t = 20; warper chain
[plasma_uv(20), product-1D exponential(20, 1/Gamma)]; unshifted Sobol points. One step
= 2^20 Sobol points per GPU through Sobol -> warpers -> Wick-determinant integrand ->
QMC sum. Synthetic g0 tables built on the host from the model's closed form.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Under torchrun each rank takes its own contiguous block of Sobol indices (weak
scaling); the per-rank sums are combined with one all_reduce, as keldy's
integrator::reduce_result does.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GAMMA, EPS_D, BIAS, BETA, T_MAX, NPTS = 1.0, 0.0, 0.0, 50.0, 20.0, 40001
# DRAM bytes (read + write) of one tree_kernel launch of this workload (2^20 points,
# order 8) from an ncu capture (dram__bytes_read.sum + dram__bytes_write.sum), keyed by
# the hash of the kernel's code (tree_source_hash, comments stripped) at the time of the capture. A build
# whose sources hash differently reports no traffic figure until it is captured again.
TREE_DRAM_CAPTURES = {"e99222e79bec14ce": 2335744 + 204688384}
TREE_SOURCES = ("tree.cu", "kb_device.cuh", "kb_types.h", "kb_launch.h", "kb_spline.cuh", "kb_flow.h")
E2E_REPEATS = 5


def _code_only(text):
    """C++ source without its comments and with runs of white space collapsed (these sources
    hold no string literal with a comment marker), so that a comment edit keeps the hash."""
    import re
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    text = re.sub(r"//[^\n]*", " ", text)
    return " ".join(text.split())


def tree_source_hash():
    """First 16 hex digits of the SHA-256 of the tree kernel's source files, comments
    stripped."""
    import hashlib
    h = hashlib.sha256()
    for f in TREE_SOURCES:
        with open(os.path.join(ROOT, "keldy_b200", "csrc", f), encoding="utf-8") as fh:
            h.update(_code_only(fh.read()).encode())
    return h.hexdigest()[:16]


def flop_lu(m):
    """FLOPs of an m x m complex LU with determinant (complex FMA = 8, multiply = 6)."""
    return 8 * (m - 1) * m * (2 * m - 1) // 6 + 6 * m * (m - 1) // 2 + 6 * (m - 1)


def reference_flops(n):
    """keldy's algorithm: 2^n configurations x (LU(n+1) + LU(n) + product)."""
    return (1 << n) * (flop_lu(n + 1) + flop_lu(n) + 8)


def tree_flops(n):
    """FLOPs the Schur-complement tree executes per point: per child of a level-k node
    of size m = 2(n-k)+1, one reciprocal (~8), the prefix product (6), (m-2) scaled
    pivot entries (6 each) and (m-2)^2 complex FMAs (8 each); per leaf ~34."""
    total = 0
    for k in range(n - 1):
        m = 2 * (n - k) + 1
        total += (1 << (k + 1)) * (8 + 6 + 6 * (m - 2) + 8 * (m - 2) ** 2)
    return total + (1 << n) * 34


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples while the timed region runs."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.lines = []
        self.proc = None

    def start(self, wait_first=True):
        """Starts sampling; waits (up to 10 s) for the first sample, so that nvidia-smi's
        start-up, which stalls this process's CUDA calls for up to a second, ends before the
        measured regions."""
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except OSError:
            self.proc = None
            return
        t0 = time.time()
        while wait_first and not self.lines and time.time() - t0 < 10.0:
            time.sleep(0.05)
        time.sleep(0.3)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def mark(self):
        """Index of the next sample (start/end of a measured window)."""
        return len(self.lines)

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self, a=0, b=None):
        """Median SM clock, max clock and throttle reasons of samples a..b."""
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines[a:b]:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx = max(mx, float(parts[1]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[4:8]):
                if flag.lower() in ("active", "1", "yes"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


class CpuReference:
    """keldy's own integrand (oracle/_ref: wick_direct.cpp, digitalseq_b2g.hpp and the
    warper headers) on the host cores, on bounded samples of the workload. It picks the
    faster of keldy's two parallel modes: OpenMP over the Keldysh configurations inside
    one integrand call (as shipped), or one worker per core keeping every P-th Sobol point
    (its MPI round robin). Without a built oracle/_ref it times the C restatement."""

    def __init__(self, order, threads=None):
        import numpy as np  # noqa: F401
        from keldy_b200.g0_tables import flatband
        from oracle import pyoracle as po
        self.order = order
        self.threads = threads or os.cpu_count() or 1
        _, le, gr = flatband(GAMMA, EPS_D, BIAS, BETA, T_MAX, NPTS)
        self.A, self.B = (T_MAX, 0, 0, 0, 0), (T_MAX, 0, 1, 0, 0)
        self.chain = [(po.W_PLASMA_UV, T_MAX, 0.0), (po.W_EXPONENTIAL, T_MAX, 1.0 / GAMMA)]
        if po.reference_available():
            self.ref = po.Reference(timed=True)
            self.model = self.ref.model(T_MAX, le, gr)
            self.kind = "reference"
            best = None
            for mode in (0, 1):
                n = max(self.threads, 64)
                dt = self._run(n, mode)
                if best is None or n / dt > best[1]:
                    best = (mode, n / dt)
            self.mode, self.rate = best
            self.desc = ("keldy wick_direct.cpp + digitalseq_b2g.hpp + warper headers, g++ -O3 -march=x86-64-v3, "
                         + ("OpenMP over Keldysh configurations" if self.mode == 0
                            else f"{self.threads} round-robin workers"))
        else:
            self.ref = None
            self.oracle = po.Oracle()
            self.model = self.oracle.model(T_MAX, le, gr)
            self.kind = "port"
            self.threads = 1
            self.mode = None
            self.rate = 200 / self._run(200, None)
            self.desc = "C restatement, 1 thread"

    def _run(self, n, mode):
        t0 = time.perf_counter()
        if self.ref is not None:
            self.ref.integrate(self.model, self.A, self.B, self.chain, self.order, n, mode=mode, threads=self.threads)
        else:
            self.oracle.integrate(self.model, self.A, self.B, self.chain, self.order, n)
        return time.perf_counter() - t0

    def sample_size(self, seconds):
        return int(max(self.threads * 4, min(1 << 20, self.rate * seconds)))

    def measure(self, n):
        dt = self._run(n, self.mode)
        return {"value": n / dt, "unit": "evals/s", "cores": self.threads, "kind": self.kind, "n": n, "seconds": dt,
                "sample": f"{n} Sobol points of the order-{self.order} workload ({self.desc})"}


def run_reference_arm(args, rank, world):
    if rank != 0:
        return
    order = args.order
    cpu = CpuReference(order)
    n = cpu.sample_size(args.ref_seconds)
    for _ in range(args.warmup):
        cpu.measure(max(cpu.threads, n // 8))
    res = [cpu.measure(n) for _ in range(args.steps)]
    pts = sum(r["n"] for r in res)
    secs = sum(r["seconds"] for r in res)
    value = pts / secs
    line = {"metric": f"integrand evals/s at order {order}", "value": value, "unit": "evals/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": workload_config(order, args.points),
            "cpu_baseline": {"value": value, "unit": "evals/s", "cores": res[0]["cores"], "kind": res[0]["kind"],
                             "sample": res[0]["sample"]},
            "e2e": {"value": value, "unit": "evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def workload_config(order, points):
    return {"workload": f"flat-band dot Gamma=1 eps_d=0 V=0 beta=50, charge G^<(t=20), g0 {NPTS} points on "
                        f"[-20,20], chain [plasma_uv(20), exponential(20, 1/Gamma)], order {order}, "
                        f"{points} Sobol points per GPU per step",
            "order": order, "points_per_gpu_per_step": points, "g0_points": NPTS, "t": T_MAX, "beta": BETA,
            "l2": "flushed between timed steps (256 MiB write)"}


def measure_biased_dot(ctx):
    """Biased dot, orders 6..12 in one CUDA-graph plan: V = 1, eps_d = 0.5, beta = 100,
    Gamma = 1, g0 on 100,001 points over [-50, 50] (built on the GPU), charge at t = 50,
    chain [plasma_uv(50), exponential(50, 1)], 2^22 Sobol points per order."""
    from keldy_b200 import capi
    t0 = time.perf_counter()
    model, = capi.flatband_models(ctx, [(1.0, 0.5, 1.0, 100.0)], 50.0, 100001)
    ctx.synchronize()
    build_s = time.perf_counter() - t0
    chain = [(capi.WARPER_PLASMA_UV, 50.0, 0.0), (capi.WARPER_EXPONENTIAL, 50.0, 1.0)]
    orders = list(range(6, 13))
    items = [dict(model=model, rng=ctx.sobol(n), chain=chain, A=(50.0, 0, 0, 0, 0), B=(50.0, 0, 1, 0, 0), order=n,
                  n_points=1 << 22) for n in orders]
    plan = capi.Plan(ctx, items)
    plan.run()
    res = plan.run()
    ms = ctx.last_timing()[0]
    plan.close()
    ref = sum(reference_flops(n) << 22 for n in orders)
    out = {"workload": "biased dot V=1 eps_d=0.5 beta=100, charge G^<(t=50), g0 100,001 points on [-50,50] "
                       "(GPU-built, linear interpolation), chain [plasma_uv(50), exponential(50,1)], "
                       "orders 6..12 x 2^22 Sobol points, one graph launch",
           "ms": ms, "evals_per_s": len(orders) * (1 << 22) / (ms * 1e-3),
           "reference_equivalent_tflops": ref / (ms * 1e-3) / 1e12, "g0_build_s": build_s,
           "charge_by_order": {str(n): [r[0].real / r[1], r[0].imag / r[1]] for n, r in zip(orders, res)},
           "fallback_points": sum(r[3] for r in res)}
    # the same with cubic g0 interpolation (the workload's own setting; no keldy counterpart)
    model.set_interpolation(3)
    plan = capi.Plan(ctx, items)
    plan.run()
    res_c = plan.run()
    ms_c = ctx.last_timing()[0]
    plan.close()
    out["cubic_interpolation"] = {
        "ms": ms_c, "evals_per_s": len(orders) * (1 << 22) / (ms_c * 1e-3),
        "charge_by_order": {str(n): [r[0].real / r[1], r[0].imag / r[1]] for n, r in zip(orders, res_c)},
        "max_abs_diff_vs_linear": max(abs(a[0] / a[1] - b[0] / b[1]) for a, b in zip(res, res_c))}
    return out


def measure_observables(ctx, model, chain, cpu=True):
    """The binned observables on the order-8 workload's model (t = 20): the time-binned charge
    (compute_charge_Q_direct_time: 100 bins of [0, t], order 8, 2^20 points) beside the plain
    integral of the same points, and the kernel method (compute_gf_kernel: fixed point
    (t, up, forward), 100 bins, orders 2..8 x 2^20 points). Device time of the integrand
    kernel (CUDA events); the kernel method's CPU oracle (C restatement, one thread) on a
    bounded sample of each order as its reported baseline."""
    from keldy_b200 import capi
    A, B = (T_MAX, 0, 0, 0, 0), (T_MAX, 0, 1, 0, 0)
    n = 1 << 20
    item = dict(model=model, rng=ctx.sobol(8), chain=chain, A=A, B=B, order=8, k_first=1, n_points=n)
    capi.integrate(ctx, [item])
    capi.integrate(ctx, [item])
    plain_ms = ctx.last_timing()[0]
    capi.integrate_binned(ctx, [item], 100, 0.0, T_MAX)
    binned = capi.integrate_binned(ctx, [item], 100, 0.0, T_MAX)[0]
    binned_ms = ctx.last_timing()[0]
    out = {"time_binned_order8": {"workload": "compute_charge_Q_direct_time, order 8, 2^20 points, 100 bins of "
                                              "[0, 20]", "ms": binned_ms, "evals_per_s": n / (binned_ms * 1e-3),
                                  "plain_ms": plain_ms, "overhead": binned_ms / plain_ms - 1.0,
                                  "bins_sum_minus_total": abs(binned[4].sum() - binned[0])}}
    kern = {}
    oracle = None
    if cpu:
        from oracle.pyoracle import Oracle
        oracle = Oracle()
        _, le, gr = _flatband_tables()
        om = oracle.model(T_MAX, le, gr)
    for order in range(2, 9):
        kit = dict(model=model, rng=ctx.sobol(order), chain=chain, A=A, order=order, k_first=1, n_points=n)
        capi.integrate_kernel(ctx, [kit], 100, 0.0, T_MAX)
        capi.integrate_kernel(ctx, [kit], 100, 0.0, T_MAX)
        ms = ctx.last_timing()[0]
        row = {"ms": ms, "evals_per_s": n / (ms * 1e-3)}
        if oracle is not None:
            m = max(64, int(2e6 / (2 ** order * order ** 3)))
            t0 = time.perf_counter()
            oracle.integrate_kernel(om, A, chain, order, m, 100, 0.0, T_MAX)
            row["cpu_oracle_evals_per_s"] = m / (time.perf_counter() - t0)
            row["cpu_sample_points"] = m
        kern[str(order)] = row
    out["kernel_method"] = {"workload": "compute_gf_kernel at X = (20, up, forward), 100 bins of [0, 20], "
                                        "2^20 points per order", "orders": kern,
                            "cpu": "oracle/keldy_oracle.c or_integrate_kernel, 1 thread (a C restatement)"}
    return out


def _flatband_tables():
    from keldy_b200.g0_tables import flatband
    return flatband(GAMMA, EPS_D, BIAS, BETA, T_MAX, NPTS)


def measure_semicircle_build(ctx):
    """Tables of the dot with semicircular leads (D = 2, Gamma = 1, eps_d = 0.3, V = 0.5,
    beta = 20, t in [-50, 50], 100,001 points, dot and dot-lead blocks): the band
    quadrature's Fourier sums on the GPU (kb_model_set_fourier) and the same sums on the
    host in numpy (g0_tables.semicircle)."""
    from keldy_b200 import capi, g0_tables
    args = (1.0, 0.3, 0.5, 20.0, 2.0, 50.0, 100001)
    capi.semicircle_model(ctx, *args, dot_lead=True).close()  # warm-up
    ctx.synchronize()
    t0 = time.perf_counter()
    m = capi.semicircle_model(ctx, *args, dot_lead=True)
    ctx.synchronize()
    gpu_s = time.perf_counter() - t0
    m.close()
    t0 = time.perf_counter()
    g0_tables.semicircle(*args, dot_lead=True)
    host_s = time.perf_counter() - t0
    nodes = len(g0_tables.semicircle_nodes(*args[:6])[0])
    return {"workload": "semicircular bath D=2 Gamma=1 eps_d=0.3 V=0.5 beta=20, 100,001 points on [-50,50], "
                        f"dot + dot-lead blocks, {nodes} quadrature nodes",
            "gpu_ms": gpu_s * 1e3, "host_numpy_s": host_s}


def measure_sweep(ctx, learned_every=True):
    """256 models (V in [0,2] x eps_d in [-1,1] x beta in {10,50,200}, Gamma = 1), each with
    its own 20,001-point g0 table built on the GPU in one launch; model i integrates order
    2 + i % 9 (uneven costs) with 2^18 Sobol points; all 256 items in one graph launch."""
    import numpy as np
    from keldy_b200 import capi
    params = [(1.0, e, v, b) for b in (10.0, 50.0, 200.0) for v in np.linspace(0.0, 2.0, 8)
              for e in np.linspace(-1.0, 1.0, 11)][:256]
    ctx.synchronize()
    t0 = time.perf_counter()
    models = capi.flatband_models(ctx, params, 20.0, 20001)
    ctx.synchronize()
    build_s = time.perf_counter() - t0
    chain = [(capi.WARPER_PLASMA_UV, 20.0, 0.0), (capi.WARPER_EXPONENTIAL, 20.0, 1.0)]
    rngs = {n: ctx.sobol(n) for n in range(2, 11)}
    items = [dict(model=models[i], rng=rngs[2 + i % 9], chain=chain, A=(20.0, 0, 0, 0, 0), B=(20.0, 0, 1, 0, 0),
                  order=2 + i % 9, n_points=1 << 18) for i in range(len(models))]
    plan = capi.Plan(ctx, items)
    plan.run()
    plan.run()
    ms = ctx.last_timing()[0]
    plan.close()
    ref = sum(reference_flops(it["order"]) << 18 for it in items)
    learned_sweep = measure_sweep_learned(ctx, models, items, chain) if learned_every else None
    for m in models:
        m.close()
    out = {"workload": "256 flat-band models (V in [0,2] x eps_d in [-1,1] x beta in {10,50,200}), own "
                       "20,001-point g0 table each (GPU-built in one launch), orders 2..10 by model, "
                       "2^18 Sobol points per (model, order), one graph launch",
           "ms": ms, "evals_per_s": len(items) * (1 << 18) / (ms * 1e-3),
           "reference_equivalent_tflops": ref / (ms * 1e-3) / 1e12, "g0_build_ms": build_s * 1e3}
    if learned_sweep is not None:
        out["learned_where_trained"] = learned_sweep
    return out


def measure_sweep_learned(ctx, models, items, chain, every=16):
    """The sweep with learned warpers where trained, the plain chain otherwise: a separable
    spline flow is trained for every `every`-th model whose order has flows (up to 8; 2^16
    plain-method samples), kept
    when an RQMC pilot (16 shifts x 2^14 points) shows its standard error below the plain
    chain's, and the 256 items run again as one graph launch with those flows applied in
    line by the integrand kernel."""
    from keldy_b200 import capi, learned
    ctx.synchronize()
    t0 = time.perf_counter()
    flows, kept = {}, []
    for i in range(0, len(items), every):
        it = items[i]
        if it["order"] > 8:
            continue
        fl, _, _ = learned.fit(ctx, models[i], it["A"], it["B"], chain, it["order"], 1 << 16, seed=i,
                               kind=capi.FLOW_SPLINE)
        sel, c = learned.select(ctx, models[i], it["A"], it["B"], chain, it["order"], fl)
        flows[i] = fl
        if sel is not None:
            kept.append((i, it["order"], c["stderr_ratio"]))
    train_s = time.perf_counter() - t0
    keep = {i for i, _, _ in kept}
    litems = [dict(it, flow=flows[i]) if i in keep else it for i, it in enumerate(items)]
    plan = capi.Plan(ctx, litems)
    plan.run()
    plan.run()
    ms = ctx.last_timing()[0]
    plan.close()
    for fl in flows.values():
        fl.close()
    return {"trained": len(flows), "kept": len(kept),
            "kept_models": [{"model": i, "order": n, "pilot_stderr_ratio_plain_over_learned": r} for i, n, r in kept],
            "train_and_select_s": train_s, "ms": ms, "evals_per_s": len(items) * (1 << 18) / (ms * 1e-3),
            "flows": "separable spline flows, mapped in line in the integrand kernel"}


def measure_learned(ctx, model, A, B, chain, orders=(4, 5, 6, 7, 8), ladders=8):
    """Learned flows (coupling layers, the separable spline flow and the autoregressive
    spline flow) vs the plain chain per order: training time, per-point variance gain,
    RQMC standard errors at a fixed 2^24-evaluation budget (16 shifts x 2^20 points) and
    wall time to a 1e-3 (and, at order 6, 1e-4) relative standard error: `ladders`
    independent ladders of 16 shifts each (disjoint shift seeds), points per shift on a
    sqrt(2) grid from 2^8 to 2^20, median and interquartile range over the ladders. The adaptive
    plain warper (make_warper_from_proj: 100 bins per axis, 2^14 samples, sigma 0.05,
    appended to the chain) is measured beside them as the stronger plain baseline."""
    from keldy_b200 import capi, learned, rqmc

    def ladder(ch, n, target, flow=None):
        r = rqmc.time_to_relative_error_ladders(ctx, model, A, B, ch, n, target, ladders=ladders, flow=flow,
                                                max_points=1 << 20)
        return {k: r[k] for k in ("seconds_median", "seconds_iqr", "points_median", "points_iqr", "all_reached")}

    out = {}
    for n in orders:
        flow, fit_s, loss = learned.fit(ctx, model, A, B, chain, n, 1 << 18, seed=n)
        sflow, sfit_s, sloss = learned.fit(ctx, model, A, B, chain, n, 1 << 18, seed=n, kind=capi.FLOW_SPLINE)
        rflow, rfit_s, rloss = learned.fit(ctx, model, A, B, chain, n, 1 << 18, seed=n, kind=capi.FLOW_AR_SPLINE)
        budget = learned.compare(ctx, model, A, B, chain, n, flow, 1 << 20, 16)
        sbudget = learned.compare(ctx, model, A, B, chain, n, sflow, 1 << 20, 16)
        rbudget = learned.compare(ctx, model, A, B, chain, n, rflow, 1 << 20, 16)
        ctx.synchronize()
        t0 = time.perf_counter()
        table = capi.WarperTable.from_projection(ctx, model, A, B, chain, n, 100, 1 << 14, 0.05)
        build_s = time.perf_counter() - t0
        achain = chain + [table.entry()]
        ma, ea, _ = rqmc.estimate(ctx, model, A, B, achain, n, 1 << 20, 16)
        mp = budget["plain"]["mean"]
        targets = (1e-3, 1e-4) if n == 6 else (1e-3,)
        ttr = {}
        for tgt in targets:
            tp, tl, ta = ladder(chain, n, tgt), ladder(chain, n, tgt, flow), ladder(achain, n, tgt)
            ts, tr = ladder(chain, n, tgt, sflow), ladder(chain, n, tgt, rflow)
            ttr[f"{tgt:g}"] = {"plain": tp, "learned": tl, "learned_spline": ts, "learned_ar_spline": tr,
                              "adaptive_plain": ta,
                              "speedup_learned_over_plain": tp["seconds_median"] / tl["seconds_median"],
                              "speedup_spline_over_plain": tp["seconds_median"] / ts["seconds_median"],
                              "speedup_ar_spline_over_plain": tp["seconds_median"] / tr["seconds_median"],
                              "speedup_adaptive_over_plain": tp["seconds_median"] / ta["seconds_median"],
                              "learned_incl_training_s": tl["seconds_median"] + fit_s,
                              "spline_incl_training_s": ts["seconds_median"] + sfit_s,
                              "ar_spline_incl_training_s": tr["seconds_median"] + rfit_s}
        adaptive = {"build_s": build_s, "budget_2e24_stderr": ea, "budget_2e24_rel": ea / abs(ma),
                    "stderr_ratio_plain_over_adaptive": budget["plain"]["stderr"] / ea,
                    "diff_in_combined_sigma": abs(ma - mp) / math.hypot(ea, budget["plain"]["stderr"])}
        table.close()
        out[str(n)] = {
            "fit_s": fit_s, "fit_loss": loss,
            "per_point_variance_gain": learned.variance_gain(ctx, model, A, B, chain, flow),
            "budget_2e24": {"plain_stderr": budget["plain"]["stderr"], "learned_stderr": budget["learned"]["stderr"],
                            "plain_rel": budget["plain"]["rel"], "learned_rel": budget["learned"]["rel"],
                            "stderr_ratio_plain_over_learned": budget["stderr_ratio"],
                            "diff_in_combined_sigma": budget["diff_sigma"],
                            "plain_s": budget["plain"]["seconds"], "learned_s": budget["learned"]["seconds"]},
            "time_to_target": ttr,
            "adaptive_plain": adaptive,
            "learned_spline": {"fit_s": sfit_s, "fit_loss": sloss,
                               "per_point_variance_gain": learned.variance_gain(ctx, model, A, B, chain, sflow),
                               "budget_2e24_stderr": sbudget["learned"]["stderr"],
                               "stderr_ratio_plain_over_spline": sbudget["stderr_ratio"],
                               "diff_in_combined_sigma": sbudget["diff_sigma"]},
            "learned_ar_spline": {"fit_s": rfit_s, "fit_loss": rloss,
                                  "per_point_variance_gain": learned.variance_gain(ctx, model, A, B, chain, rflow),
                                  "budget_2e24_stderr": rbudget["learned"]["stderr"],
                                  "stderr_ratio_plain_over_ar_spline": rbudget["stderr_ratio"],
                                  "diff_in_combined_sigma": rbudget["diff_sigma"]},
        }
        flow.close()
        sflow.close()
        rflow.close()
    return out


def run_ours(args, rank, world, local_rank):
    import numpy as np
    import torch
    torch.cuda.set_device(local_rank)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    from keldy_b200 import capi
    from keldy_b200.g0_tables import flatband

    order, N = args.order, args.points
    ctx = capi.Context(local_rank)
    _, le, gr = flatband(GAMMA, EPS_D, BIAS, BETA, T_MAX, NPTS)
    # pinned host copies of the per-step inputs (end-to-end leg)
    le_pin = torch.empty(2 * NPTS, dtype=torch.float64, pin_memory=True).numpy()
    gr_pin = torch.empty(2 * NPTS, dtype=torch.float64, pin_memory=True).numpy()
    le_pin[:] = le.view(np.float64)
    gr_pin[:] = gr.view(np.float64)
    model = ctx.model(T_MAX, le, gr)
    rng = ctx.sobol(order)
    chain = [(capi.WARPER_PLASMA_UV, T_MAX, 0.0), (capi.WARPER_EXPONENTIAL, T_MAX, 1.0 / GAMMA)]
    A, B = (T_MAX, 0, 0, 0, 0), (T_MAX, 0, 1, 0, 0)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    peak = ctx.fp64_peak()

    def item(step, mdl=model):
        k_first = 1 + ((step * world + rank) * N) % ((1 << 31) - N - 1)
        return dict(model=mdl, rng=rng, chain=chain, A=A, B=B, order=order, k_first=k_first, n_points=N)

    def allreduce(res):
        if world == 1:
            return res
        import torch.distributed as dist
        t = torch.tensor([res[0][0].real, res[0][0].imag, res[0][1], res[0][2]], dtype=torch.float64, device="cuda")
        dist.all_reduce(t)
        return [(complex(t[0].item(), t[1].item()), int(t[2].item()), int(t[3].item()), res[0][3])]

    ctx.set_timing(True)
    from keldy_b200 import autotune
    tuned = autotune.tune(ctx, orders=sorted({order} | set(range(1, 11))), repeats=2)
    autotune.apply(ctx, tuned)
    plan = capi.Plan(ctx, [item(0)])
    sampler = ClockSampler(local_rank)
    sampler.start()
    for s in range(args.warmup):
        plan.set_k_first(0, item(s)["k_first"])
        allreduce(plan.run())

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize()

    barrier()
    w0 = sampler.mark()
    dev_ms, integ_ms, launches, in_domain, fallback = 0.0, 0.0, 0, 0, 0
    for s in range(args.steps):
        flush.fill_(s & 0xFF)
        torch.cuda.synchronize()
        plan.set_k_first(0, item(args.warmup + s)["k_first"])
        res = allreduce(plan.run())
        a = ctx.last_timing()[0]
        dev_ms += a
        integ_ms += a
        launches += 3  # tree kernel, guarded-pivot pass, reduction (one graph)
        in_domain += res[0][2]
        fallback += res[0][3]
    barrier()
    w1 = sampler.mark()
    plan.close()
    # end to end through the public API with host buffers: per step, upload the g0
    # tables from pinned memory (kb_model_set_table), integrate, read the sums back. The
    # K steps run E2E_REPEATS times; the median run is reported with all of them listed.
    m2 = capi.Model(ctx, T_MAX, le_pin.view(np.complex128), gr_pin.view(np.complex128))
    e2e_runs = []
    for r in range(E2E_REPEATS):
        barrier()
        t0 = time.perf_counter()
        for s in range(args.steps):
            m2.set_table(0, 0, 0, le_pin.view(np.complex128), gr_pin.view(np.complex128))
            allreduce(capi.integrate(ctx, [item(args.warmup + (1 + r) * args.steps + s, m2)]))
        barrier()
        e2e_runs.append(time.perf_counter() - t0)
    e2e_s = statistics.median(e2e_runs)
    sampler.stop()
    clocks = sampler.summary(w0, max(w1, w0 + 1))
    clocks["e2e"] = sampler.summary(w1)

    t_max_ms = dev_ms
    e2e_max = e2e_s
    integ_max = integ_ms
    if world > 1:
        import torch.distributed as dist
        v = torch.tensor([dev_ms, e2e_s, integ_ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(v, op=dist.ReduceOp.MAX)
        t_max_ms, e2e_max, integ_max = v.tolist()

    total_points = world * N * args.steps
    value = total_points / (t_max_ms * 1e-3)
    line = None
    if rank == 0:
        # batched launch: orders 1..10, 2^20 points each, one plan (one graph launch)
        rngs = {n: ctx.sobol(n) for n in range(1, 11)}
        batch = [dict(model=model, rng=rngs[n], chain=chain, A=A, B=B, order=n, k_first=1, n_points=1 << 20)
                 for n in range(1, 11)]
        bplan = capi.Plan(ctx, batch)
        bplan.run()
        bt = []
        for _ in range(2):
            bplan.run()
            bt.append(ctx.last_timing()[0])
        bplan.close()
        b_ms = min(bt)
        b_ref_flop = sum(reference_flops(n) << 20 for n in range(1, 11))
        ref_flop_launch = N * reference_flops(order)
        achieved = ref_flop_launch / (integ_max * 1e-3 / args.steps)
        cpu = None
        if world == 1 and not args.no_cpu:
            cref = CpuReference(order)
            cpu = cref.measure(cref.sample_size(10.0))
        h2d = 2 * NPTS * 16 + 8 * 1024
        src_hash = tree_source_hash()
        traffic = TREE_DRAM_CAPTURES.get(src_hash) if (order == 8 and N == 1 << 20) else None
        traffic_source = (f"dram__bytes_read.sum + dram__bytes_write.sum of one 2^20-point order-8 tree_kernel launch "
                          f"(ncu) of the kernel sources with hash {src_hash}: the g0 table and set-up data read once, "
                          f"and the part of the staged G matrices (4.6 KB per evaluation) that L2 writes back; the "
                          f"table gathers are served by L2/L1"
                          if traffic is not None else
                          f"no ncu capture of the kernel sources with hash {src_hash} at this workload")
        line = {
            "metric": f"integrand evals/s at order {order}", "value": value, "unit": "evals/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_max_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(order, N),
            "e2e": {"value": total_points / e2e_max, "unit": "evals/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": 40, "statistic": f"median of {E2E_REPEATS} runs of the K steps",
                    "runs_evals_per_s": [total_points / t for t in e2e_runs]},
            "gpu_launches": launches,
            "roofline": {"bound": "fp64", "achieved": achieved / 1e12, "peak": peak / 1e12, "unit": "TFLOP/s",
                         "frac": achieved / peak,
                         "executed_frac": N * tree_flops(order) / (integ_max * 1e-3 / args.steps) / peak,
                         "traffic": traffic,
                         "traffic_source": traffic_source,
                         "numerator": f"reference-equivalent: {reference_flops(order)} FLOP per evaluation "
                                      f"(keldy's 2^n LU pairs); the tree executes ~{tree_flops(order)}",
                         "peak_source": "FP64 FMA rate measured in this run (kb_fp64_peak, 8 independent "
                                        "chains per thread); MEASURED_PEAKS.json has no FP64 figure",
                         "executed_tflops": N * tree_flops(order) / (integ_max * 1e-3 / args.steps) / 1e12,
                         "kernel_ms": integ_max / args.steps},
            "in_domain_evals_per_s": in_domain / (t_max_ms * 1e-3),
            "fallback_points": fallback,
            "batched_orders_1_10": {"ms": b_ms, "evals_per_s": 10 * (1 << 20) / (b_ms * 1e-3),
                                    "reference_equivalent_tflops": b_ref_flop / (b_ms * 1e-3) / 1e12,
                                    "launch": "one CUDA-graph plan over the ten orders"},
            "launch_shape": {str(k): {"chunk_points": v["chunk_points"], "ctas_per_sm": v["ctas_per_sm"]}
                             for k, v in tuned.items()},
            "clocks": clocks,
        }
        if not args.no_extras:
            line["biased_dot_orders_6_12"] = measure_biased_dot(ctx)
            line["sweep_256_models"] = measure_sweep(ctx)
            line["semicircle_g0_build"] = measure_semicircle_build(ctx)
            line["binned_observables"] = measure_observables(ctx, model, chain, cpu=not args.no_cpu)
            line["learned_vs_plain"] = measure_learned(ctx, model, A, B, chain)
        if cpu is not None:
            line["cpu_baseline"] = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")}
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    ctx.close()


def run_single(args):
    from keldy_b200 import capi
    from keldy_b200.g0_tables import flatband
    ctx = capi.Context(0)
    _, le, gr = flatband(GAMMA, EPS_D, BIAS, BETA, T_MAX, NPTS)
    model = ctx.model(T_MAX, le, gr)
    chain = [(capi.WARPER_PLASMA_UV, T_MAX, 0.0), (capi.WARPER_EXPONENTIAL, T_MAX, 1.0 / GAMMA)]
    res = capi.integrate(ctx, [dict(model=model, rng=ctx.sobol(args.order), chain=chain, A=(T_MAX, 0, 0, 0, 0),
                                    B=(T_MAX, 0, 1, 0, 0), order=args.order, k_first=1, n_points=args.points)])
    print("single", args.order, args.points, res[0])
    if args.single_flow:
        # a learned flow of the same order: one epoch of training (flow_train_kernel), then
        # the same integration through it (flow_map_kernel)
        flow = ctx.flow(args.order, seed=1)
        loss = flow.fit(model, (T_MAX, 0, 0, 0, 0), (T_MAX, 0, 1, 0, 0), chain, ctx.sobol(args.order), 1 << 16,
                        epochs=1, batch=8192)
        res = capi.integrate(ctx, [dict(model=model, rng=ctx.sobol(args.order), chain=chain, A=(T_MAX, 0, 0, 0, 0),
                                        B=(T_MAX, 0, 1, 0, 0), order=args.order, k_first=1, n_points=args.points,
                                        flow=flow)])
        print("single-flow", args.order, args.points, loss, res[0])
    if args.single_kernel:
        # the kernel method at the same order: one km_tree_kernel launch
        res = capi.integrate_kernel(ctx, [dict(model=model, rng=ctx.sobol(args.order), chain=chain,
                                               A=(T_MAX, 0, 0, 0, 0), order=args.order, k_first=1,
                                               n_points=args.points)], 100, 0.0, T_MAX)
        print("single-kernel", args.order, args.points, res[0][0])
    ctx.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--order", type=int, default=8)
    ap.add_argument("--points", type=int, default=1 << 20)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the biased-dot, 256-model sweep and learned-warper measurements")
    ap.add_argument("--ref-seconds", type=float, default=2.0, help="seconds of CPU work per reference-arm step")
    ap.add_argument("--single", action="store_true",
                    help="one integrate call of --points points at --order and exit (for profiler captures)")
    ap.add_argument("--single-kernel", action="store_true",
                    help="with --single: also one kernel-method integration (compute_gf_kernel) of the same size")
    ap.add_argument("--single-flow", action="store_true",
                    help="with --single: also train a learned flow for one epoch and integrate through it")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.single:
        run_single(args)
    elif args.impl == "reference":
        run_reference_arm(args, rank, world)
    else:
        run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
