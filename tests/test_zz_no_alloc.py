"""kb_integrate_noalloc: the integrate path for callers that cannot call cudaMalloc
(a host application whose own allocator owns the device's memory, or a latency-bound
loop that must not pay cudaMalloc's implicit synchronisation). Its scratch is a fixed
device array inside the library, so its sums must equal kb_integrate's, call after call.

Collected last on purpose: the array is shared by all calls and keeps the previous call's
contents, so the test runs both in a fresh process and after every other test.
"""
import numpy as np
import pytest

from keldy_b200 import capi
from keldy_b200.g0_tables import flatband

pytestmark = pytest.mark.gpu

PLASMA_EXP = [(capi.WARPER_PLASMA_UV, 10.0, 0.0), (capi.WARPER_EXPONENTIAL, 10.0, 1.0)]


def _items(ctx):
    _, le, gr = flatband(1.0, 0.2, 0.5, 20.0, 10.0, 4001)
    sym = ctx.model(10.0, le, gr)
    asym = ctx.model(10.0, le, gr, 0.0, 0.5 * le, 0.5 * gr)  # different spin-down tables: pivoted-LU group
    items = []
    for n in range(1, 8):
        items.append(dict(model=sym, rng=ctx.sobol(n), chain=PLASMA_EXP, A=(10.0, 0, 0), B=(10.0, 0, 1), order=n,
                          k_first=1 + 3 * n, n_points=1500 + 211 * n))
    items.append(dict(model=asym, rng=ctx.sobol(3, 31, True, True, 5), chain=PLASMA_EXP, A=(10.0, 0, 0),
                      B=(10.0, 0, 1), order=3, k_first=1, n_points=700))
    return items, (sym, asym)


def _scale(ctx, it):
    """sum over the points of |f J| (the tolerance scale of a QMC sum)."""
    li = it["rng"].points(it["k_first"], it["n_points"])[:, :it["order"]]
    v, _, _ = it["model"].evaluate_warped(it["A"], it["B"], it["chain"], li)
    return np.abs(v).sum()


def test_noalloc_equals_integrate_twice(ctx):
    items, keep = _items(ctx)
    want = capi.integrate(ctx, items)
    scales = [_scale(ctx, it) for it in items]
    for call in range(2):  # two calls in a row: the shared scratch must not leak between them
        got = capi.integrate_noalloc(ctx, items)
        for (s, n, d, fb), (ws, wn, wd, wfb), sc in zip(got, want, scales):
            assert (n, d, fb) == (wn, wd, wfb)
            assert abs(s - ws) <= 1e-12 * sc, (call, abs(s - ws) / sc)


def test_noalloc_allocates_nothing(ctx):
    """The defining property: after a first call (which looks up the array's address), a
    call makes no device allocation at all, while kb_integrate does."""
    items, keep = _items(ctx)
    capi.integrate_noalloc(ctx, items)
    before = capi.device_allocations()
    capi.integrate_noalloc(ctx, items)
    capi.integrate_noalloc(ctx, items)
    assert capi.device_allocations() == before
    capi.integrate(ctx, items[:1])
    assert capi.device_allocations() > before


def test_noalloc_follows_the_launch_shape(ctx):
    """With a non-default launch shape (chunk size, CTAs per SM) both entry points split the
    points into the same chunks and add them in the same order: equal sums."""
    items, keep = _items(ctx)
    saved = {n: ctx.get_launch(n) for n in range(1, 8)}
    try:
        ctx.set_launch(-1, 48, 1)
        want = capi.integrate(ctx, items)
        assert capi.integrate_noalloc(ctx, items) == want
    finally:
        for n, (cp, k) in saved.items():
            ctx.set_launch(n, cp, k)


def test_noalloc_limits(ctx):
    items, keep = _items(ctx)
    with pytest.raises(capi.KbError) as e:
        capi.integrate_noalloc(ctx, [dict(items[0], n_points=capi.NOALLOC_MAX_CHUNKS * 128 + 1)])
    assert e.value.code == capi.KB_E_INVALID and "scheduling chunks in" in str(e.value)
    with pytest.raises(capi.KbError) as e:
        capi.integrate_noalloc(ctx, [items[0]] * (capi.NOALLOC_MAX_ITEMS + 1))
    assert e.value.code == capi.KB_E_INVALID
