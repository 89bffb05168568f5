"""Sobol points, warper chains and the g0 contour adaptor on the GPU, through the C ABI,
against keldy's own outputs (golden.npz) and the CPU oracle."""
import numpy as np
import pytest

from keldy_b200 import capi
from tests.golden.make_golden import CHAINS, SOBOL_CASES, SOBOL_COUNT

pytestmark = pytest.mark.gpu


def test_sobol_bit_exact_vs_keldy(ctx, golden):
    for i, (dim, seed, sh, sc, ss) in enumerate(SOBOL_CASES):
        s = ctx.sobol(dim, 31, bool(sh), bool(sc), ss)
        got = s.points(seed + 1, SOBOL_COUNT)  # keldy's sobol(dim, seed) first draws k = seed+1
        assert np.array_equal(got, golden[f"sobol_{i}"]), (dim, seed, sh, sc, ss)


def test_sobol_far_indices_and_short_sequences(ctx, oracle):
    for dim, m, sh, sc, ss, k0 in [(12, 31, 0, 0, 0, (1 << 31) - 300), (9, 20, 1, 1, 6, (1 << 20) - 100),
                                   (16, 31, 1, 0, 2, 123456789)]:
        got = ctx.sobol(dim, m, bool(sh), bool(sc), ss).points(k0, 99)
        want = oracle.sobol_points(dim, k0 - 1, 99, bool(sh), bool(sc), ss, log_max_points=m)
        assert np.array_equal(got, want)


def test_sobol_last_points(ctx, oracle):
    # keldy checks past_end() before next(): with 2^m points, k = 2^m is the last one drawn
    for dim, m, sh, sc in [(5, 10, 0, 0), (7, 12, 1, 1)]:
        got = ctx.sobol(dim, m, bool(sh), bool(sc), 4).points((1 << m) - 3, 4)
        want = oracle.sobol_points(dim, (1 << m) - 4, 4, bool(sh), bool(sc), 4, log_max_points=m)
        assert np.array_equal(got, want)


def test_sobol_errors(ctx):
    s = ctx.sobol(4, 10)
    with pytest.raises(capi.KbError) as e:
        s.points((1 << 10) - 5, 10)  # past the last point: keldy's "More sample points requested"
    assert e.value.code == capi.KB_E_EXHAUSTED
    with pytest.raises(capi.KbError):
        s.points(0, 1)
    with pytest.raises(capi.KbError):
        ctx.sobol(4, 32)
    with pytest.raises(capi.KbError):
        ctx.sobol(251)


def _close(a, b, rtol=1e-12):
    a, b = np.asarray(a), np.asarray(b)
    return np.all(np.abs(a - b) <= rtol * np.maximum(np.abs(b), 1.0))


@pytest.mark.parametrize("name", sorted(CHAINS))
def test_warpers_vs_keldy(ctx, golden, name):
    chain = CHAINS[name]
    u, j = ctx.warp(chain, golden[f"warp_{name}_li"], capi.REVERSE)
    assert _close(u, golden[f"warp_{name}_ui"]) and _close(j, golden[f"warp_{name}_jr"])
    l, jf = ctx.warp(chain, golden[f"warp_{name}_fin"], capi.FORWARD)
    assert _close(l, golden[f"warp_{name}_fout"]) and _close(jf, golden[f"warp_{name}_jf"])


def test_warper_partial_chain(ctx, oracle):
    chain = [(capi.WARPER_INVERSE, 10.0, 1.0), (capi.WARPER_PLASMA_UV, 10.0, 0.0), (capi.WARPER_EXPONENTIAL, 1.0, 1.0)]
    x = np.random.default_rng(3).random((50, 5))
    for start, end in [(3, 0), (2, 0), (3, 1), (1, 1), (2, 1)]:
        u, j = ctx.warp(chain, x, capi.REVERSE, start, end)
        uo, jo = oracle.warp(chain, x, "reverse", start, end)
        assert _close(u, uo) and _close(j, jo)


def test_warper_errors(ctx):
    with pytest.raises(capi.KbError):
        ctx.warp([(capi.WARPER_EXPONENTIAL, -1.0, 1.0)], np.zeros((1, 2)))
    with pytest.raises(capi.KbError):
        ctx.warp([(capi.WARPER_IDENTITY, 0, 0)], np.zeros((1, 2)), capi.REVERSE, 2, 0)


def _random_indices(rng, n, time_max):
    idx = []
    for _ in range(n):
        t = rng.choice([rng.random() * time_max, 0.0, time_max, 3.0])
        idx.append((float(t), int(rng.integers(0, 2)), int(rng.integers(0, 2)), int(rng.integers(0, 3)), 0))
    return idx


def test_g0_adaptor_bit_exact(ctx, oracle, golden):
    rng = np.random.default_rng(11)
    for tname in ("T0", "beta20"):
        le, gr = golden[f"table_{tname}_lesser"], golden[f"table_{tname}_greater"]
        for alpha in (0.0, 0.8):
            gm = ctx.model(10.0, le, gr, alpha)
            om = oracle.model(10.0, le, gr, alpha)
            a = _random_indices(rng, 300, 10.0)
            b = _random_indices(rng, 300, 10.0)
            b[:40] = a[:40]  # equal contour points
            internal = rng.integers(0, 2, 300)
            got = gm.g0(a, b, internal)
            want = np.array([oracle.g0(om, x, y, bool(i)) for x, y, i in zip(a, b, internal)])
            assert np.array_equal(got, want)


def test_g0_out_of_window(ctx, golden):
    gm = ctx.model(10.0, golden["table_T0_lesser"], golden["table_T0_greater"])
    with pytest.raises(capi.KbError) as e:
        gm.g0([(10.5, 0, 0, 0, 0)], [(0.0, 0, 0, 0, 0)])
    assert e.value.code == capi.KB_E_RANGE
