"""The time-binned direct integrand (keldy's integrand_g_direct_time with
compute_charge_Q_direct_time, wick_direct_time.cpp:42-163, compute_obs.hpp:85-101):
each point's f*J binned by its earliest vertex time. Against the oracle's restatement bin
by bin, and keldy's own consistency checks (wick_direct_time_test.cpp: the bins sum to
the direct charge)."""
import numpy as np
import pytest

from keldy_b200 import capi, impurity_oneband as io, warpers
from tests.golden.make_golden import EXTERNALS

pytestmark = pytest.mark.gpu

CHARGE = (EXTERNALS[0][1], EXTERNALS[0][2])
PLASMA_EXP = [(capi.WARPER_PLASMA_UV, 10.0, 0.0), (capi.WARPER_EXPONENTIAL, 10.0, 1.0)]
UNIFORM = [(capi.WARPER_UNIFORM, 10.0, 0.0)]


def _item(model, rng, chain, order, n, A=CHARGE[0], B=CHARGE[1]):
    return dict(model=model, rng=rng, chain=chain, A=A, B=B, order=order, k_first=1, n_points=n)


@pytest.mark.parametrize("nbins,xmin,xmax", [(10, 0.0, 10.0), (7, 1.0, 6.5), (1, 0.0, 10.0), (600, 0.0, 10.0)])
def test_bins_vs_oracle(ctx, oracle, golden, nbins, xmin, xmax):
    le, gr = golden["table_beta20_lesser"], golden["table_beta20_greater"]
    gm = ctx.model(10.0, le, gr)
    om = oracle.model(10.0, le, gr)
    for chain in (PLASMA_EXP, UNIFORM):
        for n in (1, 2, 4, 6):
            npts = 2048 if n <= 4 else 256
            s, npt, nd, _, bins, counts, dropped = capi.integrate_binned(
                ctx, [_item(gm, ctx.sobol(n), chain, n, npts)], nbins, xmin, xmax)[0]
            ws, onp, ond, sc, obins, ocounts, odropped = oracle.integrate_binned(om, CHARGE[0], CHARGE[1], chain, n,
                                                                                 npts, nbins, xmin, xmax)
            assert (npt, nd) == (onp, ond)
            assert np.array_equal(counts, ocounts) and dropped == odropped, (n, counts, ocounts)
            assert np.abs(bins - obins).max() <= 1e-12 * sc
            assert abs(s - ws) <= 1e-12 * sc


def test_bins_sum_to_the_direct_charge(ctx, golden):
    le, gr = golden["table_beta20_lesser"], golden["table_beta20_greater"]
    gm = ctx.model(10.0, le, gr)
    for n in (3, 5, 8):
        item = _item(gm, ctx.sobol(n), PLASMA_EXP, n, 5000)
        direct = capi.integrate(ctx, [item])[0]
        s, npt, nd, _, bins, counts, dropped = capi.integrate_binned(ctx, [item], 10, 0.0, 10.0)[0]
        assert (s, npt, nd) == direct[:3]
        assert counts.sum() + dropped == npt
        scale = np.abs(gm.evaluate_warped(CHARGE[0], CHARGE[1], PLASMA_EXP, ctx.sobol(n).points(1, 5000))[0]).sum()
        assert abs(bins.sum() - s) <= 1e-12 * scale


def test_compute_charge_q_direct_time_like_keldy(golden):
    """wick_direct_time_test.cpp:63-88: the bins of compute_charge_Q_direct_time sum to
    compute_charge_Q_direct's result (same warpers, same points)."""
    model = io.from_tables(10.0, golden["table_beta20_lesser"], golden["table_beta20_greater"])
    direct = io.ComputeChargeQDirect(model, 10.0, 4, 0.0)
    binned = io.ComputeChargeQDirectTime(model, 10.0, 4, 10, 0.0)
    for c in (direct, binned):
        c.warper.emplace_back(warpers.WarperPlasmaUvT(10.0))
        c.warper.emplace_back(warpers.make_product_1d_simple_exponential(10.0, 1.0))
        c.run(10)
        c.run(1000)
    res = binned.reduce_result()
    assert res.get_nr_bins() == 10 and abs(res.get_bin_size() - 1.0) < 1e-15
    assert np.allclose(res.get_bin_coord(), np.arange(10) + 0.5)
    assert sum(res.get_nr_values_added()) + res.get_nr_values_dropped() == 1010
    assert abs(sum(res.get_data()) - direct.reduce_result()) <= 1e-14 * abs(direct.reduce_result())


def test_binning_errors(ctx, golden):
    gm = ctx.model(10.0, golden["table_beta20_lesser"], golden["table_beta20_greater"])
    item = _item(gm, ctx.sobol(2), PLASMA_EXP, 2, 10)
    with pytest.raises(capi.KbError, match="wrong order"):
        capi.integrate_binned(ctx, [item], 10, 5.0, 5.0)
    with pytest.raises(capi.KbError):
        capi.integrate_binned(ctx, [item], 0, 0.0, 1.0)
    with pytest.raises(RuntimeError, match="wrong order"):
        io.BinnerT1(2.0, 1.0, 5)


def test_bins_with_a_flow_and_pivoted_lu(ctx, golden):
    """Items through a learned flow and through the pivoted-LU algorithm bin the same way
    as the tree's plain items."""
    le, gr = golden["table_beta20_lesser"], golden["table_beta20_greater"]
    gm = ctx.model(10.0, le, gr)
    item = _item(gm, ctx.sobol(4), PLASMA_EXP, 4, 3000)
    base = capi.integrate_binned(ctx, [item], 8, 0.0, 10.0)[0]
    flow = capi.integrate_binned(ctx, [dict(item, flow=ctx.flow(4))], 8, 0.0, 10.0)[0]
    lu = capi.integrate_binned(ctx, [item], 8, 0.0, 10.0, algo=capi.ALGO_DIRECT)[0]
    for other in (flow, lu):
        assert np.array_equal(other[5], base[5]) and other[6] == base[6], (other[:4], other[6], base[:4], base[6])
        assert np.abs(other[4] - base[4]).max() <= 1e-12 * np.abs(base[4]).sum()


def test_bins_with_guarded_pivots(ctx, oracle):
    """A table that vanishes at t = 0 sends every point to the pivoted-LU pass; their
    values still land in their bins."""
    t = np.linspace(-10, 10, 2001)
    le = 1j * t * np.exp(-t * t / 8) + 0.2 * np.sin(t)
    gr = -np.conj(le[::-1])
    gm = ctx.model(10.0, le, gr)
    om = oracle.model(10.0, le, gr)
    for n in (3, 5):
        s, npt, nd, nfb, bins, counts, dropped = capi.integrate_binned(
            ctx, [_item(gm, ctx.sobol(n), PLASMA_EXP, n, 300)], 6, 0.0, 10.0)[0]
        ws, _, ond, sc, obins, ocounts, odropped = oracle.integrate_binned(om, CHARGE[0], CHARGE[1], PLASMA_EXP, n, 300,
                                                                           6, 0.0, 10.0)
        assert nfb > 0 and nd == ond
        assert np.array_equal(counts, ocounts) and dropped == odropped
        assert np.abs(bins - obins).max() <= 1e-12 * sc
