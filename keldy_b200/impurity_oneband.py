"""keldy.impurity_oneband (python/keldy/impurity_oneband_desc.py) on keldy_b200.

The model parameters are a dict with keldy's keys and defaults (model_param_t,
model.hpp:37-50). G0Model builds the g0 tables on the host (keldy_b200.g0_tables) and
uploads them; everything downstream (g0 contour adaptor, Wick-determinant integrand,
integrators) runs on the GPU.
"""
from __future__ import annotations

import math
import warnings

import numpy as np

from . import g0_tables
from ._keldy import (BinnerT1, BinnerT11, ComputeGfKernel as _ComputeGfKernel, IntegrandGKernel,  # noqa: F401
                     ComputeGfKernelSingleOmega as _ComputeGfKernelSingleOmega, IntegrandGKernelSingleOmega,
                     ComputeChargeQDirect as _ComputeChargeQDirect,
                     ComputeChargeQDirectTime as _ComputeChargeQDirectTime,
                     ComputeCurrentJDirect as _ComputeCurrentJDirect, FT_MIRROR, FT_SYMMETRIC, G0KeldyshContourT,
                     G0ModelTables, GfIndexT, IntegrandGDirect)

MODEL_PARAM_DEFAULTS = {
    "beta": 1.0,
    "bias_V": 0.0,
    "eps_d": 0.0,
    "Gamma": 1.0,
    "alpha": 0.0,
    "half_bandwidth": 2.0,
    "bath_type": "semicircle",
    "time_max": 100.0,
    "nr_time_points_gf": 1000,
    "ft_method": "fft",
}


def model_param_t(params=None, **kw):
    """keldy's model_param_t as a dict: defaults, then `params`, then keywords. Unknown keys
    raise, as the cpp2py converter does."""
    p = dict(MODEL_PARAM_DEFAULTS)
    for src in (params or {}), kw:
        for k, v in src.items():
            if k not in MODEL_PARAM_DEFAULTS:
                raise KeyError(f"model_param_t has no member '{k}'")
            p[k] = v
    return p


def G0Model(params=None, make_dot_lead=False, **kw):
    """g0_model{g0_model_omega{params}, make_dot_lead} (model.cpp:79-177): the lesser and
    greater tables on [-time_max, time_max], spin up = spin down.

    ft_method "fft" (keldy's default, make_g0_by_fft, model.cpp:179-212), any bath: keldy's
    frequency functions on the mesh adjoint to the time mesh (g0_tables.fft_samples, on the
    host) and their discrete transform on the GPU (kb_model_set_fft), with the dot-lead
    blocks when make_dot_lead. ft_method "contour": flatband in closed form; semicircle by
    the band integral of keldy's finite-contour method (Fourier sums on the GPU);
    lorentzian in closed form from the poles of its rational functions (on the GPU); with the
    dot-lead blocks when make_dot_lead.
    ft_method "analytic": keldy's zero-temperature flat-band formula and its restrictions."""
    p = model_param_t(params, **kw)
    beta = float(p["beta"])
    if beta < 0:
        warnings.warn("beta < 0. Interpret this as beta = +infinity.")
        beta = math.inf
    npts = int(p["nr_time_points_gf"])
    if npts % 2 == 0:
        warnings.warn("number of time points has been increased to make it odd.")
        npts += 1
    bath, ft = p["bath_type"], p["ft_method"]
    if bath not in ("semicircle", "flatband", "lorentzian"):
        raise RuntimeError("bath_type not defined")
    if ft not in ("fft", "contour", "analytic"):
        raise RuntimeError(f"ft_method '{ft}' is not defined")
    blocks = {}
    if bath == "flatband" and make_dot_lead:
        raise RuntimeError("The dot-lead g0 for flatband bath is singular and not implemented accurately.")
    if ft == "fft":
        samples = g0_tables.fft_samples(bath, p["Gamma"], p["eps_d"], p["bias_V"], beta, p["half_bandwidth"],
                                        p["time_max"], npts, dot_lead=make_dot_lead)
        g = G0ModelTables.empty(float(p["time_max"]), npts, float(p["alpha"]))
        g.set_fft(0, 0, *samples[(0, 0)])
        if make_dot_lead:
            g.set_fft(1, 0, *samples[(1, 0)], FT_MIRROR)
        g.make_dot_lead = bool(make_dot_lead)
        g.param = dict(p)
        g.g0_lesser, g.g0_greater = g.get_table(0, 0, 0)
        return g
    if bath == "flatband":
        if make_dot_lead:
            raise RuntimeError("The dot-lead g0 for flatband bath is singular and not implemented accurately.")
        if ft == "analytic":
            if math.isfinite(beta) or p["bias_V"] != 0.0 or p["eps_d"] != 0.0:
                raise RuntimeError("Analytic flatband covers only the following parameters: beta=infinity (zero "
                                   "temperature), bias_V=0, eps_d=0.")
            _, le, gr = g0_tables.flatband_analytic(p["Gamma"], p["time_max"], npts)
        else:
            _, le, gr = g0_tables.flatband(p["Gamma"], p["eps_d"], p["bias_V"], beta, p["time_max"], npts)
    elif bath == "semicircle":
        if ft == "analytic":
            raise RuntimeError("analytic ft only works for flatband")
        # the band quadrature's nodes on the host, its Fourier sums on the GPU
        w, f_less, f_great, f_l10, f_g10 = g0_tables.semicircle_nodes(p["Gamma"], p["eps_d"], p["bias_V"], beta,
                                                                      p["half_bandwidth"], p["time_max"])
        g = G0ModelTables.empty(float(p["time_max"]), npts, float(p["alpha"]))
        g.set_fourier(0, 0, w, f_less, f_great, FT_SYMMETRIC)
        if make_dot_lead:
            g.set_fourier(1, 0, w, f_l10, f_g10, FT_MIRROR)
        g.make_dot_lead = bool(make_dot_lead)
        g.param = dict(p)
        g.g0_lesser, g.g0_greater = g.get_table(0, 0, 0)
        return g
    else:
        if ft == "analytic":
            raise RuntimeError("analytic ft only works for flatband")
        # lorentzian, "contour": the transform keldy's contour integral computes, in closed form
        # from the poles of the bath's rational functions (kb_model_set_rational)
        terms = g0_tables.rational_terms(bath, p["Gamma"], p["eps_d"], p["bias_V"], p["half_bandwidth"],
                                         dot_lead=make_dot_lead)
        g = G0ModelTables.empty(float(p["time_max"]), npts, float(p["alpha"]))
        g.set_rational(0, 0, [tuple(t) for t in terms[(0, 0)]], beta, FT_SYMMETRIC)
        if make_dot_lead:
            g.set_rational(1, 0, [tuple(t) for t in terms[(1, 0)]], beta, FT_MIRROR)
        g.make_dot_lead = bool(make_dot_lead)
        g.param = dict(p)
        g.g0_lesser, g.g0_greater = g.get_table(0, 0, 0)
        return g
    return from_tables(p["time_max"], le, gr, p["alpha"], blocks=blocks, make_dot_lead=make_dot_lead, param=p)


def from_tables(time_max, lesser, greater, alpha=0.0, blocks=None, make_dot_lead=False, param=None,
                lesser_down=None, greater_down=None):
    """A G0Model from given tables on the uniform mesh [-time_max, time_max]: spin-up
    (0,0) block, optional dot-lead blocks {(o1, o2): (lesser, greater)} (applied to both
    spins) and optional different spin-down (0,0) tables."""
    g = G0ModelTables.from_tables(float(time_max), np.asarray(lesser, np.complex128),
                                  np.asarray(greater, np.complex128), float(alpha))
    for (o1, o2), (le, gr) in (blocks or {}).items():
        for spin in (0, 1):
            g.set_table(spin, o1, o2, np.asarray(le, np.complex128), np.asarray(gr, np.complex128))
    if lesser_down is not None:
        g.set_table(1, 0, 0, np.asarray(lesser_down, np.complex128), np.asarray(greater_down, np.complex128))
    g.make_dot_lead = bool(make_dot_lead)
    g.param = dict(param) if param else model_param_t(time_max=time_max, alpha=alpha,
                                                       nr_time_points_gf=len(lesser))
    g.g0_lesser = np.asarray(lesser, np.complex128)
    g.g0_greater = np.asarray(greater, np.complex128)
    return g


G0Model.from_tables = from_tables


def _model(m, make_dot_lead):
    return m if isinstance(m, G0ModelTables) else G0Model(m, make_dot_lead)


def ComputeChargeQDirect(model, time, order, cutoff_integrand):
    """compute_charge_Q_direct(model or params, time, order, cutoff) (compute_obs.hpp:51-64)."""
    return _ComputeChargeQDirect(_model(model, False), float(time), int(order), float(cutoff_integrand))


def ComputeChargeQDirectTime(model, time, order, nr_time_slices, cutoff_integrand):
    """compute_charge_Q_direct_time(model or params, time, order, nr_time_slices, cutoff)
    (compute_obs.hpp:85-101): the charge binned by the earliest vertex time over [0, time];
    reduce_result() returns the binner (BinnerT1)."""
    return _ComputeChargeQDirectTime(_model(model, False), float(time), int(order), int(nr_time_slices),
                                     float(cutoff_integrand))


def ComputeGfKernel(model, time, order, nr_bins=100):
    """compute_gf_kernel(model or params, time, order, nr_bins) (compute_obs.hpp:105-117): G(t)
    by the kernel method, binned over [0, time] x Keldysh index; reduce_result() returns the
    binner (BinnerT11; get_data() gives the [nr_bins][2] array)."""
    return _ComputeGfKernel(_model(model, False), float(time), int(order), int(nr_bins))


def ComputeGfKernelSingleOmega(model, time, omega, order):
    """compute_gf_kernel_single_omega(model or params, time, omega, order)
    (compute_obs.hpp:119-133): the kernel method's G at frequency omega; reduce_result()
    returns the complex mean."""
    return _ComputeGfKernelSingleOmega(_model(model, False), float(time), float(omega), int(order))


def binner_data(b):
    """The [nr_bins][2] data of a BinnerT11 (or [nr_bins] of a BinnerT1) as a numpy array."""
    if isinstance(b, BinnerT11):
        return np.array(b.get_data_flat()).reshape(b.get_nr_bins(), 2)
    return np.array(b.get_data())


def ComputeCurrentJDirect(model, time, order, cutoff_integrand):
    """compute_current_J_direct(model or params, time, order, cutoff) (compute_obs.hpp:66-80)."""
    m = _model(model, True)
    if not m.make_dot_lead:
        raise RuntimeError("Need g0_model with make_dot_lead == true to calculate off_diagonal gf.")
    return _ComputeCurrentJDirect(m, float(time), int(order), float(cutoff_integrand))


__all__ = ["GfIndexT", "G0Model", "G0KeldyshContourT", "IntegrandGDirect", "ComputeChargeQDirect",
           "ComputeChargeQDirectTime", "BinnerT1", "BinnerT11", "ComputeGfKernel", "IntegrandGKernel", "binner_data",
           "ComputeGfKernelSingleOmega", "IntegrandGKernelSingleOmega",
           "ComputeCurrentJDirect", "model_param_t", "MODEL_PARAM_DEFAULTS"]
