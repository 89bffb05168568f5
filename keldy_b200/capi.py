"""ctypes binding of the keldy_b200 C ABI (include/keldy_b200.h).

This is the thinnest way into the library: plain pointers and sizes, numpy arrays on
the Python side. Every call runs on the GPU; there is no CPU path, and loading the
library or creating a context fails loudly when the shared library or a CUDA device is
missing.
"""
from __future__ import annotations

import ctypes as C
import os
import weakref

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libkeldy_b200.so")

KB_OK = 0
KB_E_INVALID, KB_E_CUDA, KB_E_NOMEM, KB_E_RANGE, KB_E_EXHAUSTED, KB_E_NODEVICE = -1, -2, -3, -4, -5, -6

WARPER_IDENTITY, WARPER_PLASMA_UV, WARPER_EXPONENTIAL, WARPER_INVERSE = 0, 1, 2, 3
WARPER_INVERSE_SQUARE, WARPER_INVERSE_POWER, WARPER_UNIFORM = 4, 5, 6
WARPER_TABLE = 7
MAX_CHAIN = 8
REVERSE, FORWARD = 0, 1
ALGO_AUTO, ALGO_TREE, ALGO_DIRECT = 0, 1, 2

# every symbol include/keldy_b200.h declares
EXPORTS = [
    "kb_last_error", "kb_version", "kb_context_create", "kb_context_destroy", "kb_context_synchronize",
    "kb_context_stream", "kb_context_set_timing", "kb_context_last_timing", "kb_sobol_create", "kb_sobol_destroy", "kb_sobol_matrices", "kb_sobol_points",
    "kb_sobol_points_dev", "kb_models_set_flatband", "kb_model_get_table",
    "kb_warp", "kb_model_create", "kb_model_destroy", "kb_model_set_table", "kb_model_set_table_dev",
    "kb_g0_eval", "kb_integrand_eval", "kb_integrand_eval_no_det", "kb_evaluate_warped", "kb_integrate",
    "kb_fp64_peak", "kb_integrate_noalloc", "kb_plan_create", "kb_plan_destroy", "kb_plan_launch",
    "kb_plan_result", "kb_plan_set_k_first", "kb_context_set_launch", "kb_context_get_launch",
    "kb_flow_create", "kb_flow_destroy", "kb_flow_dim", "kb_flow_get_params", "kb_flow_set_params", "kb_flow_map",
    "kb_flow_sample", "kb_flow_gradient", "kb_flow_train", "kb_flow_fit", "kb_integrate_binned",
    "kb_integrate_kernel", "kb_integrand_kernel_eval", "kb_warper_table_create", "kb_warper_table_destroy",
    "kb_warper_table_from_projection", "kb_warper_table_analytic", "kb_warper_table_hybrid", "kb_warper_table_info",
    "kb_warper_table_points", "kb_model_set_fourier", "kb_model_set_interpolation", "kb_model_set_fft",
    "kb_model_set_rational",
    "kb_warper_table_from_samples", "kb_warper_projection_create", "kb_warper_projection_axis",
    "kb_warper_projection_from_integrand", "kb_device_allocations", "kb_integrate_kernel_single_omega",
    "kb_flow_create_kind", "kb_flow_num_params",
]
FLOW_LAYERS, FLOW_WIDTH, FLOW_MAX_DIM = 6, 128, 8
FLOW_PARAMS = FLOW_LAYERS * 3 * FLOW_WIDTH * FLOW_WIDTH
NOALLOC_MAX_ITEMS, NOALLOC_MAX_CHUNKS = 64, 65536


class KbError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


class Warper(C.Structure):
    _fields_ = [("kind", C.c_int), ("power", C.c_int), ("u_max", C.c_double), ("w", C.c_double),
                ("table", C.c_void_p)]


class GfIndex(C.Structure):
    _fields_ = [("time", C.c_double), ("spin", C.c_int), ("k_idx", C.c_int), ("timesplit", C.c_int),
                ("orbital", C.c_int)]


class Integrand(C.Structure):
    _fields_ = [("A", GfIndex), ("B", GfIndex), ("cutoff", C.c_double)]


class Accum(C.Structure):
    _fields_ = [("sum_re", C.c_double), ("sum_im", C.c_double), ("n_points", C.c_uint64),
                ("n_in_domain", C.c_uint64), ("n_fallback", C.c_uint64)]


class Work(C.Structure):
    _fields_ = [("m", C.c_void_p), ("rng", C.c_void_p), ("chain", C.POINTER(Warper)), ("chain_len", C.c_int),
                ("f", Integrand), ("order", C.c_int), ("k_first", C.c_uint32), ("n_points", C.c_int64),
                ("flow", C.c_void_p)]


class TimeBins(C.Structure):
    _fields_ = [("nbins", C.c_int), ("xmin", C.c_double), ("xmax", C.c_double)]


class FlowTrainCfg(C.Structure):
    _fields_ = [("epochs", C.c_int), ("batch", C.c_int), ("lr", C.c_float), ("lr_final", C.c_float),
                ("beta1", C.c_float), ("beta2", C.c_float), ("eps", C.c_float), ("seed", C.c_uint64)]


_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)
_VP = C.c_void_p
_lib = None


def load():
    """The library handle; raises if libkeldy_b200.so has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m keldy_b200.build` "
                          "(keldy_b200 has no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    L.kb_last_error.restype = C.c_char_p
    L.kb_context_create.argtypes = [C.c_int, C.POINTER(_VP)]
    L.kb_context_destroy.argtypes = [_VP]
    L.kb_context_synchronize.argtypes = [_VP]
    L.kb_context_stream.argtypes = [_VP]
    L.kb_context_stream.restype = _VP
    L.kb_context_set_timing.argtypes = [_VP, C.c_int]
    L.kb_context_last_timing.argtypes = [_VP, _D, _D, _D, _I]
    L.kb_sobol_create.argtypes = [_VP, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(_VP)]
    L.kb_sobol_destroy.argtypes = [_VP]
    L.kb_sobol_matrices.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_uint32),
                                    C.POINTER(C.c_uint32)]
    L.kb_sobol_points.argtypes = [_VP, _VP, C.c_uint32, C.c_int64, _D]
    L.kb_sobol_points_dev.argtypes = [_VP, _VP, C.c_uint32, C.c_int64, _VP]
    L.kb_warp.argtypes = [_VP, C.POINTER(Warper), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int64, _D, _D,
                          _D]
    L.kb_model_create.argtypes = [_VP, C.c_int, C.c_double, C.c_double, C.POINTER(_VP)]
    L.kb_model_destroy.argtypes = [_VP]
    L.kb_model_set_table.argtypes = [_VP, C.c_int, C.c_int, C.c_int, _D, _D]
    L.kb_model_set_table_dev.argtypes = [_VP, C.c_int, C.c_int, C.c_int, _VP, _VP]
    L.kb_models_set_flatband.argtypes = [C.c_int, C.POINTER(_VP), _D]
    L.kb_model_get_table.argtypes = [_VP, C.c_int, C.c_int, C.c_int, _D, _D]
    L.kb_g0_eval.argtypes = [_VP, _VP, C.POINTER(GfIndex), C.POINTER(GfIndex), _I, C.c_int64, _D]
    L.kb_integrand_eval.argtypes = [_VP, _VP, C.POINTER(Integrand), C.c_int, C.c_int64, _D, C.c_int, C.c_int, _D,
                                    _I, _D]
    L.kb_integrand_eval_no_det.argtypes = [_VP, _VP, C.POINTER(Integrand), C.c_int, C.c_int64, _D, C.c_int, _D,
                                           _I]
    L.kb_evaluate_warped.argtypes = [_VP, _VP, C.POINTER(Integrand), C.POINTER(Warper), C.c_int, C.c_int, C.c_int,
                                     C.c_int64, _D, C.c_int, C.c_int, _D, _D, _I]
    L.kb_integrate.argtypes = [_VP, C.POINTER(Work), C.c_int, C.c_int, C.POINTER(Accum)]
    L.kb_warper_table_create.argtypes = [_VP, C.c_int, _I, _D, _D, C.POINTER(_VP)]
    L.kb_warper_table_destroy.argtypes = [_VP]
    L.kb_warper_table_analytic.argtypes = [_VP, C.c_int, C.POINTER(Warper), C.POINTER(_VP)]
    L.kb_warper_table_hybrid.argtypes = [_VP, C.c_int, C.POINTER(Warper), _I, C.POINTER(_VP)]
    L.kb_model_set_fourier.argtypes = [_VP, C.c_int, C.c_int, C.c_int, _D, _D, _D, C.c_int]
    L.kb_model_set_fft.argtypes = [_VP, C.c_int, C.c_int, _D, _D, C.c_int]
    L.kb_model_set_rational.argtypes = [_VP, C.c_int, C.c_int, C.c_int, _D, _I, _D, _D, C.c_double, C.c_int]
    L.kb_model_set_interpolation.argtypes = [_VP, C.c_int]
    L.kb_warper_table_info.argtypes = [_VP, _I, _I, _I]
    L.kb_warper_table_points.argtypes = [_VP, C.c_int, _D, _D]
    L.kb_warper_table_from_samples.argtypes = [_VP, C.c_int, C.c_int, C.c_int64, _D, _D, C.c_double, C.POINTER(_VP)]
    L.kb_warper_projection_create.argtypes = [_VP, C.c_int, C.c_int, C.c_int64, _D, _D, C.c_double, C.c_int,
                                              C.POINTER(_VP)]
    L.kb_warper_projection_axis.argtypes = [_VP, C.c_int, _D, _D, C.POINTER(C.c_uint64), _D]
    L.kb_warper_projection_from_integrand.argtypes = [_VP, _VP, C.POINTER(Integrand), C.POINTER(Warper), C.c_int,
                                                      C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int,
                                                      C.POINTER(_VP)]
    L.kb_warper_table_from_projection.argtypes = [_VP, _VP, C.POINTER(Integrand), C.POINTER(Warper), C.c_int, C.c_int,
                                                  C.c_int, C.c_int, C.c_double, C.c_int, C.POINTER(_VP)]
    L.kb_integrate_kernel.argtypes = [_VP, C.POINTER(Work), C.c_int, C.POINTER(TimeBins), C.POINTER(Accum), _D,
                                      C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
    L.kb_integrate_kernel_single_omega.argtypes = [_VP, C.POINTER(Work), C.c_int, C.c_double, C.POINTER(Accum)]
    L.kb_integrand_kernel_eval.argtypes = [_VP, _VP, C.POINTER(GfIndex), C.c_int, C.c_int64, _D, C.c_int, _D, _I]
    L.kb_integrate_binned.argtypes = [_VP, C.POINTER(Work), C.c_int, C.c_int, C.POINTER(TimeBins), C.POINTER(Accum),
                                      _D, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
    L.kb_fp64_peak.argtypes = [_VP, C.c_int, _D]
    L.kb_integrate_noalloc.argtypes = [_VP, C.POINTER(Work), C.c_int, C.POINTER(Accum)]
    L.kb_device_allocations.argtypes = []
    L.kb_device_allocations.restype = C.c_uint64
    L.kb_plan_create.argtypes = [_VP, C.POINTER(Work), C.c_int, C.c_int, C.POINTER(_VP)]
    L.kb_plan_destroy.argtypes = [_VP]
    L.kb_plan_launch.argtypes = [_VP, _VP]
    L.kb_plan_result.argtypes = [_VP, _VP, C.POINTER(Accum)]
    L.kb_plan_set_k_first.argtypes = [_VP, _VP, C.c_int, C.c_uint32]
    L.kb_context_set_launch.argtypes = [_VP, C.c_int, C.c_int, C.c_int]
    L.kb_context_get_launch.argtypes = [_VP, C.c_int, _I, _I]
    _F = C.POINTER(C.c_float)
    L.kb_flow_create.argtypes = [_VP, C.c_int, C.c_uint64, C.POINTER(_VP)]
    L.kb_flow_create_kind.argtypes = [_VP, C.c_int, C.c_int, C.c_uint64, C.POINTER(_VP)]
    L.kb_flow_num_params.argtypes = [_VP]
    L.kb_flow_destroy.argtypes = [_VP]
    L.kb_flow_dim.argtypes = [_VP]
    L.kb_flow_get_params.argtypes = [_VP, _F]
    L.kb_flow_set_params.argtypes = [_VP, _F]
    L.kb_flow_map.argtypes = [_VP, C.c_int, C.c_int64, _D, _D, _D]
    L.kb_flow_sample.argtypes = [_VP, _VP, C.c_uint32, C.c_int64, _D, _D]
    L.kb_flow_gradient.argtypes = [_VP, C.c_int64, _D, _D, _F, _D]
    L.kb_flow_train.argtypes = [_VP, C.c_int64, _D, _D, C.POINTER(FlowTrainCfg), _D, _I]
    L.kb_flow_fit.argtypes = [_VP, _VP, C.POINTER(Integrand), C.POINTER(Warper), C.c_int, _VP, C.c_uint32, C.c_int64,
                              C.POINTER(FlowTrainCfg), _D]
    _lib = L
    return L


def check(code):
    if code != KB_OK:
        raise KbError(code, load().kb_last_error().decode())


def sobol_matrices(dim, log_max_points=31, do_shift=False, do_scramble=False, seed_shift=0):
    """Host-only: (Csr[dim, m], shfr[dim]) as keldy::sobol would build them."""
    L = load()
    Csr = np.zeros(dim * log_max_points, dtype=np.uint32)
    shfr = np.zeros(dim, dtype=np.uint32)
    U = C.POINTER(C.c_uint32)
    check(L.kb_sobol_matrices(dim, log_max_points, int(do_shift), int(do_scramble), int(seed_shift),
                              Csr.ctypes.data_as(U), shfr.ctypes.data_as(U)))
    return Csr.reshape(dim, log_max_points), shfr


def _dp(a):
    return None if a is None else a.ctypes.data_as(_D)


def _ip(a):
    return None if a is None else a.ctypes.data_as(_I)


_WARPER_P = C.POINTER(Warper)


def chain_array(chain):
    """chain: list of (kind, u_max, w[, power]) or (WARPER_TABLE, WarperTable) -> (ctypes array,
    length)."""
    arr = (Warper * MAX_CHAIN)()
    for i, c in enumerate(chain):
        if int(c[0]) == WARPER_TABLE:
            arr[i] = Warper(WARPER_TABLE, 0, 0.0, 0.0, c[1].h.value)
        else:
            arr[i] = Warper(int(c[0]), int(c[3]) if len(c) > 3 else 0, float(c[1]), float(c[2]), None)
    return arr, len(chain)


TABLE_NEAREST, TABLE_PROJECTION, TABLE_ANALYTIC, TABLE_HYBRID = 0, 1, 2, 3


def _samples(li, values):
    li = np.ascontiguousarray(np.atleast_2d(li), dtype=np.float64)
    values = np.ascontiguousarray(values, dtype=np.float64)
    if len(values) != len(li):
        raise ValueError("one value per sample point")
    return li, values


class WarperTable:
    """Device-resident product warper (kb_warper_table): one 1D warper for every
    coordinate or one per coordinate; use in a chain as (WARPER_TABLE, self).
    WarperTable(ctx, tables): interp-nearest tables from a list of (u_points, f1_values);
    the classmethods build the other kinds."""

    def __init__(self, ctx, tables=None, _handle=None):
        self.ctx = ctx
        if _handle is not None:
            self.h = _handle
        else:
            npts = np.array([len(u) for u, _ in tables], dtype=np.int32)
            u = np.ascontiguousarray(np.concatenate([np.asarray(u, dtype=np.float64) for u, _ in tables]))
            f1 = np.ascontiguousarray(np.concatenate([np.asarray(f, dtype=np.float64) for _, f in tables]))
            h = _VP()
            check(ctx.L.kb_warper_table_create(ctx.h, len(tables), npts.ctypes.data_as(_I), _dp(u), _dp(f1),
                                               C.byref(h)))
            self.h = h
        ctx._deps.add(self)

    @classmethod
    def from_projection(cls, ctx, model, A, B, chain, order, num_bins, nr_samples, sigma, keep_u_hypercube=True,
                        cutoff=0.0):
        """make_warper_from_proj: one table per axis from the projections of |f J|."""
        arr, L = chain_array(chain)
        f = Integrand(gf_index(A), gf_index(B), float(cutoff))
        h = _VP()
        check(ctx.L.kb_warper_table_from_projection(ctx.h, model.h, C.byref(f), arr, L, int(order), int(num_bins),
                                                    int(nr_samples), float(sigma), int(keep_u_hypercube),
                                                    C.byref(h)))
        return cls(ctx, _handle=h)

    @classmethod
    def analytic(cls, ctx, dims):
        """warper_product_1d_t: dims = [(kind, u_max, w[, power])] per coordinate."""
        arr = (Warper * len(dims))()
        for i, c in enumerate(dims):
            arr[i] = Warper(int(c[0]), int(c[3]) if len(c) > 3 else 0, float(c[1]), float(c[2]), None)
        h = _VP()
        check(ctx.L.kb_warper_table_analytic(ctx.h, len(dims), arr, C.byref(h)))
        return cls(ctx, _handle=h)

    @classmethod
    def hybrid(cls, ctx, shapes, npts):
        """warper_product_1d_simple_interp_hybrid_t per coordinate: shapes = [(kind, u_max,
        w[, power])], the closed form of f1 (up to a factor) and the domain; npts points each."""
        arr = (Warper * len(shapes))()
        for i, c in enumerate(shapes):
            arr[i] = Warper(int(c[0]), int(c[3]) if len(c) > 3 else 0, float(c[1]), float(c[2]), None)
        n = np.ascontiguousarray(np.broadcast_to(np.asarray(npts, dtype=np.int32), (len(shapes),)))
        h = _VP()
        check(ctx.L.kb_warper_table_hybrid(ctx.h, len(shapes), arr, n.ctypes.data_as(_I), C.byref(h)))
        return cls(ctx, _handle=h)

    @classmethod
    def from_samples(cls, ctx, li, values, num_bins, sigma):
        """make_warper_from_proj from samples li [n, order] with values |f J|."""
        li, values = _samples(li, values)
        h = _VP()
        check(ctx.L.kb_warper_table_from_samples(ctx.h, li.shape[1], int(num_bins), len(li), _dp(li), _dp(values),
                                                 float(sigma), C.byref(h)))
        return cls(ctx, _handle=h)

    @classmethod
    def projection(cls, ctx, li, values, num_bins, sigma, optimize_sigma=True):
        """warper_projection_t from samples li [n, order] with values |f J|."""
        li, values = _samples(li, values)
        h = _VP()
        check(ctx.L.kb_warper_projection_create(ctx.h, li.shape[1], int(num_bins), len(li), _dp(li), _dp(values),
                                                float(sigma), int(bool(optimize_sigma)), C.byref(h)))
        return cls(ctx, _handle=h)

    @classmethod
    def projection_from_integrand(cls, ctx, model, A, B, chain, order, num_bins, nr_samples, sigma,
                                  optimize_sigma=True, keep_u_hypercube=True, cutoff=0.0):
        """warper_projection_t for the integrand through `chain`, sampled on the GPU."""
        arr, L = chain_array(chain)
        f = Integrand(gf_index(A), gf_index(B), float(cutoff))
        h = _VP()
        check(ctx.L.kb_warper_projection_from_integrand(ctx.h, model.h, C.byref(f), arr, L, int(order),
                                                        int(num_bins), int(nr_samples), float(sigma),
                                                        int(bool(optimize_sigma)), int(keep_u_hypercube),
                                                        C.byref(h)))
        return cls(ctx, _handle=h)

    def info(self):
        """(type, ndims, points of each coordinate's first table)."""
        t, n = C.c_int(), C.c_int()
        check(self.ctx.L.kb_warper_table_info(self.h, C.byref(t), C.byref(n), None))
        pts = np.zeros(n.value, dtype=np.int32)
        check(self.ctx.L.kb_warper_table_info(self.h, None, None, pts.ctypes.data_as(_I)))
        return t.value, n.value, pts

    def projection_axis(self, axis):
        """Projection warper: (sigma, xi means, xi counts, fn) of one axis."""
        nb = int(self.info()[2][axis])
        s = C.c_double()
        xi, fn = np.zeros(nb), np.zeros(nb)
        cnt = np.zeros(nb, dtype=np.uint64)
        check(self.ctx.L.kb_warper_projection_axis(self.h, int(axis), C.byref(s), _dp(xi),
                                                   cnt.ctypes.data_as(C.POINTER(C.c_uint64)), _dp(fn)))
        return s.value, xi, cnt, fn

    def entry(self):
        return (WARPER_TABLE, self)

    def close(self):
        if self.h:
            self.ctx.L.kb_warper_table_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def gf_index(x):
    if isinstance(x, GfIndex):
        return x
    t = tuple(x) + (0,) * (5 - len(x))
    return GfIndex(float(t[0]), int(t[1]), int(t[2]), int(t[3]), int(t[4]))


class Context:
    """One CUDA device: a stream plus the library's bookkeeping."""

    def __init__(self, device=0):
        L = load()
        h = _VP()
        check(L.kb_context_create(device, C.byref(h)))
        self.h = h
        self.L = L
        self._deps = weakref.WeakSet()  # models and generators, destroyed before the context

    def close(self):
        if self.h:
            for d in list(self._deps):
                d.close()
            self.L.kb_context_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self):
        return self.L.kb_context_stream(self.h)

    def synchronize(self):
        check(self.L.kb_context_synchronize(self.h))

    def set_timing(self, enable=True):
        check(self.L.kb_context_set_timing(self.h, int(enable)))

    def set_launch(self, order=-1, chunk_points=128, ctas_per_sm=0):
        """Tree-kernel launch shape: points per scheduling chunk of `order` (-1: all) and
        resident CTAs per SM (0 keeps the current value)."""
        check(self.L.kb_context_set_launch(self.h, order, chunk_points, ctas_per_sm))

    def get_launch(self, order):
        a, b = C.c_int(), C.c_int()
        check(self.L.kb_context_get_launch(self.h, order, C.byref(a), C.byref(b)))
        return a.value, b.value

    def last_timing(self):
        """(integrand_ms, fallback_ms, reduce_ms, launches) of the last kb_integrate."""
        a, b, c, n = C.c_double(), C.c_double(), C.c_double(), C.c_int()
        check(self.L.kb_context_last_timing(self.h, C.byref(a), C.byref(b), C.byref(c), C.byref(n)))
        return a.value, b.value, c.value, n.value

    def fp64_peak(self, iters=1 << 16):
        v = C.c_double()
        check(self.L.kb_fp64_peak(self.h, iters, C.byref(v)))
        return v.value

    # --- Sobol -------------------------------------------------------------
    def sobol(self, dim, log_max_points=31, do_shift=False, do_scramble=False, seed_shift=0):
        return Sobol(self, dim, log_max_points, do_shift, do_scramble, seed_shift)

    # --- warpers -----------------------------------------------------------
    def warp(self, chain, x, direction=REVERSE, start=None, end=None, want_jac=True):
        x = np.ascontiguousarray(np.atleast_2d(x), dtype=np.float64)
        count, n = x.shape
        arr, L = chain_array(chain)
        if direction == REVERSE:
            start = L if start is None else start
            end = 0 if end is None else end
        else:
            start = 0 if start is None else start
            end = L if end is None else end
        out = np.empty_like(x)
        jac = np.empty(count) if want_jac else None
        check(self.L.kb_warp(self.h, arr, L, direction, start, end, n, count, _dp(x), _dp(out), _dp(jac)))
        return out, jac

    # --- model ---------------------------------------------------------------
    def model(self, time_max, lesser, greater, alpha=0.0, lesser_down=None, greater_down=None, blocks=None):
        return Model(self, time_max, lesser, greater, alpha, lesser_down, greater_down, blocks)

    # --- learned flow ------------------------------------------------------
    def flow(self, dim, seed=0, kind=0):
        """A learned warper (kind FLOW_COUPLING or FLOW_SPLINE)."""
        return Flow(self, dim, seed, kind)


class Sobol:
    def __init__(self, ctx, dim, log_max_points=31, do_shift=False, do_scramble=False, seed_shift=0):
        self.ctx = ctx
        self.dim = dim
        self.m = log_max_points
        h = _VP()
        check(ctx.L.kb_sobol_create(ctx.h, dim, log_max_points, int(do_shift), int(do_scramble), int(seed_shift),
                                    C.byref(h)))
        self.h = h
        ctx._deps.add(self)

    def close(self):
        if self.h:
            self.ctx.L.kb_sobol_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def points(self, k_first, count):
        out = np.empty((count, self.dim))
        check(self.ctx.L.kb_sobol_points(self.ctx.h, self.h, k_first, count, _dp(out)))
        return out


class Model:
    """g0 tables (complex arrays on [-time_max, time_max]) uploaded to the device."""

    def __init__(self, ctx, time_max, lesser, greater, alpha=0.0, lesser_down=None, greater_down=None, blocks=None,
                 npts=None):
        """lesser/greater None: no table uploaded (npts gives the mesh; see flatband_models)."""
        self.ctx = ctx
        self.npts = int(npts) if lesser is None else len(lesser)
        self.time_max = time_max
        h = _VP()
        check(ctx.L.kb_model_create(ctx.h, self.npts, float(time_max), float(alpha), C.byref(h)))
        self.h = h
        ctx._deps.add(self)
        if lesser is None:
            return
        self.set_table(0, 0, 0, lesser, greater)
        if lesser_down is not None:
            self.set_table(1, 0, 0, lesser_down, greater_down)
        for (spin, o1, o2), (le, gr) in (blocks or {}).items():
            self.set_table(spin, o1, o2, le, gr)

    def set_table(self, spin, o1, o2, lesser, greater):
        le = np.ascontiguousarray(lesser, dtype=np.complex128).view(np.float64)
        gr = np.ascontiguousarray(greater, dtype=np.complex128).view(np.float64)
        assert le.size == 2 * self.npts and gr.size == 2 * self.npts
        check(self.ctx.L.kb_model_set_table(self.h, spin, o1, o2, _dp(le), _dp(gr)))

    def set_interpolation(self, order):
        """1: linear (keldy's); 3: cubic Lagrange through 4 mesh points (an extension)."""
        check(self.ctx.L.kb_model_set_interpolation(self.h, int(order)))

    def set_fourier(self, o1, o2, w, cl, cg, flags=0):
        """Block (o1, o2) as the Fourier sums g(t) = sum_k c_k e^{-i w_k t} on the GPU
        (kb_model_set_fourier; flags FT_SYMMETRIC, FT_MIRROR)."""
        w = np.ascontiguousarray(w, dtype=np.float64)
        cl = np.ascontiguousarray(cl, dtype=np.complex128).view(np.float64)
        cg = np.ascontiguousarray(cg, dtype=np.complex128).view(np.float64)
        assert cl.size == 2 * w.size and cg.size == 2 * w.size
        check(self.ctx.L.kb_model_set_fourier(self.h, int(o1), int(o2), w.size, _dp(w), _dp(cl), _dp(cg), int(flags)))

    def set_fft(self, o1, o2, gl_w, gg_w, flags=0):
        """Block (o1, o2) as keldy's "fft" tables: the discrete transform on the GPU of the
        values on the frequency mesh adjoint to the time mesh (kb_model_set_fft; flags
        FT_MIRROR)."""
        gl = np.ascontiguousarray(gl_w, dtype=np.complex128).view(np.float64)
        gg = np.ascontiguousarray(gg_w, dtype=np.complex128).view(np.float64)
        assert gl.size == 2 * self.npts and gg.size == 2 * self.npts
        check(self.ctx.L.kb_model_set_fft(self.h, int(o1), int(o2), _dp(gl), _dp(gg), int(flags)))

    def set_rational(self, o1, o2, terms, beta, flags=0):
        """Block (o1, o2) of a bath with a rational hybridisation in closed form
        (kb_model_set_rational): terms = [(mu, poles, residues), ...] as from
        g0_tables.rational_terms; flags FT_SYMMETRIC, FT_MIRROR."""
        mu = np.array([t[0] for t in terms], dtype=np.float64)
        npl = np.array([len(t[1]) for t in terms], dtype=np.int32)
        z = np.ascontiguousarray(np.concatenate([np.asarray(t[1], np.complex128) for t in terms])).view(np.float64)
        r = np.ascontiguousarray(np.concatenate([np.asarray(t[2], np.complex128) for t in terms])).view(np.float64)
        check(self.ctx.L.kb_model_set_rational(self.h, int(o1), int(o2), len(terms), _dp(mu), _ip(npl), _dp(z),
                                               _dp(r), float(beta), int(flags)))

    def table(self, spin=0, o1=0, o2=0):
        """(lesser, greater) complex arrays of one block, read back from the device."""
        le = np.empty(self.npts, dtype=np.complex128)
        gr = np.empty(self.npts, dtype=np.complex128)
        check(self.ctx.L.kb_model_get_table(self.h, spin, o1, o2, _dp(le.view(np.float64)), _dp(gr.view(np.float64))))
        return le, gr

    def close(self):
        if self.h:
            self.ctx.L.kb_model_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def g0(self, a, b, internal=None):
        a = list(a)
        b = list(b)
        count = len(a)
        A = (GfIndex * count)(*[gf_index(x) for x in a])
        B = (GfIndex * count)(*[gf_index(x) for x in b])
        inte = None if internal is None else np.ascontiguousarray(internal, dtype=np.int32)
        out = np.empty(count, dtype=np.complex128)
        check(self.ctx.L.kb_g0_eval(self.ctx.h, self.h, A, B, _ip(inte), count, _dp(out.view(np.float64))))
        return out

    def integrand(self, A, B, times, cutoff=0.0, keep_u_hypercube=True, algo=ALGO_AUTO, want_scale=False,
                  order=None):
        times = np.ascontiguousarray(times, dtype=np.float64)
        if times.ndim == 1:
            times = times[None, :] if order is None or order > 0 else times.reshape(-1, 0)
        count, n = times.shape
        f = Integrand(gf_index(A), gf_index(B), float(cutoff))
        out = np.empty(count, dtype=np.complex128)
        dom = np.empty(count, dtype=np.int32)
        sc = np.empty(count) if want_scale else None
        check(self.ctx.L.kb_integrand_eval(self.ctx.h, self.h, C.byref(f), n, count, _dp(times),
                                           int(keep_u_hypercube), algo, _dp(out.view(np.float64)), _ip(dom),
                                           _dp(sc)))
        return (out, dom, sc) if want_scale else (out, dom)

    def integrand_kernel(self, X, times, keep_u_hypercube=True):
        """integrand_g_kernel for fixed point X: (sums [count][order][2] complex per (vertex,
        Keldysh index), in_domain)."""
        times = np.ascontiguousarray(np.atleast_2d(times), dtype=np.float64)
        count, n = times.shape
        out = np.empty((count, n, 2), dtype=np.complex128)
        dom = np.empty(count, dtype=np.int32)
        check(self.ctx.L.kb_integrand_kernel_eval(self.ctx.h, self.h, C.byref(gf_index(X)), n, count, _dp(times),
                                                  int(keep_u_hypercube), _dp(out.view(np.float64)), _ip(dom)))
        return out, dom

    def integrand_no_det(self, A, B, times, cutoff=0.0, keep_u_hypercube=True):
        times = np.ascontiguousarray(np.atleast_2d(times), dtype=np.float64)
        count, n = times.shape
        f = Integrand(gf_index(A), gf_index(B), float(cutoff))
        out = np.empty(count, dtype=np.complex128)
        dom = np.empty(count, dtype=np.int32)
        check(self.ctx.L.kb_integrand_eval_no_det(self.ctx.h, self.h, C.byref(f), n, count, _dp(times),
                                                  int(keep_u_hypercube), _dp(out.view(np.float64)), _ip(dom)))
        return out, dom

    def evaluate_warped(self, A, B, chain, li, cutoff=0.0, start=None, keep_u_hypercube=True, algo=ALGO_AUTO):
        li = np.ascontiguousarray(np.atleast_2d(li), dtype=np.float64)
        count, n = li.shape
        arr, L = chain_array(chain)
        f = Integrand(gf_index(A), gf_index(B), float(cutoff))
        out = np.empty(count, dtype=np.complex128)
        jac = np.empty(count)
        dom = np.empty(count, dtype=np.int32)
        check(self.ctx.L.kb_evaluate_warped(self.ctx.h, self.h, C.byref(f), arr, L, L if start is None else start, n,
                                            count, _dp(li), int(keep_u_hypercube), algo, _dp(out.view(np.float64)),
                                            _dp(jac), _ip(dom)))
        return out, jac, dom


def flatband_models(ctx, params, time_max, npts, alpha=0.0):
    """Models of the dot with flat-band leads, their g0 tables built on the GPU in one
    launch (kb_models_set_flatband). params: rows (Gamma, eps_d, V, beta); npts odd."""
    params = np.ascontiguousarray(np.atleast_2d(params), dtype=np.float64)
    models = [Model(ctx, time_max, None, None, alpha, npts=npts) for _ in range(len(params))]
    hs = (_VP * max(1, len(models)))(*[m.h for m in models])
    check(ctx.L.kb_models_set_flatband(len(models), hs, _dp(params)))
    return models


FT_SYMMETRIC, FT_MIRROR = 1, 2


def semicircle_model(ctx, gamma, eps_d, bias_V, beta, half_bandwidth, time_max, npts, alpha=0.0, dot_lead=False,
                     nodes=None):
    """A model of the dot with semicircular leads, its tables built on the GPU: the band
    quadrature of g0_tables.semicircle_nodes summed by kb_model_set_fourier (the dot block
    on t >= 0 and mirrored; with dot_lead the (1,0) block and its mirror (0,1))."""
    from .g0_tables import semicircle_nodes
    w, f_less, f_great, f_l10, f_g10 = semicircle_nodes(gamma, eps_d, bias_V, beta, half_bandwidth, time_max, nodes)
    m = Model(ctx, time_max, None, None, alpha, npts=npts)
    m.set_fourier(0, 0, w, f_less, f_great, FT_SYMMETRIC)
    if dot_lead:
        m.set_fourier(1, 0, w, f_l10, f_g10, FT_MIRROR)
    return m


def _works(items):
    """The kb_work array of `items` and the ctypes objects it points into (keep them alive
    during the call). Items that share a chain list or external-point objects share one
    converted copy: a call over many replicas of one integrand converts them once."""
    n = len(items)
    works = (Work * max(1, n))()
    keep, chains, fs = [], {}, {}
    for i, it in enumerate(items):
        ch = it["chain"]
        c = chains.get(id(ch))
        if c is None:
            arr, L = chain_array(ch)
            keep.append(arr)
            c = chains[id(ch)] = (C.cast(arr, _WARPER_P), L)
        A = it["A"]
        B = it.get("B", A)
        cut = it.get("cutoff", 0.0)
        f = fs.get((id(A), id(B), cut))
        if f is None:
            f = fs[(id(A), id(B), cut)] = Integrand(gf_index(A), gf_index(B), float(cut))
        flow = it.get("flow")
        works[i] = Work(it["model"].h.value, it["rng"].h.value, c[0], c[1], f, int(it["order"]),
                        int(it.get("k_first", 1)), int(it["n_points"]), flow.h.value if flow is not None else None)
    keep.append((chains, fs, items))
    return works, keep


class Plan:
    """A batched integration set up once and launched many times (captured into a CUDA
    graph on its first launch)."""

    def __init__(self, ctx, items, algo=ALGO_AUTO):
        self.ctx = ctx
        self.items = list(items)
        works, self._keep = _works(self.items)
        h = _VP()
        check(ctx.L.kb_plan_create(ctx.h, works, len(self.items), algo, C.byref(h)))
        self.h = h
        ctx._deps.add(self)

    def launch(self):
        check(self.ctx.L.kb_plan_launch(self.ctx.h, self.h))

    def result(self):
        acc = (Accum * max(1, len(self.items)))()
        check(self.ctx.L.kb_plan_result(self.ctx.h, self.h, acc))
        return [(complex(a.sum_re, a.sum_im), a.n_points, a.n_in_domain, a.n_fallback) for a in acc[:len(self.items)]]

    def run(self):
        self.launch()
        return self.result()

    def set_k_first(self, item, k_first):
        check(self.ctx.L.kb_plan_set_k_first(self.ctx.h, self.h, item, k_first))

    def close(self):
        if self.h:
            self.ctx.L.kb_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def integrate_binned(ctx, items, nbins, xmin, xmax, algo=ALGO_AUTO):
    """kb_integrate_binned: per item (sum, n_points, n_in_domain, n_fallback, bins complex[nbins],
    counts[nbins], dropped) - keldy's integrand_g_direct_time binned by the earliest vertex
    time into binner_t(xmin, xmax, nbins)."""
    works, keep = _works(items)
    n = len(items)
    acc = (Accum * max(1, n))()
    sums = np.zeros((max(1, n), nbins), dtype=np.complex128)
    counts = np.zeros((max(1, n), nbins), dtype=np.uint64)
    dropped = np.zeros(max(1, n), dtype=np.uint64)
    U = C.POINTER(C.c_uint64)
    check(ctx.L.kb_integrate_binned(ctx.h, works, n, algo, C.byref(TimeBins(int(nbins), float(xmin), float(xmax))),
                                    acc, _dp(sums.view(np.float64)), counts.ctypes.data_as(U),
                                    dropped.ctypes.data_as(U)))
    return [(complex(a.sum_re, a.sum_im), a.n_points, a.n_in_domain, a.n_fallback, sums[i], counts[i].astype(np.int64),
             int(dropped[i])) for i, a in enumerate(acc[:n])]


def integrate_kernel(ctx, items, nbins, xmin, xmax):
    """kb_integrate_kernel (keldy's kernel method, fixed point X = item["A"]): per item (sum,
    n_points, n_in_domain, bins complex[nbins][2], counts[nbins][2], dropped)."""
    items = [dict(it, B=it.get("B", it["A"])) for it in items]
    works, keep = _works(items)
    n = len(items)
    acc = (Accum * max(1, n))()
    sums = np.zeros((max(1, n), nbins, 2), dtype=np.complex128)
    counts = np.zeros((max(1, n), nbins, 2), dtype=np.uint64)
    dropped = np.zeros(max(1, n), dtype=np.uint64)
    U = C.POINTER(C.c_uint64)
    check(ctx.L.kb_integrate_kernel(ctx.h, works, n, C.byref(TimeBins(int(nbins), float(xmin), float(xmax))), acc,
                                    _dp(sums.view(np.float64)), counts.ctypes.data_as(U), dropped.ctypes.data_as(U)))
    return [(complex(a.sum_re, a.sum_im), a.n_points, a.n_in_domain, sums[i], counts[i].astype(np.int64),
             int(dropped[i])) for i, a in enumerate(acc[:n])]


def integrate_kernel_single_omega(ctx, items, omega):
    """kb_integrate_kernel_single_omega (keldy's kernel method at one frequency, fixed point
    X = item["A"]): per item (sum, n_points, n_in_domain)."""
    items = [dict(it, B=it.get("B", it["A"])) for it in items]
    works, keep = _works(items)
    n = len(items)
    acc = (Accum * max(1, n))()
    check(ctx.L.kb_integrate_kernel_single_omega(ctx.h, works, n, float(omega), acc))
    return [(complex(a.sum_re, a.sum_im), a.n_points, a.n_in_domain) for a in acc[:n]]


def device_allocations():
    """kb_device_allocations: device allocations the library has made in this process."""
    return int(load().kb_device_allocations())


def integrate_noalloc(ctx, items):
    """kb_integrate_noalloc: as integrate(algo=ALGO_AUTO), for callers that cannot allocate
    device memory; its scratch is a fixed device array inside the library (at most 64
    items and 65,536 scheduling chunks per call: 8,388,608 points with 128-point chunks)."""
    works, keep = _works(items)
    acc = (Accum * max(1, len(items)))()
    check(ctx.L.kb_integrate_noalloc(ctx.h, works, len(items), acc))
    return [(complex(a.sum_re, a.sum_im), a.n_points, a.n_in_domain, a.n_fallback) for a in acc[:len(items)]]


def integrate(ctx, items, algo=ALGO_AUTO):
    """items: list of dicts {model, rng, chain, A, B, cutoff, order, k_first, n_points}.
    Returns a list of (sum f*J, n_points, n_in_domain, n_fallback)."""
    n = len(items)
    works, keep = _works(items)
    acc = (Accum * max(1, n))()
    check(ctx.L.kb_integrate(ctx.h, works, n, algo, acc))
    return [(complex(a.sum_re, a.sum_im), a.n_points, a.n_in_domain, a.n_fallback) for a in acc[:n]]


def train_cfg(epochs=20, batch=16384, lr=2e-3, lr_final=1e-4, beta1=0.9, beta2=0.999, eps=1e-8, seed=0):
    return FlowTrainCfg(int(epochs), int(batch), float(lr), float(lr_final), float(beta1), float(beta2), float(eps),
                        int(seed))


FLOW_COUPLING, FLOW_SPLINE, FLOW_AR_SPLINE = 0, 1, 2


class Flow:
    """Learned warper of dimension `dim` on the device, a first stage before the warper
    chain trained on |integrand| samples of the plain method (kb_flow_* in
    include/keldy_b200.h): kind FLOW_COUPLING (coupling layers with tensor-core MLP
    conditioners, dim 2..8), FLOW_SPLINE (separable rational-quadratic splines, dim 1..8)
    or FLOW_AR_SPLINE (autoregressive splines whose parameters are linear in Legendre
    features of the earlier dimensions, dim 1..8)."""

    def __init__(self, ctx, dim, seed=0, kind=FLOW_COUPLING):
        self.ctx = ctx
        self.dim = dim
        self.kind = kind
        h = _VP()
        check(ctx.L.kb_flow_create_kind(ctx.h, dim, int(kind), int(seed), C.byref(h)))
        self.h = h
        self.n_params = int(ctx.L.kb_flow_num_params(h))
        ctx._deps.add(self)

    def _pshape(self):
        if self.kind == FLOW_COUPLING:
            return (FLOW_LAYERS, 3, FLOW_WIDTH, FLOW_WIDTH)
        return (self.dim, 49) if self.kind == FLOW_SPLINE else (self.n_params,)

    def close(self):
        if self.h:
            self.ctx.L.kb_flow_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self):
        """float32 [layer][matrix W1, W2, W3][out][in] (coupling), [dim][49] (spline) or the
        flat [A_0, A_1, ...] (autoregressive spline)."""
        p = np.empty(self._pshape(), dtype=np.float32)
        check(self.ctx.L.kb_flow_get_params(self.h, p.ctypes.data_as(C.POINTER(C.c_float))))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == self.n_params
        check(self.ctx.L.kb_flow_set_params(self.h, p.ctypes.data_as(C.POINTER(C.c_float))))

    def map(self, x, direction):
        x = np.ascontiguousarray(np.atleast_2d(x), dtype=np.float64)
        count = x.shape[0]
        assert x.shape[1] == self.dim
        out = np.empty_like(x)
        out2 = np.empty(count)
        check(self.ctx.L.kb_flow_map(self.h, int(direction), count, _dp(x), _dp(out), _dp(out2)))
        return out, out2

    def density(self, x):
        """(z, log q(x)): normalising direction."""
        return self.map(x, 0)

    def sample(self, z):
        """(x, dx/dz): sampling direction."""
        return self.map(z, 1)

    def sample_sobol(self, rng, k_first, count):
        x = np.empty((count, self.dim))
        jac = np.empty(count)
        check(self.ctx.L.kb_flow_sample(self.h, rng.h, k_first, count, _dp(x), _dp(jac)))
        return x, jac

    def gradient(self, x, w):
        """(loss, grad [layer][matrix][out][in]) of sum w (-log q(x)) / len(x)."""
        x = np.ascontiguousarray(np.atleast_2d(x), dtype=np.float64)
        w = np.ascontiguousarray(w, dtype=np.float64)
        g = np.empty(self._pshape(), dtype=np.float32)
        loss = C.c_double()
        check(self.ctx.L.kb_flow_gradient(self.h, x.shape[0], _dp(x), _dp(w), g.ctypes.data_as(C.POINTER(C.c_float)),
                                          C.byref(loss)))
        return loss.value, g

    def train(self, x, w, **cfg):
        x = np.ascontiguousarray(np.atleast_2d(x), dtype=np.float64)
        w = np.ascontiguousarray(w, dtype=np.float64)
        c = train_cfg(**cfg)
        b = min(c.batch, x.shape[0])
        steps = max(1, x.shape[0] // b) * c.epochs
        hist = np.empty(steps)
        ns = C.c_int()
        check(self.ctx.L.kb_flow_train(self.h, x.shape[0], _dp(x), _dp(w), C.byref(c), _dp(hist), C.byref(ns)))
        return hist[:ns.value]

    def fit(self, model, A, B, chain, rng, n_samples, k_first=1, cutoff=0.0, **cfg):
        """Samples the plain method (Sobol points k_first.. of rng through chain, weights
        |f J|) and trains on them; returns the mean loss of the last epoch."""
        arr, L = chain_array(chain)
        f = Integrand(gf_index(A), gf_index(B), float(cutoff))
        c = train_cfg(**cfg)
        loss = C.c_double()
        check(self.ctx.L.kb_flow_fit(self.h, model.h, C.byref(f), arr, L, rng.h, k_first, n_samples, C.byref(c),
                                     C.byref(loss)))
        return loss.value
