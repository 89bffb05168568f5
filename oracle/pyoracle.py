"""ctypes access to the CPU oracle (test infrastructure only).

Two libraries, both built by ``oracle/Makefile``:

* ``liboracle.so``: the plain-C restatement of keldy's hot path (``keldy_oracle.c``).
* ``_ref/libkeldy_ref.so``: keldy's own ``wick_direct.cpp``, ``common.cpp``,
  ``digitalseq_b2g.hpp`` and warper headers compiled against ``oracle/ref_stubs``
  (present only where keldy's sources were available at build time).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg import
this module; the keldy_b200 package never does.
"""
from __future__ import annotations

import ctypes as C
import os
import platform

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

# warper kinds shared by both libraries
W_IDENTITY, W_PLASMA_UV, W_EXPONENTIAL, W_INVERSE, W_INVERSE_SQUARE, W_INVERSE_POWER, W_UNIFORM = range(7)


class Warper(C.Structure):
    _fields_ = [("kind", C.c_int), ("power", C.c_int), ("u_max", C.c_double), ("w", C.c_double)]


class GfIndex(C.Structure):
    _fields_ = [("time", C.c_double), ("spin", C.c_int), ("k_idx", C.c_int), ("timesplit", C.c_int),
                ("orbital", C.c_int)]


class Model(C.Structure):
    _fields_ = [("npts", C.c_int), ("time_max", C.c_double), ("alpha", C.c_double),
                ("tab", C.c_void_p * 16), ("interp", C.c_int)]


_D = C.POINTER(C.c_double)
_U32 = C.POINTER(C.c_uint32)
_I = C.POINTER(C.c_int)


def _dp(a):
    return a.ctypes.data_as(_D)


def chain_array(chain):
    """chain: list of (kind, u_max, w[, power]) tuples -> ctypes Warper array."""
    arr = (Warper * max(1, len(chain)))()
    for i, c in enumerate(chain):
        kind, u_max, w = c[0], float(c[1]), float(c[2])
        power = int(c[3]) if len(c) > 3 else 0
        arr[i] = Warper(kind, power, u_max, w)
    return arr


def build():
    """Build liboracle.so (and oracle/_ref when keldy's sources are present)."""
    import subprocess
    subprocess.run(["make", "-s", "-C", HERE], check=True)


class Oracle:
    """The C restatement."""

    def __init__(self):
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = self.lib = C.CDLL(path)
        L.or_sobol_setup.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _U32, _U32]
        L.or_sobol_points.argtypes = [C.c_int, C.c_int, _U32, _U32, C.c_uint32, C.c_int64, _D]
        L.or_sobol_matrices.argtypes = [C.c_int, C.c_int, _U32]
        L.or_map_reverse.argtypes = [C.POINTER(Warper), C.c_int, C.c_int, C.c_int, C.c_int, _D, _D, _D]
        L.or_map_forward.argtypes = L.or_map_reverse.argtypes
        L.or_g0.argtypes = [C.POINTER(Model), C.POINTER(GfIndex), C.POINTER(GfIndex), C.c_int, _D]
        L.or_integrand.argtypes = [C.POINTER(Model), C.POINTER(GfIndex), C.POINTER(GfIndex), C.c_double, C.c_int,
                                   _D, C.c_int, _D, _I, _D]
        L.or_integrand_no_det.argtypes = [C.POINTER(Model), C.POINTER(GfIndex), C.POINTER(GfIndex), C.c_double,
                                          C.c_int, _D, C.c_int, _D, _I]
        L.or_evaluate_warped.argtypes = [C.POINTER(Model), C.POINTER(GfIndex), C.POINTER(GfIndex), C.c_double,
                                         C.POINTER(Warper), C.c_int, C.c_int, _D, _D, _I, _D]
        L.or_integrate.argtypes = [C.POINTER(Model), C.POINTER(GfIndex), C.POINTER(GfIndex), C.c_double,
                                   C.POINTER(Warper), C.c_int, C.c_int, _U32, _U32, C.c_int, C.c_uint32, C.c_int64,
                                   C.c_int, C.c_int, _D]
        L.or_compare_3way.argtypes = [C.c_double, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int]
        L.or_integrand_kernel.argtypes = [C.POINTER(Model), C.POINTER(GfIndex), C.c_int, _D, C.c_int, _D, _I, _D]
        L.or_integrate_kernel.argtypes = [C.POINTER(Model), C.POINTER(GfIndex), C.POINTER(Warper), C.c_int, C.c_int,
                                          _U32, _U32, C.c_int, C.c_uint32, C.c_int64, C.c_int, C.c_double, C.c_double,
                                          _D, _D, _D, _D]
        L.or_integrate_binned.argtypes = [C.POINTER(Model), C.POINTER(GfIndex), C.POINTER(GfIndex), C.c_double,
                                          C.POINTER(Warper), C.c_int, C.c_int, _U32, _U32, C.c_int, C.c_uint32,
                                          C.c_int64, C.c_int, C.c_double, C.c_double, _D, _D, _D, _D]

    # --- Sobol -------------------------------------------------------------
    def sobol_matrices(self, dim, m=32):
        out = np.zeros(dim * m, dtype=np.uint32)
        assert self.lib.or_sobol_matrices(dim, m, out.ctypes.data_as(_U32)) == 0
        return out.reshape(dim, m)

    def sobol_setup(self, dim, log_max_points=31, do_shift=False, do_scramble=False, seed_shift=0):
        Csr = np.zeros(dim * log_max_points, dtype=np.uint32)
        shfr = np.zeros(dim, dtype=np.uint32)
        st = self.lib.or_sobol_setup(dim, log_max_points, int(do_shift), int(do_scramble), seed_shift,
                                     Csr.ctypes.data_as(_U32), shfr.ctypes.data_as(_U32))
        assert st == 0
        return Csr, shfr

    def sobol_points(self, dim, seed, count, do_shift=False, do_scramble=False, seed_shift=0, log_max_points=31):
        """`count` successive draws of keldy::sobol(dim, seed[, ...])."""
        Csr, shfr = self.sobol_setup(dim, log_max_points, do_shift, do_scramble, seed_shift)
        out = np.zeros((count, dim))
        st = self.lib.or_sobol_points(dim, log_max_points, Csr.ctypes.data_as(_U32), shfr.ctypes.data_as(_U32),
                                      seed + 1, count, _dp(out))
        assert st == 0
        return out

    # --- Warpers -----------------------------------------------------------
    def warp(self, chain, x, direction="reverse", start=None, end=None):
        x = np.ascontiguousarray(x, dtype=np.float64)
        count, n = x.shape
        arr = chain_array(chain)
        L = len(chain)
        fn = self.lib.or_map_reverse if direction == "reverse" else self.lib.or_map_forward
        if direction == "reverse":
            start = L if start is None else start
            end = 0 if end is None else end
        else:
            start = 0 if start is None else start
            end = L if end is None else end
        out = np.zeros_like(x)
        jac = np.zeros(count)
        for p in range(count):
            j = C.c_double()
            st = fn(arr, L, start, end, n, _dp(x[p]), _dp(out[p]), C.byref(j))
            assert st == 0
            jac[p] = j.value
        return out, jac

    # --- Model / integrand -------------------------------------------------
    def model(self, time_max, lesser, greater, alpha=0.0, lesser_down=None, greater_down=None, interp=1):
        """Tables: complex arrays on the uniform mesh [-time_max, time_max], orbital (0,0).
        interp 3: cubic interpolation (an extension; keldy interpolates linearly)."""
        m = Model()
        npts = len(lesser)
        m.npts = npts
        m.time_max = time_max
        m.alpha = alpha
        m.interp = int(interp)
        keep = []
        def ptr(a):
            a = np.ascontiguousarray(np.asarray(a, dtype=np.complex128).view(np.float64))
            keep.append(a)
            return a.ctypes.data
        # tab index: ((spin*2 + o1)*2 + o2)*2 + lesser/greater
        m.tab[0] = ptr(lesser)
        m.tab[1] = ptr(greater)
        m.tab[8] = ptr(lesser if lesser_down is None else lesser_down)
        m.tab[9] = ptr(greater if greater_down is None else greater_down)
        m._keep = keep
        return m

    def g0(self, model, a, b, internal=True):
        out = np.zeros(2)
        st = self.lib.or_g0(C.byref(model), C.byref(GfIndex(*a)), C.byref(GfIndex(*b)), int(internal), _dp(out))
        assert st == 0
        return complex(out[0], out[1])

    def integrand(self, model, A, B, times, cutoff=0.0, keep_u_hypercube=True, no_det=False):
        """Returns (values complex[count], in_domain int[count], scale[count])."""
        times = np.ascontiguousarray(np.atleast_2d(times), dtype=np.float64)
        count, n = times.shape
        vals = np.zeros(count, dtype=np.complex128)
        dom = np.zeros(count, dtype=np.int32)
        sc = np.zeros(count)
        out = np.zeros(2)
        d = C.c_int()
        s = C.c_double()
        gA, gB = GfIndex(*A), GfIndex(*B)
        for p in range(count):
            if no_det:
                st = self.lib.or_integrand_no_det(C.byref(model), C.byref(gA), C.byref(gB), cutoff, n,
                                                  _dp(times[p]), int(keep_u_hypercube), _dp(out), C.byref(d))
            else:
                st = self.lib.or_integrand(C.byref(model), C.byref(gA), C.byref(gB), cutoff, n, _dp(times[p]),
                                           int(keep_u_hypercube), _dp(out), C.byref(d), C.byref(s))
            assert st == 0, st
            vals[p] = complex(out[0], out[1])
            dom[p] = d.value
            sc[p] = s.value
        return vals, dom, sc

    def evaluate_warped(self, model, A, B, chain, li, cutoff=0.0):
        """Returns (f*J complex[count], J[count], in_domain[count], scale*|J| [count])."""
        li = np.ascontiguousarray(np.atleast_2d(li), dtype=np.float64)
        count, n = li.shape
        arr = chain_array(chain)
        vals = np.zeros(count, dtype=np.complex128)
        jac = np.zeros(count)
        dom = np.zeros(count, dtype=np.int32)
        sc = np.zeros(count)
        out = np.zeros(3)
        d = C.c_int()
        s = C.c_double()
        gA, gB = GfIndex(*A), GfIndex(*B)
        for p in range(count):
            st = self.lib.or_evaluate_warped(C.byref(model), C.byref(gA), C.byref(gB), cutoff, arr, len(chain), n,
                                             _dp(li[p]), _dp(out), C.byref(d), C.byref(s))
            assert st == 0
            vals[p] = complex(out[0], out[1])
            jac[p] = out[2]
            dom[p] = d.value
            sc[p] = s.value
        return vals, jac, dom, sc

    def integrate(self, model, A, B, chain, order, nr_steps, seed=0, cutoff=0.0, do_shift=False, do_scramble=False,
                  seed_shift=0, rank=0, world=1):
        """integrator::run + sums: (sum f*J, n_points, n_in_domain, sum of per-point scales)."""
        Csr, shfr = self.sobol_setup(order, 31, do_shift, do_scramble, seed_shift)
        arr = chain_array(chain)
        res = np.zeros(5)
        st = self.lib.or_integrate(C.byref(model), C.byref(GfIndex(*A)), C.byref(GfIndex(*B)), cutoff, arr,
                                   len(chain), order, Csr.ctypes.data_as(_U32), shfr.ctypes.data_as(_U32), 31,
                                   seed + 1, nr_steps, rank, world, _dp(res))
        assert st == 0
        return complex(res[0], res[1]), int(res[2]), int(res[3]), res[4]

    def integrate_binned(self, model, A, B, chain, order, nr_steps, nbins, xmin, xmax, seed=0, cutoff=0.0,
                         do_shift=False, do_scramble=False, seed_shift=0):
        """integrator<binner_t<1>, integrand_g_direct_time>::run: (sum f*J, n_points, n_in_domain,
        sum of scales, bins complex[nbins], counts[nbins], dropped)."""
        Csr, shfr = self.sobol_setup(order, 31, do_shift, do_scramble, seed_shift)
        arr = chain_array(chain)
        res = np.zeros(5)
        bins = np.zeros(2 * nbins)
        counts = np.zeros(nbins)
        dropped = np.zeros(1)
        st = self.lib.or_integrate_binned(C.byref(model), C.byref(GfIndex(*A)), C.byref(GfIndex(*B)), cutoff, arr,
                                          len(chain), order, Csr.ctypes.data_as(_U32), shfr.ctypes.data_as(_U32), 31,
                                          seed + 1, nr_steps, nbins, xmin, xmax, _dp(res), _dp(bins), _dp(counts),
                                          _dp(dropped))
        assert st == 0
        return (complex(res[0], res[1]), int(res[2]), int(res[3]), res[4], bins.view(np.complex128),
                counts.astype(np.int64), int(dropped[0]))

    def integrand_kernel(self, model, X, times, keep_u_hypercube=True):
        """integrand_g_kernel per point: (sums [count][n][2] complex per (vertex, Keldysh index),
        in_domain, scale)."""
        times = np.ascontiguousarray(np.atleast_2d(times), dtype=np.float64)
        count, n = times.shape
        vals = np.zeros((count, n, 2), dtype=np.complex128)
        dom = np.zeros(count, dtype=np.int32)
        sc = np.zeros(count)
        out = np.zeros(4 * n)
        d = C.c_int()
        s = C.c_double()
        gX = GfIndex(*X)
        for p in range(count):
            assert self.lib.or_integrand_kernel(C.byref(model), C.byref(gX), n, _dp(times[p]), int(keep_u_hypercube),
                                                _dp(out), C.byref(d), C.byref(s)) == 0
            vals[p] = out.view(np.complex128).reshape(n, 2)
            dom[p] = d.value
            sc[p] = s.value
        return vals, dom, sc

    def integrate_kernel(self, model, X, chain, order, nr_steps, nbins, xmin, xmax, seed=0, do_shift=False,
                         do_scramble=False, seed_shift=0):
        """integrator<binner_t<1,1>, integrand_g_kernel>::run: (sum, n_points, n_in_domain, sum of
        moduli, bins complex[nbins][2], counts[nbins][2], dropped)."""
        Csr, shfr = self.sobol_setup(order, 31, do_shift, do_scramble, seed_shift)
        arr = chain_array(chain)
        res = np.zeros(5)
        bins = np.zeros(4 * nbins)
        counts = np.zeros(2 * nbins)
        dropped = np.zeros(1)
        st = self.lib.or_integrate_kernel(C.byref(model), C.byref(GfIndex(*X)), arr, len(chain), order,
                                          Csr.ctypes.data_as(_U32), shfr.ctypes.data_as(_U32), 31, seed + 1, nr_steps,
                                          nbins, xmin, xmax, _dp(res), _dp(bins), _dp(counts), _dp(dropped))
        assert st == 0
        return (complex(res[0], res[1]), int(res[2]), int(res[3]), res[4], bins.view(np.complex128).reshape(nbins, 2),
                counts.reshape(nbins, 2).astype(np.int64), int(dropped[0]))

    def compare_3way(self, a, b):
        return self.lib.or_compare_3way(a[0], a[1], a[2], b[0], b[1], b[2])


def _cpu_has_v3():
    if platform.machine() not in ("x86_64", "AMD64"):
        return False
    try:
        flags = open("/proc/cpuinfo").read()
    except OSError:
        return False
    return all(f in flags for f in (" avx2", " fma", " bmi2", " movbe"))


class Reference:
    """keldy's own sources compiled against the stand-in headers (oracle/_ref)."""

    def __init__(self, timed=False):
        """timed=True picks the x86-64-v3 build when the host supports it (the CPU baseline);
        the default build has no FMA contraction, for validating the restatement."""
        name = "libkeldy_ref_v3.so" if (timed and _cpu_has_v3()) else "libkeldy_ref.so"
        path = os.path.join(HERE, "_ref", name)
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.path = path
        L = self.lib = C.CDLL(path)
        L.ref_last_error.restype = C.c_char_p
        L.ref_sobol_points.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_long, _D]
        L.ref_sobol_matrices.argtypes = [C.c_int, C.c_int, _U32]
        L.ref_warp.argtypes = [C.POINTER(Warper), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_long, _D, _D, _D]
        L.ref_model_create.argtypes = [C.c_int, C.c_double, C.c_double, _D, _D]
        L.ref_model_create.restype = C.c_void_p
        L.ref_model_destroy.argtypes = [C.c_void_p]
        L.ref_g0.argtypes = [C.c_void_p, C.POINTER(GfIndex), C.POINTER(GfIndex), C.c_int, _D]
        L.ref_integrand.argtypes = [C.c_void_p, C.POINTER(GfIndex), C.POINTER(GfIndex), C.c_double, C.c_int,
                                    C.c_long, _D, C.c_int, C.c_int, _D, _I]
        L.ref_integrate.argtypes = [C.c_void_p, C.POINTER(GfIndex), C.POINTER(GfIndex), C.c_double,
                                    C.POINTER(Warper), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                    C.c_long, C.c_int, C.c_int, _D]
        L.ref_interp_nearest.argtypes = [C.c_int, _D, _D, C.c_int, C.c_int, C.c_long, _D, _D, _D]

    def _check(self, st):
        if st != 0:
            raise RuntimeError(self.lib.ref_last_error().decode())

    def interp_nearest(self, u, f1, x, direction="reverse"):
        """keldy's warper_product_1d_simple_interp_nearest_t(u, f1).map_reverse / map_forward
        on the rows of x."""
        u = np.ascontiguousarray(u, dtype=np.float64)
        f1 = np.ascontiguousarray(f1, dtype=np.float64)
        x = np.ascontiguousarray(np.atleast_2d(x), dtype=np.float64)
        out = np.zeros_like(x)
        jac = np.zeros(len(x))
        self._check(self.lib.ref_interp_nearest(len(u), _dp(u), _dp(f1), 0 if direction == "reverse" else 1,
                                                x.shape[1], len(x), _dp(x), _dp(out), _dp(jac)))
        return out, jac

    def sobol_matrices(self, dim, m=32):
        out = np.zeros(dim * m, dtype=np.uint32)
        self._check(self.lib.ref_sobol_matrices(dim, m, out.ctypes.data_as(_U32)))
        return out.reshape(dim, m)

    def sobol_points(self, dim, seed, count, do_shift=False, do_scramble=False, seed_shift=0, log_max_points=31):
        out = np.zeros((count, dim))
        self._check(self.lib.ref_sobol_points(dim, seed, int(do_shift), int(do_scramble), seed_shift,
                                              log_max_points, count, _dp(out)))
        return out

    def warp(self, chain, x, direction="reverse", start=None, end=None):
        x = np.ascontiguousarray(x, dtype=np.float64)
        count, n = x.shape
        L = len(chain)
        if direction == "reverse":
            start = L if start is None else start
            end = 0 if end is None else end
        else:
            start = 0 if start is None else start
            end = L if end is None else end
        out = np.zeros_like(x)
        jac = np.zeros(count)
        self._check(self.lib.ref_warp(chain_array(chain), L, 0 if direction == "reverse" else 1, start, end, n,
                                      count, _dp(x), _dp(out), _dp(jac)))
        return out, jac

    def model(self, time_max, lesser, greater, alpha=0.0):
        le = np.ascontiguousarray(np.asarray(lesser, dtype=np.complex128).view(np.float64))
        gr = np.ascontiguousarray(np.asarray(greater, dtype=np.complex128).view(np.float64))
        h = self.lib.ref_model_create(len(lesser), time_max, alpha, _dp(le), _dp(gr))
        return _RefModel(self, h)

    def g0(self, model, a, b, internal=True):
        out = np.zeros(2)
        self._check(self.lib.ref_g0(model.h, C.byref(GfIndex(*a)), C.byref(GfIndex(*b)), int(internal), _dp(out)))
        return complex(out[0], out[1])

    def integrand(self, model, A, B, times, cutoff=0.0, keep_u_hypercube=True, no_det=False):
        times = np.ascontiguousarray(np.atleast_2d(times), dtype=np.float64)
        count, n = times.shape
        out = np.zeros(2 * count)
        dom = np.zeros(count, dtype=np.int32)
        self._check(self.lib.ref_integrand(model.h, C.byref(GfIndex(*A)), C.byref(GfIndex(*B)), cutoff, n, count,
                                           _dp(times), int(keep_u_hypercube), int(no_det), _dp(out),
                                           dom.ctypes.data_as(_I)))
        return out.view(np.complex128), dom

    def integrate(self, model, A, B, chain, order, nr_steps, seed=0, cutoff=0.0, do_shift=False, do_scramble=False,
                  seed_shift=0, mode=0, threads=1):
        res = np.zeros(4)
        self._check(self.lib.ref_integrate(model.h, C.byref(GfIndex(*A)), C.byref(GfIndex(*B)), cutoff,
                                           chain_array(chain), len(chain), order, seed, int(do_shift),
                                           int(do_scramble), seed_shift, nr_steps, mode, threads, _dp(res)))
        return complex(res[0], res[1]), int(res[2]), int(res[3])


class _RefModel:
    def __init__(self, ref, h):
        self.ref, self.h = ref, h

    def __del__(self):
        try:
            self.ref.lib.ref_model_destroy(self.h)
        except Exception:
            pass


def reference_available():
    return os.path.exists(os.path.join(HERE, "_ref", "libkeldy_ref.so"))
