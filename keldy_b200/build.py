"""Builds the keldy_b200 shared libraries in-tree for sm_100a.

* ``keldy_b200/libkeldy_b200.so``: the CUDA kernels and the C ABI (include/keldy_b200.h).
* ``keldy_b200/_keldy*.so``: the Python bindings of the C++ host classes
  (include/keldy_b200.hpp), linked against libkeldy_b200.so.

nvcc cross-compiles for sm_100a without a GPU, so this runs anywhere the CUDA toolkit is.
"""
from __future__ import annotations

import os
import subprocess
import sys
import sysconfig

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(PKG, "libkeldy_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I" + INCLUDE, "-I" + CSRC] + ARCH
CUDA_SOURCES = ["tree.cu", "misc_kernels.cu", "flow.cu", "flow_spline.cu", "flow_arspline.cu", "g0_build.cu", "capi.cu", "flow_capi.cu", "table_capi.cu", "host_sobol.cpp"]
HEADERS = ["kb_types.h", "kb_device.cuh", "kb_launch.h", "kb_flow.h", "kb_host.h", "kb_spline.cuh", "sobol_joe_kuo.h"]


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build_cuda(verbose=False, ptxas_verbose=False):
    deps = [os.path.join(CSRC, f) for f in CUDA_SOURCES + HEADERS] + [os.path.join(INCLUDE, "keldy_b200.h")]
    objs = []
    for src in CUDA_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(CSRC, "_build", src + ".o")
        os.makedirs(os.path.dirname(o), exist_ok=True)
        hdeps = [s] + [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "keldy_b200.h")]
        if _stale(o, hdeps):
            extra = ["-Xptxas", "-v"] if (ptxas_verbose and src.endswith(".cu")) else []
            lang = ["-x", "cu"] if src.endswith(".cu") else []
            _run([_nvcc()] + NVCC_FLAGS + extra + lang + ["-c", s, "-o", o], verbose)
        objs.append(o)
    if _stale(LIB, objs + deps):
        _run([_nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"], verbose)
    return LIB


def build_bindings(verbose=False):
    import pybind11

    src = os.path.join(CSRC, "bindings.cpp")
    if not os.path.exists(src):
        return None
    suffix = sysconfig.get_config_var("EXT_SUFFIX") or ".so"
    out = os.path.join(PKG, "_keldy" + suffix)
    deps = [src, LIB, os.path.join(INCLUDE, "keldy_b200.hpp"), os.path.join(INCLUDE, "keldy_b200.h")]
    if _stale(out, deps):
        py_inc = sysconfig.get_paths()["include"]
        cmd = ["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-I" + INCLUDE, "-I" + pybind11.get_include(),
               "-I" + py_inc, src, "-o", out, "-L" + PKG, "-lkeldy_b200", "-Wl,-rpath,$ORIGIN"]
        _run(cmd, verbose)
    return out


def build(verbose=False, ptxas_verbose=False):
    build_cuda(verbose, ptxas_verbose)
    build_bindings(verbose)


if __name__ == "__main__":
    build(verbose=True, ptxas_verbose="-v" in sys.argv)
