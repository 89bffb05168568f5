"""Host-side checks that need no GPU: the C ABI library loads and exports every symbol
of include/keldy_b200.h, and the host Sobol set-up equals keldy's."""
import os
import re

import numpy as np
import pytest

from keldy_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "keldy_b200.h")).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(kb_\w+)\(", src, re.M)))


def test_library_exports_every_declared_symbol():
    L = capi.load()
    names = declared_symbols()
    assert len(names) >= 20
    for name in names:
        assert hasattr(L, name), name
    assert sorted(capi.EXPORTS) == names


def test_host_sobol_matrices_equal_keldy(oracle):
    for dim, m, sh, sc, ss in [(1, 31, 0, 0, 0), (12, 31, 0, 0, 0), (12, 31, 1, 0, 3), (30, 31, 0, 1, 7),
                               (250, 31, 1, 1, -2), (7, 16, 1, 1, 99)]:
        Csr, shfr = capi.sobol_matrices(dim, m, sh, sc, ss)
        c, s = oracle.sobol_setup(dim, m, bool(sh), bool(sc), ss)
        assert np.array_equal(Csr.ravel(), c) and np.array_equal(shfr, s)


def test_host_sobol_errors():
    with pytest.raises(capi.KbError):
        capi.sobol_matrices(0)
    with pytest.raises(capi.KbError):
        capi.sobol_matrices(251)
    with pytest.raises(capi.KbError):
        capi.sobol_matrices(3, 32)


def test_no_cpu_path_without_device():
    """Without a CUDA device the library refuses to run instead of computing on the CPU."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(capi.KbError) as e:
        capi.Context(0)
    assert e.value.code in (capi.KB_E_NODEVICE, capi.KB_E_CUDA)
