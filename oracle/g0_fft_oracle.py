"""CPU restatement of keldy's ft_method "fft" table construction (test infrastructure only).

keldy's make_g0_by_fft (c++/keldy/impurity_oneband/model.cpp:179-212) samples the dot's
frequency functions on the mesh adjoint to the time mesh and transforms them with TRIQS's
make_gf_from_fourier (TRIQS 3.0.x, triqs/gfs/transform/fourier_real.cpp, absent from the
reference tree). Its published convention, restated here with numpy's FFT:

* time mesh t_k = (k - c) dt, k = 0..L-1, c = (L-1)/2, L odd (model.cpp:87-90);
* adjoint frequency mesh w_j = (j - c) dw, dw = 2 pi/(L dt) (make_adjoint_mesh);
* g(t_k) = dw/(2 pi) sum_j g(w_j) e^{-i w_j t_k}, the 1/w^2 tails beyond the mesh taken into
  account by subtracting m2/(w^2 + a^2) (a = dw sqrt(L)) before the sum and adding its exact
  transform m2 e^{-a|t|}/(2a) after; m2 = the mean of w^2 g(w) at the mesh's two ends.

Pinned by keldy's fft known answers (model_flatband_test.cpp:60-269,
model_semicircle_test.cpp:20-60) in tests/test_g0_fft_oracle.py. Only tests/ import this.
"""
from __future__ import annotations

import numpy as np


def transform(g_w, time_max):
    """The fft-method table of frequency values g_w (length L, odd) on the adjoint mesh of the
    time mesh [-time_max, time_max]."""
    g_w = np.asarray(g_w, dtype=np.complex128)
    L = len(g_w)
    assert L % 2 == 1
    c = (L - 1) // 2
    dt = 2.0 * time_max / (L - 1)
    dw = 2.0 * np.pi / (L * dt)
    a = dw * np.sqrt(L)
    w = (np.arange(L) - c) * dw
    t = (np.arange(L) - c) * dt
    wmax = np.pi * (L - 1) / (L * dt)
    m2 = 0.5 * wmax * wmax * (g_w[0] + g_w[-1])
    h = g_w - m2 / (w * w + a * a)
    # sum_j h_j e^{-2 pi i (j-c)(k-c)/L} = e^{2 pi i c (k-c)/L} sum_j h_j e^{-2 pi i j (k-c)/L}
    kc = np.arange(L) - c
    s = np.exp(2j * np.pi * c * kc / L) * np.fft.fft(h)[kc % L]
    return dw / (2.0 * np.pi) * s + m2 * np.exp(-a * np.abs(t)) / (2.0 * a)
