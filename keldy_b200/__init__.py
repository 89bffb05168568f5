"""keldy_b200: keldy's quasi-Monte-Carlo integrand pipeline (Sobol points -> warper
chain -> Wick-determinant integrand -> QMC sum) on NVIDIA B200 (sm_100a).

Layers:
  * ``libkeldy_b200.so`` (csrc/): the CUDA kernels behind a C ABI (include/keldy_b200.h);
  * ``capi``: ctypes binding of that C ABI;
  * ``g0_tables``: host-side g0 tables of the flat-band dot model.
There is no CPU implementation of the path: without the shared library or a CUDA device
the calls raise.
"""
__version__ = "0.1.0"
