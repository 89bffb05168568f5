"""keldy.common (python/keldy/common_desc.py) on keldy_b200: Sobol points on the GPU."""
from ._keldy import ContourPtT, Sobol, compare_3way, keldysh_idx_t, spin_t  # noqa: F401

up, down = spin_t.up, spin_t.down
forward, backward = keldysh_idx_t.forward, keldysh_idx_t.backward

__all__ = ["ContourPtT", "Sobol", "compare_3way", "spin_t", "keldysh_idx_t", "up", "down", "forward", "backward"]
