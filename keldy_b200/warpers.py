"""keldy.warpers (python/keldy/warpers_desc.py) on keldy_b200: the analytic warpers and
their chains, evaluated on the GPU."""
from ._keldy import (WarperIdentityT, WarperPlasmaUvT, WarperProduct1dSimpleT, WarperTrainT,  # noqa: F401
                     make_product_1d_simple_exponential, make_product_1d_simple_inverse,
                     make_product_1d_simple_inverse_power, make_product_1d_simple_inverse_square,
                     make_product_1d_simple_uniform, ui_from_vi, vi_from_ui)

__all__ = ["WarperIdentityT", "WarperPlasmaUvT", "WarperProduct1dSimpleT", "WarperTrainT",
           "make_product_1d_simple_exponential", "make_product_1d_simple_inverse",
           "make_product_1d_simple_inverse_square", "make_product_1d_simple_inverse_power",
           "make_product_1d_simple_uniform", "vi_from_ui", "ui_from_vi"]
