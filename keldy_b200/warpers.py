"""keldy.warpers (python/keldy/warpers_desc.py) on keldy_b200: the analytic and tabulated
warpers and their chains, evaluated on the GPU, and make_warper_from_proj."""
from ._keldy import (WarperIdentityT, WarperPlasmaUvT, WarperProduct1dInterpNearestT,  # noqa: F401
                     WarperProduct1dSimpleInterpNearestT, WarperProduct1dSimpleT, WarperTrainT,
                     make_product_1d_simple_exponential, make_product_1d_simple_inverse,
                     make_product_1d_simple_inverse_power, make_product_1d_simple_inverse_square,
                     make_product_1d_simple_uniform, make_warper_from_proj, ui_from_vi, vi_from_ui)

__all__ = ["WarperIdentityT", "WarperPlasmaUvT", "WarperProduct1dSimpleT", "WarperTrainT",
           "WarperProduct1dSimpleInterpNearestT", "WarperProduct1dInterpNearestT", "make_warper_from_proj",
           "make_product_1d_simple_exponential", "make_product_1d_simple_inverse",
           "make_product_1d_simple_inverse_square", "make_product_1d_simple_inverse_power",
           "make_product_1d_simple_uniform", "vi_from_ui", "ui_from_vi"]
