"""keldy.warpers (python/keldy/warpers_desc.py) on keldy_b200: the analytic, tabulated,
hybrid and projection warpers and their chains, evaluated on the GPU, make_warper_from_proj
and the makers of warper_product_1d_t."""
from ._keldy import (WarperIdentityT, WarperPlasmaUvT, WarperProduct1dInterpHybridT,  # noqa: F401
                     WarperProduct1dInterpNearestT, WarperProduct1dSimpleInterpHybridT,
                     WarperProduct1dSimpleInterpNearestT, WarperProduct1dSimpleT, WarperProduct1dT, WarperProjectionT,
                     WarperTrainT, make_product_1d_inverse_cube_alternate,
                     make_product_1d_inverse_cube_alternate_interp_hybrid,
                     make_product_1d_inverse_cube_alternate_interp_nearest, make_product_1d_simple_exponential,
                     make_product_1d_simple_inverse, make_product_1d_simple_inverse_power,
                     make_product_1d_simple_inverse_square, make_product_1d_simple_uniform, make_projection_warper,
                     make_warper_from_proj, ui_from_vi, vi_from_ui)

__all__ = ["WarperIdentityT", "WarperPlasmaUvT", "WarperProduct1dSimpleT", "WarperTrainT",
           "WarperProduct1dSimpleInterpNearestT", "WarperProduct1dInterpNearestT", "WarperProduct1dT",
           "WarperProduct1dSimpleInterpHybridT", "WarperProduct1dInterpHybridT", "WarperProjectionT",
           "make_warper_from_proj", "make_projection_warper", "make_product_1d_inverse_cube_alternate",
           "make_product_1d_inverse_cube_alternate_interp_nearest",
           "make_product_1d_inverse_cube_alternate_interp_hybrid",
           "make_product_1d_simple_exponential", "make_product_1d_simple_inverse",
           "make_product_1d_simple_inverse_square", "make_product_1d_simple_inverse_power",
           "make_product_1d_simple_uniform", "vi_from_ui", "ui_from_vi"]
