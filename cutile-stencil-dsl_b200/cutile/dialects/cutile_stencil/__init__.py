"""Dialect 1 (``cutile_stencil``): the ``@stencil`` function as parsed.

Same op and attribute set as the reference (cutile/dialects/cutile_stencil/
dialect.py:59-369): ``func`` (func_name, ndim, order, dtype, boundary,
constants, arg_names), ``access`` (field, offset, index_names), ``yield``,
plus the unused ``compute`` op and ``spec`` attribute.
"""

from cutile.dialects.cutile_stencil.dialect import (
    AccessOp,
    BoundaryAttr,
    ComputeOp,
    CutileStencilDialect,
    FuncOp,
    StencilSpecAttr,
    YieldOp,
)

__all__ = ["AccessOp", "BoundaryAttr", "ComputeOp", "CutileStencilDialect", "FuncOp",
           "StencilSpecAttr", "YieldOp"]
