"""Normalization: Dialect 1 -> standard ``stencil`` dialect (Dialect 2).

Follows cutile/lowering/normalize.py:47-156: every ``cutile_stencil.func``
becomes ``func.func`` wrapping one ``stencil.apply`` whose body has one
``TempType`` argument per input array, ``stencil.access`` per D1 access, the
cloned arith/math ops and ``stencil.return``.  ``ndim``, ``order``, ``dtype``,
``num_arrays``, ``boundary`` and ``constants`` become attributes of the apply;
the func carries ``stencil_ndim/order/dtype`` (and ``boundary``).
"""

from __future__ import annotations

from dataclasses import dataclass

from cutile.dialects.cutile_stencil.dialect import AccessOp as D1AccessOp
from cutile.dialects.cutile_stencil.dialect import FuncOp as D1FuncOp
from cutile.dialects.cutile_stencil.dialect import YieldOp as D1YieldOp
from cutile.dialects.stencil import AccessOp as StdAccessOp
from cutile.dialects.stencil import ApplyOp, ReturnOp, StdFuncOp
from cutile.ir.core import (
    Block,
    Context,
    FunctionType,
    IntAttr,
    ModuleOp,
    ModulePass,
    Region,
    StringAttr,
    TempType,
    f32,
    f64,
)


@dataclass(frozen=True)
class NormalizePass(ModulePass):
    name = "normalize"

    def apply(self, ctx: Context, op: ModuleOp) -> None:
        for d1 in [c for c in op.walk() if isinstance(c, D1FuncOp)]:
            self._convert_func(d1)

    @staticmethod
    def _convert_func(d1: D1FuncOp) -> None:
        func_name = d1.func_name.data
        ndim = d1.ndim.data
        order = d1.order.data
        dtype_str = d1.dtype.data if d1.dtype is not None else "float64"
        float_type = f32 if dtype_str == "float32" else f64
        d1_body = d1.body.blocks[0]
        n_scalars = len(d1.scalar_names.data) if d1.scalar_names is not None else 0
        num_arrays = len(d1_body.args) - n_scalars
        temp_type = TempType(ndim, float_type)

        block = Block()
        vmap = {}
        for idx in range(num_arrays):
            vmap[d1_body.args[idx]] = block.insert_arg(temp_type, idx)
        for k in range(n_scalars):
            vmap[d1_body.args[num_arrays + k]] = block.insert_arg(f64, num_arrays + k)
        for op in d1_body.ops:
            if isinstance(op, D1AccessOp):
                new = StdAccessOp(vmap[op.field], list(op.offset.offsets))
                block.add_op(new)
                vmap[op.res] = new.res
            elif isinstance(op, D1YieldOp):
                block.add_op(ReturnOp([vmap[v] for v in op.values]))
            else:
                new = op.clone(vmap)
                block.add_op(new)

        apply_op = ApplyOp([], block, [TempType(ndim, float_type)])
        apply_op.attributes["ndim"] = IntAttr(ndim)
        apply_op.attributes["order"] = IntAttr(order)
        apply_op.attributes["dtype"] = StringAttr(dtype_str)
        apply_op.attributes["num_arrays"] = IntAttr(num_arrays)
        if d1.boundary is not None:
            apply_op.attributes["boundary"] = d1.boundary
        if d1.constants is not None:
            apply_op.attributes["constants"] = d1.constants

        ftype = FunctionType.from_lists([temp_type] * num_arrays, [TempType(ndim, float_type)])
        std = StdFuncOp(func_name, ftype, Region(Block([apply_op])))
        std.attributes["stencil_ndim"] = IntAttr(ndim)
        std.attributes["stencil_order"] = IntAttr(order)
        std.attributes["stencil_dtype"] = StringAttr(dtype_str)
        if d1.boundary is not None:
            std.attributes["boundary"] = d1.boundary

        parent = d1.parent_block()
        parent.add_op(std)
        d1.detach()
