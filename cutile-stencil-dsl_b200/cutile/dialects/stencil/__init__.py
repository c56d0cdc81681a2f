"""Dialect 2: the standard ``stencil`` dialect subset (apply / access / return).

The reference uses ``xdsl.dialects.stencil`` (normalize.py:93-99); this is the
subset its passes touch: ``stencil.apply`` with a body block of ``TempType``
arguments and an attribute dictionary the analysis passes annotate,
``stencil.access`` (temp + ``IndexAttr`` offset) and ``stencil.return``.
``func.func`` wraps each apply.
"""

from __future__ import annotations

from cutile.dialects._base import BuildMixin, Dialect, prop
from cutile.ir.core import (
    Block,
    FunctionType,
    IndexAttr,
    Operation,
    Region,
    SSAValue,
    StringAttr,
    TempType,
)


class ApplyOp(BuildMixin, Operation):
    name = "stencil.apply"

    def __init__(self, args, body: Block | Region, result_types):
        if isinstance(body, Block):
            body = Region(body)
        super().__init__(operands=list(args), result_types=list(result_types), regions=[body])

    @property
    def region(self) -> Region:
        return self.regions[0]

    @property
    def res(self):
        return self.results


class AccessOp(BuildMixin, Operation):
    name = "stencil.access"

    def __init__(self, temp, offset):
        if not isinstance(offset, IndexAttr):
            offset = IndexAttr(list(offset))
        t = temp if isinstance(temp, SSAValue) else temp.results[0]
        elem = t.type.element_type if isinstance(t.type, TempType) else t.type
        super().__init__(operands=[temp], result_types=[elem], properties={"offset": offset})

    @property
    def temp(self) -> SSAValue:
        return self.operands[0]

    @property
    def offset(self) -> IndexAttr:
        return self.properties["offset"]

    def print_custom(self, printer):
        return (f" {printer.print_operand(self.temp)}{self.offset.print()} : "
                f"{self.temp.type.print()}")


class ReturnOp(BuildMixin, Operation):
    name = "stencil.return"

    def __init__(self, values):
        super().__init__(operands=list(values))

    def print_custom(self, printer):
        return " " + ", ".join(printer.print_operand(v) for v in self.operands)


class StdFuncOp(BuildMixin, Operation):
    """``func.func`` wrapping a ``stencil.apply``."""

    name = "func.func"
    sym_name = prop()
    function_type = prop()

    def __init__(self, name: str, function_type: FunctionType, body: Region):
        super().__init__(properties={"sym_name": StringAttr(name),
                                     "function_type": function_type}, regions=[body])


StencilDialect = Dialect("stencil", [ApplyOp, AccessOp, ReturnOp])
Func = Dialect("func", [StdFuncOp])

__all__ = ["ApplyOp", "AccessOp", "ReturnOp", "StdFuncOp", "TempType", "IndexAttr",
           "StencilDialect", "Func"]
