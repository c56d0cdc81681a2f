"""Dialect 1 ops and attributes (reference: cutile/dialects/cutile_stencil/dialect.py)."""

from __future__ import annotations

from typing import Sequence

from cutile.dialects._base import BuildMixin, Dialect, attr, prop
from cutile.ir.core import (
    ArrayAttr,
    Attribute,
    Block,
    DictionaryAttr,
    FloatAttr,
    IndexAttr,
    IntAttr,
    Operation,
    Region,
    SSAValue,
    StringAttr,
    f64,
)

VALID_BC_TYPES = frozenset({"dirichlet", "neumann", "periodic", "reflecting"})


class BoundaryAttr(Attribute):
    """Boundary-condition type and optional value (dialect.py:59-111).

    ``value`` is a ``FloatAttr`` when given, else ``IntAttr(0)`` as the
    "no value" sentinel, exactly as in the reference.
    """

    name = "cutile_stencil.boundary"

    def __init__(self, bc_type: str | StringAttr, value: float | FloatAttr | None = None):
        if isinstance(bc_type, str):
            bc_type = StringAttr(bc_type)
        if value is None:
            value_attr: Attribute = IntAttr(0)
        elif isinstance(value, (int, float)):
            value_attr = FloatAttr(float(value), f64)
        else:
            value_attr = value
        self.bc_type = bc_type
        self.value = value_attr
        self.verify()

    @property
    def has_value(self) -> bool:
        return isinstance(self.value, FloatAttr)

    @property
    def bc_type_str(self) -> str:
        return self.bc_type.data

    def verify(self) -> None:
        if self.bc_type.data not in VALID_BC_TYPES:
            raise ValueError(
                f"Invalid boundary type '{self.bc_type.data}'. "
                f"Expected one of {sorted(VALID_BC_TYPES)}.")

    def _key(self):
        return (self.bc_type.data, self.value)

    def print(self) -> str:
        v = self.value.print() if self.has_value else "none"
        return f"#cutile_stencil.boundary<{self.bc_type.data}, {v}>"


class StencilSpecAttr(Attribute):
    """Compound stencil metadata (dialect.py:114-161); not used by the passes."""

    name = "cutile_stencil.spec"

    def __init__(self, ndim, order, dtype="float64", boundary=None):
        self.ndim = ndim if isinstance(ndim, IntAttr) else IntAttr(ndim)
        self.order = order if isinstance(order, IntAttr) else IntAttr(order)
        self.dtype = dtype if isinstance(dtype, StringAttr) else StringAttr(dtype)
        self.boundary = IntAttr(0) if boundary is None else boundary

    @property
    def has_boundary(self) -> bool:
        return not isinstance(self.boundary, IntAttr)

    def _key(self):
        return (self.ndim, self.order, self.dtype, self.boundary)

    def print(self) -> str:
        return (f"#cutile_stencil.spec<{self.ndim.data}, {self.order.data}, "
                f"{self.dtype.data}, {self.boundary.print()}>")


class FuncOp(BuildMixin, Operation):
    """A complete stencil function (dialect.py:169-244)."""

    name = "cutile_stencil.func"
    func_name = prop()
    ndim = prop()
    order = prop()
    dtype = prop()
    boundary = prop()
    constants = prop()
    arg_names = prop()
    scalar_names = prop()

    def __init__(self, func_name, ndim, order, body: Region | Block, input_types=(),
                 output_types=(), dtype=None, boundary=None, constants=None,
                 arg_names: Sequence[str] | None = None, *, operands=()):
        if isinstance(body, Block):
            body = Region(body)
        props = {"func_name": func_name, "ndim": ndim, "order": order}
        if dtype is not None:
            props["dtype"] = dtype
        if boundary is not None:
            props["boundary"] = boundary
        if constants is not None:
            props["constants"] = constants
        if arg_names is not None:
            props["arg_names"] = ArrayAttr([StringAttr(n) for n in arg_names])
        super().__init__(operands=list(operands), result_types=list(output_types),
                         properties=props, regions=[body])


class AccessOp(BuildMixin, Operation):
    """Read a field at a relative offset (dialect.py:247-315)."""

    name = "cutile_stencil.access"
    offset = attr()
    index_names = attr()

    def __init__(self, field, offset: Sequence[int] | IndexAttr, result_type,
                 index_names: Sequence[str] | ArrayAttr | None = None):
        if not isinstance(offset, IndexAttr):
            offset = IndexAttr(offset)
        attrs = {"offset": offset}
        if index_names is not None:
            if not isinstance(index_names, ArrayAttr):
                index_names = ArrayAttr([StringAttr(n) for n in index_names])
            attrs["index_names"] = index_names
        super().__init__(operands=[field], result_types=[result_type], attributes=attrs)

    @property
    def field(self) -> SSAValue:
        return self.operands[0]

    def print_custom(self, printer):
        text = f" {printer.print_operand(self.field)} [" + ", ".join(
            str(o) for o in self.offset.offsets) + "]"
        if self.index_names is not None:
            text += " {" + ", ".join(f'"{a.data}"' for a in self.index_names) + "}"
        return text + " : " + self.res.type.print()


class ComputeOp(BuildMixin, Operation):
    """Region-carrying compute op (declared by the reference, never built)."""

    name = "cutile_stencil.compute"

    def __init__(self, body: Region | Block, result_type):
        if isinstance(body, Block):
            body = Region(body)
        super().__init__(result_types=[result_type], regions=[body])


class YieldOp(BuildMixin, Operation):
    """Terminator yielding the stencil's point value(s) (dialect.py:345-358;
    several values for a tuple-returning body)."""

    name = "cutile_stencil.yield"

    def __init__(self, *values):
        super().__init__(operands=list(values))

    @property
    def value(self) -> SSAValue:
        return self.operands[0]

    @property
    def values(self) -> tuple:
        return self.operands

    def print_custom(self, printer):
        return (" " + ", ".join(printer.print_operand(v) for v in self.operands) + " : "
                + ", ".join(v.type.print() for v in self.operands))


CutileStencilDialect = Dialect("cutile_stencil", [FuncOp, AccessOp, ComputeOp, YieldOp],
                               [BoundaryAttr, StencilSpecAttr])
