"""``arith`` / ``math`` ops used in stencil bodies.

The reference's parser emits xDSL's ``arith.constant/addf/subf/mulf/divf/negf/
maximumf/minimumf/cmpf/select`` and ``math.absf`` (parser.py:260-331).  The
same op set is defined here, plus ``math.sqrt`` (an extension: the nonlinear
shallow-water flux needs the wave speed ``sqrt(g*h)``).
"""

from __future__ import annotations

from cutile.dialects._base import BuildMixin, Dialect, prop
from cutile.ir.core import FloatAttr, IntAttr, Operation, SSAValue, i1

# arith.cmpf predicate encoding (MLIR): ordered comparisons and ``une``
CMPF_PREDICATES = {
    "false": 0, "oeq": 1, "ogt": 2, "oge": 3, "olt": 4, "ole": 5, "one": 6, "ord": 7,
    "ueq": 8, "ugt": 9, "uge": 10, "ult": 11, "ule": 12, "une": 13, "uno": 14, "true": 15,
}


class ConstantOp(BuildMixin, Operation):
    name = "arith.constant"
    value = prop()

    def __init__(self, value: FloatAttr):
        super().__init__(result_types=[value.type], properties={"value": value})

    def print_custom(self, printer):
        return " " + self.properties["value"].print()


class _BinaryOp(BuildMixin, Operation):
    def __init__(self, lhs, rhs):
        lhs_v = lhs if isinstance(lhs, SSAValue) else lhs.results[0]
        super().__init__(operands=[lhs, rhs], result_types=[lhs_v.type])

    @property
    def lhs(self) -> SSAValue:
        return self.operands[0]

    @property
    def rhs(self) -> SSAValue:
        return self.operands[1]

    def print_custom(self, printer):
        return (f" {printer.print_operand(self.lhs)}, {printer.print_operand(self.rhs)} : "
                f"{self.result.type.print()}")


class AddfOp(_BinaryOp):
    name = "arith.addf"


class SubfOp(_BinaryOp):
    name = "arith.subf"


class MulfOp(_BinaryOp):
    name = "arith.mulf"


class DivfOp(_BinaryOp):
    name = "arith.divf"


class MaximumfOp(_BinaryOp):
    name = "arith.maximumf"


class MinimumfOp(_BinaryOp):
    name = "arith.minimumf"


class _UnaryOp(BuildMixin, Operation):
    def __init__(self, operand):
        v = operand if isinstance(operand, SSAValue) else operand.results[0]
        super().__init__(operands=[operand], result_types=[v.type])

    @property
    def operand(self) -> SSAValue:
        return self.operands[0]

    def print_custom(self, printer):
        return f" {printer.print_operand(self.operand)} : {self.result.type.print()}"


class NegfOp(_UnaryOp):
    name = "arith.negf"


class CmpfOp(BuildMixin, Operation):
    name = "arith.cmpf"
    predicate = prop()

    def __init__(self, lhs, rhs, predicate: str | int):
        if isinstance(predicate, str):
            predicate = CMPF_PREDICATES[predicate]
        super().__init__(operands=[lhs, rhs], result_types=[i1],
                         properties={"predicate": IntAttr(predicate)})

    @property
    def lhs(self):
        return self.operands[0]

    @property
    def rhs(self):
        return self.operands[1]

    def print_custom(self, printer):
        inv = {v: k for k, v in CMPF_PREDICATES.items()}
        return (f" {inv[self.predicate.data]}, {printer.print_operand(self.lhs)}, "
                f"{printer.print_operand(self.rhs)} : {self.lhs.type.print()}")


class SelectOp(BuildMixin, Operation):
    name = "arith.select"

    def __init__(self, cond, a, b):
        av = a if isinstance(a, SSAValue) else a.results[0]
        super().__init__(operands=[cond, a, b], result_types=[av.type])

    @property
    def cond(self):
        return self.operands[0]

    def print_custom(self, printer):
        c, a, b = (printer.print_operand(o) for o in self.operands)
        return f" {c}, {a}, {b} : {self.result.type.print()}"


class AbsFOp(_UnaryOp):
    name = "math.absf"


class SqrtOp(_UnaryOp):
    name = "math.sqrt"


BINARY_FLOAT_OPS = (AddfOp, SubfOp, MulfOp, DivfOp)

Arith = Dialect("arith", [ConstantOp, AddfOp, SubfOp, MulfOp, DivfOp, MaximumfOp, MinimumfOp,
                          NegfOp, CmpfOp, SelectOp])
Math = Dialect("math", [AbsFOp, SqrtOp])

__all__ = [
    "ConstantOp", "AddfOp", "SubfOp", "MulfOp", "DivfOp", "MaximumfOp", "MinimumfOp", "NegfOp",
    "CmpfOp", "SelectOp", "AbsFOp", "SqrtOp", "CMPF_PREDICATES", "BINARY_FLOAT_OPS", "Arith",
    "Math",
]
