"""Textual form of the IR (MLIR generic syntax with per-op custom forms).

Mirrors what ``str(module)`` shows in the reference (an xDSL printout): op
names such as ``cutile_stencil.access`` / ``stencil.apply`` / ``arith.addf``,
properties in ``<{...}>`` and attributes in ``{...}``.
"""

from __future__ import annotations

from cutile.ir.core import Block, Operation, Region, SSAValue


class Printer:
    def __init__(self):
        self._names: dict[int, str] = {}
        self._counter = 0
        self._lines: list[str] = []

    # -- value naming --------------------------------------------------------
    def value_name(self, v: SSAValue) -> str:
        key = id(v)
        if key not in self._names:
            self._names[key] = f"%{self._counter}"
            self._counter += 1
        return self._names[key]

    def print_operand(self, v: SSAValue) -> str:
        return self.value_name(v)

    # -- ops -------------------------------------------------------------------
    def print_op_to_string(self, op: Operation) -> str:
        self._lines = []
        self._print_op(op, 0)
        return "\n".join(self._lines)

    def _print_op(self, op: Operation, indent: int) -> None:
        pad = "  " * indent
        results = ""
        if op.results:
            results = ", ".join(self.value_name(r) for r in op.results) + " = "
        custom = op.print_custom(self)
        if custom is not None:
            self._lines.append(f"{pad}{results}{op.name}{custom}")
            for r in op.regions:
                self._print_region(r, indent)
            return
        operands = ", ".join(self.value_name(o) for o in op.operands)
        text = f'{pad}{results}"{op.name}"({operands})'
        if op.properties:
            text += " <{" + ", ".join(f"{k} = {v.print()}" for k, v in op.properties.items()) + "}>"
        if op.regions:
            self._lines.append(text + " (")
            for k, r in enumerate(op.regions):
                self._print_region(r, indent, bare=True)
                if k + 1 < len(op.regions):
                    self._lines.append(pad + "}, {")
            tail = ")"
        else:
            tail = ""
        attr_text = ""
        if op.attributes:
            attr_text = " {" + ", ".join(f'"{k}" = {v.print()}' for k, v in op.attributes.items()) + "}"
        sig = " : (" + ", ".join(o.type.print() for o in op.operands) + ") -> (" + ", ".join(
            r.type.print() for r in op.results) + ")"
        if op.regions:
            self._lines.append(pad + tail + attr_text + sig)
        else:
            self._lines.append(text + attr_text + sig)

    def _print_region(self, region: Region, indent: int, bare: bool = False) -> None:
        pad = "  " * indent
        if not bare:
            self._lines[-1] += " {"
        else:
            self._lines.append(pad + "{")
        for b in region.blocks:
            self._print_block(b, indent + 1)
        self._lines.append(pad + "}")

    def _print_block(self, block: Block, indent: int) -> None:
        pad = "  " * (indent - 1)
        if block.args:
            args = ", ".join(f"{self.value_name(a)} : {a.type.print()}" for a in block.args)
            self._lines.append(f"{pad}^bb0({args}):")
        for op in block.ops:
            self._print_op(op, indent)


def print_module(op: Operation) -> str:
    return Printer().print_op_to_string(op)
