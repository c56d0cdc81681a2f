"""``layout`` dialect: row-major vs bricked storage (reference:
cutile/dialects/layout/dialect.py:25-65).

In the reference only tests construct these.  Here ``LayoutAttr`` has a
concrete meaning the engine and the conversion kernels share: a bricked
array of logical shape ``(N0, N1, N2)`` and brick side ``b`` is stored as
``(ceil(N0/b), ceil(N1/b), ceil(N2/b), b, b, b)`` C-contiguous (brick indices
first, then the offsets inside a brick; 2-D analogously), the order the
reference's ``to_bricks`` produces (multigpu_emitter.py:370-404).
``AddressOp`` computes that linear offset.
"""

from __future__ import annotations

from cutile.dialects._base import BuildMixin, Dialect, prop
from cutile.ir.core import Attribute, IntAttr, Operation, StringAttr


class LayoutAttr(Attribute):
    name = "layout.type"

    def __init__(self, kind: str | StringAttr, brick_size: int | IntAttr | None = None):
        self.kind = kind if isinstance(kind, StringAttr) else StringAttr(kind)
        if brick_size is not None and not isinstance(brick_size, IntAttr):
            brick_size = IntAttr(brick_size)
        self.brick_size = brick_size

    def _key(self):
        return (self.kind.data, None if self.brick_size is None else self.brick_size.data)

    def print(self) -> str:
        b = "none" if self.brick_size is None else str(self.brick_size.data)
        return f"#layout.type<{self.kind.data}, {b}>"

    def linear_offset(self, shape, index) -> int:
        """Element offset of logical *index* in an array of logical *shape*."""
        if self.kind.data != "bricked":
            off = 0
            for n, i in zip(shape, index):
                off = off * n + i
            return off
        b = self.brick_size.data
        nb = [-(-n // b) for n in shape]
        off = 0
        for n, i in zip(nb, index):
            off = off * n + i // b
        for i in index:
            off = off * b + i % b
        return off


class CastOp(BuildMixin, Operation):
    name = "layout.cast"
    from_layout = prop()
    to_layout = prop()


class AddressOp(BuildMixin, Operation):
    name = "layout.address"
    layout = prop()


LayoutDialect = Dialect("layout", [CastOp, AddressOp], [LayoutAttr])

__all__ = ["LayoutAttr", "CastOp", "AddressOp", "LayoutDialect"]
