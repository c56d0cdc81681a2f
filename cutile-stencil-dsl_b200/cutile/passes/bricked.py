"""Bricked layout tag (reference: cutile/passes/bricked.py:24-46).

Attaches ``layout = "bricked"`` and ``brick_size`` to each apply (the
attributes the reference's pass writes).  ``compile(layout="bricked")``
itself passes the layout to the lowering directly: on the B200 backend the
fields can stay resident brick-major (``cutile.dialects.layout.LayoutAttr``)
and the engine's bricked instantiation addresses bricks when it stages
chunks, stores outputs and patches boundaries, instead of the reference's
flat round-trip around a flat kernel.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import ClassVar

from cutile.dialects.stencil import ApplyOp
from cutile.ir.core import Context, IntAttr, ModuleOp, ModulePass, StringAttr


@dataclass(frozen=True)
class BrickedLayoutPass(ModulePass):
    name: ClassVar[str] = "bricked-layout"
    brick_size: int = 32

    def apply(self, ctx: Context, op: ModuleOp) -> None:
        for child in op.walk():
            if isinstance(child, ApplyOp):
                child.attributes["layout"] = StringAttr("bricked")
                child.attributes["brick_size"] = IntAttr(self.brick_size)
