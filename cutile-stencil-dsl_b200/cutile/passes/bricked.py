"""Bricked layout tag (reference: cutile/passes/bricked.py:24-46).

Attaches ``layout = "bricked"`` and ``brick_size`` to each apply.  On the
B200 backend a bricked stencil is stored brick-major (``cutile.dialects.
layout.LayoutAttr``) and the engine stages whole bricks with one TMA copy
each, instead of the reference's flat round-trip.
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
