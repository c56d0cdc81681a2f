"""Fusion-group metadata (reference: cutile/passes/fusion.py:29-138).

All applies inside one ``func.func`` share a domain and land in one group
(the reference's union-find always ends there); ``fusion_outputs`` counts
the group's results.  Actual multi-output fusion is ``compile_fused``.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import ClassVar

from cutile.dialects.stencil import ApplyOp, StdFuncOp
from cutile.ir.core import Context, IntAttr, ModuleOp, ModulePass


@dataclass(frozen=True)
class FusionPass(ModulePass):
    name: ClassVar[str] = "stencil-fusion"

    def apply(self, ctx: Context, op: ModuleOp) -> None:
        for child in op.walk():
            if isinstance(child, StdFuncOp):
                applies = [o for o in child.walk() if isinstance(o, ApplyOp)]
                outputs = sum(len(a.results) for a in applies)
                for a in applies:
                    a.attributes["fusion_group"] = IntAttr(0)
                    a.attributes["fusion_outputs"] = IntAttr(outputs)
