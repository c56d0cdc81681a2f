"""Footprint analysis: per-dimension halo widths (reference:
cutile/passes/analysis/footprint.py:21-64).

``halo_widths[d] = max |offset[d]|`` over every ``stencil.access`` of an
apply.  On the B200 engine these widths are the per-dimension stencil radius:
they size the TMA box (tile + 2 * radius) and the shared-memory ring.
"""

from __future__ import annotations

from dataclasses import dataclass

from cutile.dialects.stencil import AccessOp, ApplyOp
from cutile.ir.core import ArrayAttr, Context, IntAttr, ModuleOp, ModulePass


@dataclass(frozen=True)
class AnalysisPass(ModulePass):
    name = "stencil-analysis"

    def apply(self, ctx: Context, op: ModuleOp) -> None:
        for apply_op in [o for o in op.walk() if isinstance(o, ApplyOp)]:
            self._analyze_apply(apply_op)

    @staticmethod
    def _analyze_apply(apply_op: ApplyOp) -> None:
        ndim = None
        widths: list[int] = []
        for inner in apply_op.walk():
            if not isinstance(inner, AccessOp):
                continue
            offsets = list(inner.offset)
            if ndim is None:
                ndim = len(offsets)
                widths = [0] * ndim
            for d, off in enumerate(offsets):
                if d < len(widths):
                    widths[d] = max(widths[d], abs(off))
        if ndim is None:
            return
        apply_op.attributes["halo_widths"] = ArrayAttr([IntAttr(w) for w in widths])
