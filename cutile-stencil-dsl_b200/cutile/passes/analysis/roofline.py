"""Roofline analysis (reference: cutile/passes/analysis/roofline.py:35-135).

Per ``stencil.apply``: ``flops`` (add/sub/mul/div/max/min/select/abs count
1; negation and constants are free; ``sqrt`` counts 1), ``unique_loads``
(distinct access offsets, deduplicated by offset tuple alone as in the
reference), ``arithmetic_intensity = flops / ((unique_loads + 1) * bytes)``
and ``bound`` (``"compute"`` at or above 10 flop/byte, else ``"memory"``).

This per-access intensity is the reference's classification; the bench's
roofline instead counts one read per input field and one write per output
field per point (the engine stages each field once per tile).
"""

from __future__ import annotations

from dataclasses import dataclass

from cutile.dialects import arith as A
from cutile.dialects.stencil import AccessOp, ApplyOp
from cutile.ir.core import Context, FloatAttr, IntAttr, ModuleOp, ModulePass, StringAttr, f64

_COMPUTE_BOUND_THRESHOLD = 10.0
_DTYPE_BYTES = {"float64": 8, "float32": 4, "f64": 8, "f32": 4}
_COUNTED = (A.AddfOp, A.SubfOp, A.MulfOp, A.DivfOp, A.MaximumfOp, A.MinimumfOp, A.SelectOp,
            A.AbsFOp, A.SqrtOp)


@dataclass(frozen=True)
class RooflinePass(ModulePass):
    name = "roofline-analysis"

    def apply(self, ctx: Context, op: ModuleOp) -> None:
        for apply_op in [o for o in op.walk() if isinstance(o, ApplyOp)]:
            self._analyze_apply(apply_op)

    @staticmethod
    def _analyze_apply(apply_op: ApplyOp) -> None:
        flops = 0
        offsets: set[tuple[int, ...]] = set()
        for child in apply_op.region.walk():
            if isinstance(child, _COUNTED):
                flops += 1
            if isinstance(child, AccessOp):
                offsets.add(tuple(child.offset))
        loads = len(offsets)
        dtype_bytes = _infer_dtype_bytes(apply_op)
        traffic = (loads + 1) * dtype_bytes
        ai = flops / traffic if traffic > 0 else 0.0
        apply_op.attributes["flops"] = IntAttr(flops)
        apply_op.attributes["unique_loads"] = IntAttr(loads)
        apply_op.attributes["arithmetic_intensity"] = FloatAttr(ai, f64)
        apply_op.attributes["bound"] = StringAttr(
            "compute" if ai >= _COMPUTE_BOUND_THRESHOLD else "memory")


def _infer_dtype_bytes(apply_op: ApplyOp) -> int:
    if apply_op.results:
        elem = getattr(apply_op.results[0].type, "element_type", None)
        if elem is not None and elem.name in _DTYPE_BYTES:
            return _DTYPE_BYTES[elem.name]
    dt = apply_op.attributes.get("dtype")
    if dt is not None:
        return _DTYPE_BYTES.get(dt.data, 8)
    return 8
