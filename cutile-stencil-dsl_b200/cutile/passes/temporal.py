"""Temporal blocking depth (reference: cutile/passes/temporal.py:28-81).

The depth ``T`` is the largest ``t <= max_steps`` whose halo-expanded tile
``prod(tile + 2*t*halo) * dtype_bytes * 2`` fits ``shared_mem_bytes``
(``T = 1`` when none does).  The formula, its inputs (the reference row
tiles from ``TilingPass``) and the default 49152-byte budget are kept as is,
because ``T`` is observable: one ``launch_<name>`` call advances ``T`` steps.

How the steps run is the engine's business: the reference issues ``T``
launches through scratch buffers; the B200 engine chains the ``T`` steps
inside one pass over each tile, in shared memory (time skewing), with the
same result (intermediate steps see zero halos).
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from typing import ClassVar

from cutile.dialects.stencil import ApplyOp
from cutile.ir.core import ArrayAttr, Context, IntAttr, ModuleOp, ModulePass


@dataclass(frozen=True)
class TemporalBlockingPass(ModulePass):
    name: ClassVar[str] = "temporal-blocking"

    max_steps: int = 8
    shared_mem_bytes: int = 49152
    dtype_bytes: int = 8

    def apply(self, ctx: Context, op: ModuleOp) -> None:
        for child in op.walk():
            if isinstance(child, ApplyOp):
                self._process_apply(child)

    def depth(self, tile, halo) -> int:
        for t in range(self.max_steps, 1, -1):
            expanded = [tile[d] + 2 * t * halo[d] for d in range(len(tile))]
            if math.prod(expanded) * self.dtype_bytes * 2 <= self.shared_mem_bytes:
                return t
        return 1

    def _process_apply(self, apply_op: ApplyOp) -> None:
        tile_attr = apply_op.attributes.get("tile_sizes")
        halo_attr = apply_op.attributes.get("halo_widths")
        if tile_attr is None or halo_attr is None:
            return
        tile = [a.data for a in tile_attr]
        halo = [a.data for a in halo_attr]
        best_t = self.depth(tile, halo)
        apply_op.attributes["temporal_steps"] = IntAttr(best_t)
        apply_op.attributes["expanded_halo"] = ArrayAttr([IntAttr(best_t * h) for h in halo])
        apply_op.attributes["temporal_buffer_count"] = IntAttr(best_t + 1)
