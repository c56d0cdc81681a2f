"""IR verification (reference: cutile/passes/verify.py:31-103), extended with
the B200 engine's constraints.

The reference's checks: ``tile_sizes`` are powers of two and come with
``halo_widths``; ``temporal_steps >= 1``; ``num_gpus >= 1``.

The engine's checks, on the plan :func:`attach_engine_plan` records on each
``stencil.apply`` before lowering (``compile``, ``compile_fused`` and the RK
stage builds run it):

* every TMA box dimension (staged row width, staged tile height with halo,
  rows per chunk) is at most 256 elements (``cuTensorMapEncodeTiled``);
* the staged row width in bytes is a multiple of 16 (a TMA box's inner
  extent, and the 16-byte ``ld.shared`` strips the body reads);
* the tile row is a whole number of per-thread vectors, and the tile height
  a whole number of rows per thread;
* the dynamic shared memory of one block fits the 227 KB a B200 CTA may use;
* the block size is a whole number of warps, at most 1024 threads.

The 16-byte rule on global row pitches depends on the arrays, not the
kernel; the launch checks it and stages through the cp.async loader when a
pitch is not 16-byte aligned.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import ClassVar

from cutile.dialects.stencil import ApplyOp
from cutile.ir.core import ArrayAttr, Context, FileLineColLoc, IntAttr, ModuleOp, ModulePass

TMA_BOX_MAX = 256
SMEM_PER_BLOCK = 227 * 1024


def _format_diagnostic(op, message: str) -> str:
    loc = getattr(op, "location", None)
    if isinstance(loc, FileLineColLoc):
        return f"{loc.filename.data}:{loc.line.data} -- {message}"
    return message


@dataclass(frozen=True)
class VerifyPass(ModulePass):
    name: ClassVar[str] = "verify-ir"

    def apply(self, ctx: Context, op: ModuleOp) -> None:
        for child in op.walk():
            if isinstance(child, ApplyOp):
                self._verify_apply(child)

    @staticmethod
    def _is_power_of_2(n: int) -> bool:
        return n > 0 and (n & (n - 1)) == 0

    def _fail(self, op, msg: str):
        raise ValueError(_format_diagnostic(op, f"verify-ir: {msg}"))

    def _verify_apply(self, apply_op: ApplyOp) -> None:
        attrs = apply_op.attributes
        tile_attr = attrs.get("tile_sizes")
        if tile_attr is not None:
            for idx, ts in enumerate(tile_attr):
                if not self._is_power_of_2(ts.data):
                    self._fail(apply_op, f"tile_sizes[{idx}] = {ts.data} is not a power of 2 "
                                         f"(tile constraint)")
            if attrs.get("halo_widths") is None:
                self._fail(apply_op, "tile_sizes is set but halo_widths is missing "
                                     "(AnalysisPass must run before TilingPass)")
        t = attrs.get("temporal_steps")
        if t is not None and t.data < 1:
            self._fail(apply_op, f"temporal_steps = {t.data} must be >= 1")
        g = attrs.get("num_gpus")
        if g is not None and g.data < 1:
            self._fail(apply_op, f"num_gpus = {g.data} must be >= 1")
        if "engine_box" in attrs:
            self._verify_engine(apply_op, attrs)

    def _verify_engine(self, op, attrs) -> None:
        box_w, box_h, rows = (a.data for a in attrs["engine_box"])
        tile = [a.data for a in attrs["engine_tile"]]
        vec = attrs["engine_vec"].data
        rpy = attrs["engine_rpy"].data
        esz = attrs["engine_dtype_bytes"].data
        smem = attrs["engine_smem"].data
        threads = attrs["engine_threads"].data
        for what, n in (("row width", box_w), ("tile height with halo", box_h),
                        ("rows per chunk", rows)):
            if not 1 <= n <= TMA_BOX_MAX:
                self._fail(op, f"engine TMA box {what} = {n} is outside 1..{TMA_BOX_MAX}")
        if (box_w * esz) % 16:
            self._fail(op, f"engine TMA box row of {box_w} x {esz} B is not a multiple of 16 bytes")
        if tile[-1] % vec:
            self._fail(op, f"engine tile row {tile[-1]} is not a multiple of the {vec}-point vector")
        if len(tile) == 3 and tile[1] % rpy:
            self._fail(op, f"engine tile height {tile[1]} is not a multiple of {rpy} rows per thread")
        if smem > SMEM_PER_BLOCK:
            self._fail(op, f"engine shared memory {smem} B exceeds the {SMEM_PER_BLOCK} B a "
                           f"B200 block may use")
        if threads % 32 or not 32 <= threads <= 1024:
            self._fail(op, f"engine block of {threads} threads is not 1-32 whole warps")


def attach_engine_plan(module: ModuleOp, plan, geometry: dict, dtype_bytes: int) -> None:
    """Record an engine plan and its derived geometry on every apply."""
    for child in module.walk():
        if isinstance(child, ApplyOp):
            a = child.attributes
            a["engine_tile"] = ArrayAttr([IntAttr(t) for t in plan.tile_sizes()])
            a["engine_box"] = ArrayAttr([IntAttr(geometry["box_w"]), IntAttr(geometry["box_h"]),
                                         IntAttr(plan.rows)])
            a["engine_vec"] = IntAttr(plan.vec)
            a["engine_rpy"] = IntAttr(plan.rpy)
            a["engine_dtype_bytes"] = IntAttr(dtype_bytes)
            a["engine_smem"] = IntAttr(geometry["smem_bytes"])
            a["engine_threads"] = IntAttr(plan.threads)


def verify_engine_plan(module: ModuleOp, plan, radius, dtype_bytes: int, num_inputs: int,
                       periodic: bool = False) -> None:
    """Attach ``plan`` to a clone of the stencil's module and run VerifyPass."""
    from cutile.passes.tiling import engine_geometry, radius3

    g = engine_geometry(plan, radius3(plan.ndim, tuple(radius)), dtype_bytes, num_inputs, periodic)
    attach_engine_plan(module, plan, g, dtype_bytes)
    VerifyPass().apply(Context(), module)
