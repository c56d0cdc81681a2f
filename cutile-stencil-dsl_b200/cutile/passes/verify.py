"""IR verification (reference: cutile/passes/verify.py:31-103), extended with
the B200 engine's constraints.

Checks: ``tile_sizes`` are powers of two and come with ``halo_widths``;
``temporal_steps >= 1``; ``num_gpus >= 1``; and for an attached engine tile,
that the TMA box (tile + 2 * radius, padded to 16 bytes) stays within the
256-element box limit per dimension.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import ClassVar

from cutile.dialects.stencil import ApplyOp
from cutile.ir.core import Context, FileLineColLoc, ModuleOp, ModulePass


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

    def _verify_apply(self, apply_op: ApplyOp) -> None:
        attrs = apply_op.attributes
        tile_attr = attrs.get("tile_sizes")
        if tile_attr is not None:
            for idx, ts in enumerate(tile_attr):
                if not self._is_power_of_2(ts.data):
                    raise ValueError(_format_diagnostic(
                        apply_op, f"verify-ir: tile_sizes[{idx}] = {ts.data} is not a power of 2 "
                                  f"(tile constraint)"))
            if attrs.get("halo_widths") is None:
                raise ValueError(_format_diagnostic(
                    apply_op, "verify-ir: tile_sizes is set but halo_widths is missing "
                              "(AnalysisPass must run before TilingPass)"))
        t = attrs.get("temporal_steps")
        if t is not None and t.data < 1:
            raise ValueError(_format_diagnostic(
                apply_op, f"verify-ir: temporal_steps = {t.data} must be >= 1"))
        g = attrs.get("num_gpus")
        if g is not None and g.data < 1:
            raise ValueError(_format_diagnostic(
                apply_op, f"verify-ir: num_gpus = {g.data} must be >= 1"))
        et = attrs.get("engine_tile")
        halo = attrs.get("halo_widths")
        if et is not None and halo is not None:
            tile = [a.data for a in et]
            radius = [a.data for a in halo]
            inner = tile[-1] + 2 * radius[-1] + 4
            if inner > 256:
                raise ValueError(_format_diagnostic(
                    apply_op, f"verify-ir: engine tile row {tile[-1]} + halo exceeds the "
                              f"256-element TMA box"))
            if len(tile) == 3 and tile[1] + 2 * radius[1] > 256:
                raise ValueError(_format_diagnostic(
                    apply_op, "verify-ir: engine tile height + halo exceeds the TMA box"))
