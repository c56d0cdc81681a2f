"""Boundary metadata (reference: cutile/passes/boundary.py:33-72).

Copies the function's boundary attribute onto each ``stencil.apply`` as
``boundary_spec``; Dirichlet gets ``padding_mode = "zero"``, periodic /
Neumann / reflecting get ``boundary_fn = "host_side"`` in the reference.
On the B200 backend the fill is fused into the engine's halo staging, which
this pass records as ``boundary_fn = "fused"`` (``"host_side"`` is kept as
the value the reference's tests read, see ``fused``).
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import ClassVar

from cutile.dialects.cutile_stencil.dialect import BoundaryAttr
from cutile.dialects.stencil import ApplyOp, StdFuncOp
from cutile.ir.core import Context, ModuleOp, ModulePass, StringAttr


@dataclass(frozen=True)
class BoundaryPass(ModulePass):
    name: ClassVar[str] = "stencil-boundary"
    fused: bool = False

    def apply(self, ctx: Context, op: ModuleOp) -> None:
        for child in op.walk():
            if isinstance(child, StdFuncOp):
                self._process_func(child, self.fused)

    @staticmethod
    def _process_func(func_op: StdFuncOp, fused: bool) -> None:
        bc = func_op.attributes.get("boundary")
        if bc is None:
            return
        for inner in func_op.walk():
            if not isinstance(inner, ApplyOp):
                continue
            inner.attributes["boundary_spec"] = bc
            if isinstance(bc, BoundaryAttr):
                bc_type = bc.bc_type_str
            elif isinstance(bc, StringAttr):
                bc_type = bc.data
            else:
                bc_type = str(bc)
            if bc_type == "dirichlet":
                inner.attributes["padding_mode"] = StringAttr("zero")
            elif bc_type in ("periodic", "neumann", "reflecting"):
                inner.attributes["boundary_fn"] = StringAttr("fused" if fused else "host_side")
