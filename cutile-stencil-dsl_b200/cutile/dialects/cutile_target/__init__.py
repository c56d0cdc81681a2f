"""Dialect 3 (``cutile``): device kernel and host orchestration IR.

Same op set as the reference (cutile/dialects/cutile_target/dialect.py:31-307):
device ops ``kernel/slice/load/store/bid/return`` and host ops
``host_program/alloc/launch/sync/swap_buffers/for_loop/for_each_gpu/async/
boundary_apply/layout_cast``.

What changes is what ``KernelOp`` carries.  The reference stores a Python
expression string for cuTile; here the op also carries what the B200 engine
template needs: the field dtype, the per-dimension stencil radius, the engine
tile (rows per step, tile rows, tile columns, points per thread, threads),
the temporal depth, the layout and brick size, the boundary mode, the
distinct accesses, and the body as a list of SSA statements (``ssa_body``)
that the CUDA emitter turns into a device functor without re-parsing.
"""

from __future__ import annotations

from cutile.dialects._base import BuildMixin, Dialect, prop
from cutile.ir.core import Operation, Region


class KernelOp(BuildMixin, Operation):
    name = "cutile.kernel"
    kernel_name = prop()
    tile_shape = prop()
    halo = prop()
    ndim = prop()
    input_names = prop()
    expression = prop()
    constants = prop()
    grid_order = prop()
    kernel_constants = prop()
    kernel_hints = prop()
    expressions = prop()
    output_names = prop()
    # -- B200 engine properties ------------------------------------------
    dtype = prop()
    radius = prop()
    accesses = prop()
    ssa_body = prop()
    engine = prop()
    temporal_steps = prop()
    layout = prop()
    brick_size = prop()
    boundary_mode = prop()
    scalar_count = prop()
    dyn_count = prop()
    reduce_max = prop()


class SliceOp(BuildMixin, Operation):
    name = "cutile.slice"
    axis = prop()
    start = prop()
    stop = prop()
    var_name = prop()

    @property
    def input(self):
        return self.operands[0]


class LoadOp(BuildMixin, Operation):
    name = "cutile.load"
    view_name = prop()

    @property
    def tensor(self):
        return self.operands[0]


class StoreOp(BuildMixin, Operation):
    name = "cutile.store"

    @property
    def tile(self):
        return self.operands[0]

    @property
    def value(self):
        return self.operands[1]


class BidOp(BuildMixin, Operation):
    name = "cutile.bid"
    axis = prop()


class ReturnOp(BuildMixin, Operation):
    name = "cutile.return"


class HostProgramOp(BuildMixin, Operation):
    name = "cutile.host_program"
    program_name = prop()
    preamble = prop()


class AllocOp(BuildMixin, Operation):
    name = "cutile.alloc"
    var_name = prop()
    dtype = prop()


class LaunchOp(BuildMixin, Operation):
    name = "cutile.launch"
    kernel_name = prop()
    grid_expr = prop()
    args_expr = prop()


class SyncOp(BuildMixin, Operation):
    name = "cutile.sync"


class SwapBuffersOp(BuildMixin, Operation):
    name = "cutile.swap_buffers"


class ForLoopOp(BuildMixin, Operation):
    name = "cutile.for_loop"
    count = prop()


class ForEachGpuOp(BuildMixin, Operation):
    name = "cutile.for_each_gpu"
    num_gpus = prop()


class AsyncOp(BuildMixin, Operation):
    name = "cutile.async"


class BoundaryApplyOp(BuildMixin, Operation):
    name = "cutile.boundary_apply"
    bc_type = prop()


class LayoutCastOp(BuildMixin, Operation):
    name = "cutile.layout_cast"
    from_layout = prop()
    to_layout = prop()


CutileTargetDialect = Dialect("cutile", [
    KernelOp, SliceOp, LoadOp, StoreOp, BidOp, ReturnOp, HostProgramOp, AllocOp, LaunchOp,
    SyncOp, SwapBuffersOp, ForLoopOp, ForEachGpuOp, AsyncOp, BoundaryApplyOp, LayoutCastOp,
])

__all__ = [
    "CutileTargetDialect", "KernelOp", "SliceOp", "LoadOp", "StoreOp", "BidOp", "ReturnOp",
    "HostProgramOp", "AllocOp", "LaunchOp", "SyncOp", "SwapBuffersOp", "ForLoopOp",
    "ForEachGpuOp", "AsyncOp", "BoundaryApplyOp", "LayoutCastOp", "Region",
]
