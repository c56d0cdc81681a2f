"""Lowering: Dialect 1 -> Dialect 3 -> CUDA C++ (+ Python launcher module)."""

from cutile.lowering.emitter import CodeEmitter
from cutile.lowering.stencil_to_target import lower_fused_to_target_ir, lower_to_target_ir
from cutile.lowering.target_to_cuda import emit_cuda

__all__ = ["lower_to_target_ir", "lower_fused_to_target_ir", "emit_cuda", "CodeEmitter"]
