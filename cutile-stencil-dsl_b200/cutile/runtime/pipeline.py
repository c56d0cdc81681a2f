"""Composable pass pipeline (reference: cutile/runtime/pipeline.py:17-65)."""

from __future__ import annotations

from dataclasses import dataclass, field

from cutile.ir.core import Context, ModuleOp, ModulePass


@dataclass
class Pipeline:
    """An ordered list of passes; ``run`` applies them to a module."""

    passes: list[ModulePass] = field(default_factory=list)

    def add(self, pass_: ModulePass) -> "Pipeline":
        self.passes.append(pass_)
        return self

    def run(self, module: ModuleOp) -> ModuleOp:
        ctx = Context()
        for p in self.passes:
            p.apply(ctx, module)
        return module

    @classmethod
    def single_gpu(cls, shared_mem_bytes: int = 49152, dtype_bytes: int = 8,
                   max_temporal_steps: int = 8) -> "Pipeline":
        """normalize -> analysis -> roofline -> tiling -> boundary -> temporal.

        The defaults are the reference's (49152-byte budget), which fix the
        default temporal depth ``compile()`` reports and each launch advances.
        """
        from cutile.passes.analysis.footprint import AnalysisPass
        from cutile.passes.analysis.roofline import RooflinePass
        from cutile.passes.boundary import BoundaryPass
        from cutile.passes.normalize import NormalizePass
        from cutile.passes.temporal import TemporalBlockingPass
        from cutile.passes.tiling import TilingPass

        p = cls()
        p.add(NormalizePass())
        p.add(AnalysisPass())
        p.add(RooflinePass())
        p.add(TilingPass(shared_mem_bytes=shared_mem_bytes, dtype_bytes=dtype_bytes))
        p.add(BoundaryPass())
        p.add(TemporalBlockingPass(max_steps=max_temporal_steps, shared_mem_bytes=shared_mem_bytes,
                                   dtype_bytes=dtype_bytes))
        return p
