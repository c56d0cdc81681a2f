"""Runge-Kutta time integration with the stage combination fused on device.

Reference: cutile/runtime/rk_integrator.py:54-232.  There, ``RKIntegrator``
wraps a compiled stencil ``L`` and emits Python that runs ``launch_fn(u, k)``
per stage and combines stages with CuPy element-wise kernels, allocating a
``zeros_like`` per stage.  Here each stage is ONE engine kernel generated
from ``L``: it evaluates ``L`` on the stage state and, in the same pass,
forms

    next = a * base + b * stage + (c * dt) * L(stage)     (FP64, one rounding)
    acc  = acc + (w * dt) * L(stage)                       (RK4 only)

with ``dt`` a per-grid device scalar, so no intermediate derivative field is
written and fields may be stored in FP32 while the combination runs in FP64.
Methods (same names as the reference):

* ``euler``:  u1 = u + dt L(u)
* ``rk2``:    midpoint, u1 = u + dt/2 L(u);  u = u + dt L(u1)
* ``rk4``:    classic; s_k = u + c_k dt L(s_{k-1}); acc accumulates
              u + dt/6 L(u) + dt/3 L(s1) + dt/3 L(s2); u = acc + dt/6 L(s3)
* ``ssprk3``: Shu-Osher; u1 = u + dt L(u); u2 = 3/4 u + 1/4 u1 + 1/4 dt L(u1);
              u = 1/3 u + 2/3 u2 + 2/3 dt L(u2)

Operators may return a tuple (one derivative per state field: the first
arrays of the stencil, in order).
"""

from __future__ import annotations

import importlib.util
import tempfile
from dataclasses import dataclass, field
from typing import Any

# Stage tables: (a, b, c, w, base, stage, acc_in, out)
#   base/stage/acc_in/out name buffers: "u" (state), "s1".."s3" (workspace), "acc"
_METHODS = {
    "euler": [(1.0, 0.0, 1.0, None, "u", "u", None, "s1")],
    "rk2": [(1.0, 0.0, 0.5, None, "u", "u", None, "s1"),
            (1.0, 0.0, 1.0, None, "u", "s1", None, "u")],
    "rk4": [(1.0, 0.0, 0.5, 1.0 / 6.0, "u", "u", "u", "s1"),
            (1.0, 0.0, 0.5, 1.0 / 3.0, "u", "s1", "acc", "s2"),
            (1.0, 0.0, 1.0, 1.0 / 3.0, "u", "s2", "acc", "s3"),
            (1.0, 0.0, 1.0 / 6.0, None, "acc", "s3", None, "u")],
    "ssprk3": [(1.0, 0.0, 1.0, None, "u", "u", None, "s1"),
               (0.75, 0.25, 0.25, None, "u", "s1", None, "s2"),
               (1.0 / 3.0, 2.0 / 3.0, 2.0 / 3.0, None, "u", "s2", None, "u")],
}


def stage_table(method: str):
    return _METHODS[method]


@dataclass
class RKCompileResult:
    """Stage kernels of one method (rk_integrator.py:22-46)."""

    stencil_result: Any
    method: str
    num_stages: int
    code: str
    cuda_source: str = ""
    info: dict = field(default_factory=dict)
    _module: Any = field(default=None, repr=False)

    def emit_to_file(self, path: str) -> None:
        with open(path, "w") as f:
            f.write(self.code)

    def load_module(self):
        if self._module is not None:
            return self._module
        with tempfile.NamedTemporaryFile(suffix=".py", delete=False, mode="w") as f:
            f.write(self.code)
            path = f.name
        spec = importlib.util.spec_from_file_location("_rk", path)
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        self._module = mod
        return mod


class RKIntegrator:
    """Runge-Kutta stepping of a stencil operator (rk_integrator.py:54-117)."""

    _STAGES = {"euler": 1, "rk2": 2, "rk4": 4, "ssprk3": 3}

    def __init__(self, stencil_fn, method: str = "rk4"):
        self.stencil_fn = stencil_fn
        self.method = method.lower()
        if self.method not in self._STAGES:
            raise ValueError(f"Unknown RK method {method!r}. Supported: {', '.join(self._STAGES)}")

    def compile(self, domain=None, hw=None, *, precision: str | None = None,
                boundary=None, align_halo: bool = True, tile_sizes=None,
                kernel_hints=None) -> RKCompileResult:
        """Stage kernels for the method; ``boundary`` (a kind) is fused into
        every stage's staging of the stage state."""
        from cutile.runtime.launcher import build_variants

        variants = {}
        name = self.stencil_fn._fn.__name__
        for k, (a, b, c, w, base, stage, _acc, _out) in enumerate(_METHODS[self.method]):
            opts = {"rk": {"a": a, "b": b, "c": c, "w": w, "same_base": base == stage}}
            if boundary is not None:
                opts["boundary_mode"] = boundary if isinstance(boundary, str) else boundary["type"]
            variants[f"{name}_{self.method}_s{k}"] = opts
        cuda, info = build_variants(self.stencil_fn, variants, precision=precision,
                                    align_halo=align_halo, tile_sizes=tile_sizes,
                                    kernel_hints=kernel_hints, boundary=boundary)
        info["method"] = self.method
        info["stages"] = list(variants)
        info["ndim"] = len(info["halo"])
        from cutile.runtime.launcher import _yields

        info["state_fields"] = _yields(self.stencil_fn._ir)
        from cutile.runtime.launcher import _num_inputs

        info["fields"] = _num_inputs(self.stencil_fn._ir)
        code = _module_code(name, self.method, cuda, info)
        return RKCompileResult(stencil_result=None, method=self.method,
                               num_stages=self._STAGES[self.method], code=code, cuda_source=cuda,
                               info=info)


def _module_code(name: str, method: str, cuda: str, info: dict) -> str:
    from cutile.lowering.emitter import CodeEmitter

    spec = {k: v for k, v in info.items() if k != "kernels" and k != "analysis"}
    spec["kernels"] = {k: {"inputs": v["inputs"], "outputs": v["outputs"]}
                       for k, v in info["kernels"].items()}
    spec["halo"] = list(info["halo"])
    spec["stencil_halo"] = list(info["stencil_halo"])
    spec["name"] = name
    e = CodeEmitter()
    e.line(f'"""{method.upper()} stepping of {name} with fused FP64 stage combination (generated)."""')
    e.blank()
    e.line("from cutile.runtime.rk_runtime import RKProgram")
    e.blank()
    e.line("CUDA_SOURCE = r'''" + cuda + "'''")
    e.line(f"SPEC = {spec!r}")
    e.line("_PROGRAM = RKProgram(CUDA_SOURCE, SPEC)")
    e.blank()
    e.blank()
    e.line(f"def rk_{method}_step(u, dt, stream=None, **scalars):")
    with e.indent():
        e.line('"""Advance the state ``u`` (a field or a tuple of fields) one step, in place."""')
        e.line("_PROGRAM.step(u, dt, stream, scalars)")
        e.line("return u")
    e.blank()
    e.blank()
    e.line(f"def rk_{method}_solve(u0, dt, num_steps, stream=None, **scalars):")
    with e.indent():
        e.line(f'"""Run {method.upper()} for ``num_steps`` steps from a copy of ``u0``."""')
        e.line("u = _PROGRAM.copy_state(u0)")
        e.line("for _ in range(num_steps):")
        with e.indent():
            e.line("_PROGRAM.step(u, dt, stream, scalars)")
        e.line("return u")
    e.blank()
    e.blank()
    e.line("def program():")
    with e.indent():
        e.line("return _PROGRAM")
    return e.render()


__all__ = ["RKIntegrator", "RKCompileResult", "stage_table"]
