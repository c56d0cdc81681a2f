"""``compile`` / ``compile_fused`` / ``CompileResult`` -- the drop-in boundary.

Mirrors cutile/runtime/launcher.py of the reference (lines 27-728): same
signatures, same ``CompileResult`` fields and methods, same halo / temporal
semantics.  What the result's ``code`` holds differs: instead of cuTile
Python it is a Python module whose ``launch_<name>`` (and
``apply_boundary_<name>``, ``step_<name>``, bricked helpers) call the B200
engine kernels compiled from ``cuda_source`` through libcsd.

Semantics kept from the reference:

* ``temporal_steps`` comes from the reference's pass pipeline (49152-byte
  budget by default), so ``launch_<name>`` advances the same number of steps
  per call; intermediate steps see zero halos; the input is not modified;
* ``align_halo`` pads the innermost halo to 128 bytes (launcher.py:257-273);
* launch arguments: ``(u_in, u_out)`` for one input, ``(u, v, ..., u_out)``
  for several (input names ``u v w x y z``), fused kernels take the merged
  parameter names then ``<member>_out`` each; only output interiors are
  written.

Extensions: ``temporal_steps=`` forces a depth, ``tile_sizes=`` /
``kernel_hints=`` override the engine plan, ``dtype=`` overrides the
declared dtype.  ``num_gpus > 1`` raises: multi-GPU decomposition is not
part of this backend.
"""

from __future__ import annotations

import importlib.util
import json
import math
import tempfile
from dataclasses import dataclass, field, replace
from typing import Any, Optional

from cutile.dialects.stencil import ApplyOp
from cutile.passes.verify import verify_engine_plan
from cutile.runtime.pipeline import Pipeline


def _import_file(path: str, module_name: str):
    spec = importlib.util.spec_from_file_location(module_name, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def load_aot(module_path: str):
    """Import a launcher module written by ``CompileResult.build_aot``."""
    import hashlib
    import os

    path = os.path.abspath(module_path)
    name = os.path.splitext(os.path.basename(path))[0]
    tag = hashlib.sha256(path.encode()).hexdigest()[:12]
    return _import_file(path, f"_aot_{name}_{tag}")


@dataclass
class AotBuild:
    """Paths of an ahead-of-time build and ptxas' resources per entry."""

    cu: str
    cubin: str
    module: str
    log: str
    resources: dict = field(default_factory=dict)


@dataclass
class CompileResult:
    """Result of compiling a stencil (launcher.py:27-231)."""

    name: str
    code: str
    ndim: int
    halo_widths: tuple[int, ...]
    tile_sizes: tuple[int, ...]
    temporal_steps: int
    analysis: dict = field(default_factory=dict)
    stencil_halo: tuple[int, ...] = field(default=())
    kernel_hints: dict = field(default_factory=dict)
    resources: Any = field(default=None)
    inputs: tuple = ()
    outputs: tuple = ()
    cuda_source: str = ""
    dtype: str = "float64"
    boundary: Optional[dict] = None
    layout: str = "flat"
    brick_size: int = 0
    _ref_fn: Any = field(default=None, repr=False)
    _ref_fns: Any = field(default=None, repr=False)
    _ref_inputs: Any = field(default=None, repr=False)
    _module: Any = field(default=None, repr=False)

    def emit_to_file(self, path: str) -> None:
        """Write the generated launcher module to *path* (its CUDA source is
        embedded; ``emit_cuda_to_file`` writes the ``.cu`` alone)."""
        with open(path, "w") as f:
            f.write(self.code)

    def emit_cuda_to_file(self, path: str) -> None:
        with open(path, "w") as f:
            f.write(self.cuda_source)

    def load_module(self):
        """Load the generated launcher module (cached per result)."""
        if self._module is not None:
            return self._module
        with tempfile.NamedTemporaryFile(suffix=".py", delete=False, mode="w") as f:
            f.write(self.code)
            tmp_path = f.name
        self._module = _import_file(tmp_path, f"_gen_{self.name}")
        return self._module

    def build_aot(self, directory: str, nvcc: str | None = None) -> "AotBuild":
        """Ahead-of-time artefacts in ``directory``: ``<name>.cu`` (the CUDA
        source, compilable on its own with ``-I`` the engine headers),
        ``<name>.cubin`` (nvcc, sm_100a, the NVRTC path's flags) and
        ``<name>.py``, the launcher module that loads that cubin instead of
        compiling at first launch (same ``launch_<name>`` functions as
        ``load_module()``).  Needs nvcc, not a GPU.  Mirrors the reference's
        ``code`` / ``emit_to_file`` artefact (runtime/launcher.py:57-60)."""
        import hashlib
        import os
        import re

        from cutile.runtime import native
        from cutile.runtime.regcheck import parse_ptxas_log

        os.makedirs(directory, exist_ok=True)
        cu = os.path.join(directory, f"{self.name}.cu")
        cubin = os.path.join(directory, f"{self.name}.cubin")
        shim = os.path.join(directory, f"{self.name}.py")
        self.emit_cuda_to_file(cu)
        log = native.aot_compile(cu, cubin, nvcc)
        with open(cubin, "rb") as f:
            digest = hashlib.sha256(f.read()).hexdigest()
        code = self.code
        if code.count(_CUBIN_LINE + "\n") != 1 or code.count(_CUBIN_HASH_LINE + "\n") != 1:
            raise RuntimeError(f"{self.name}: generated module has no cubin slot")
        code = code.replace(_CUBIN_LINE + "\n", "CUBIN = os.path.join(os.path.dirname("
                            f"os.path.abspath(__file__)), {os.path.basename(cubin)!r})\n")
        code = code.replace(_CUBIN_HASH_LINE + "\n", f"CUBIN_SHA256 = {digest!r}\n")
        with open(shim, "w") as f:
            f.write(code)
        entries = re.findall(r"Compiling entry function '([^']+)'", log)
        return AotBuild(cu=cu, cubin=cubin, module=shim, log=log,
                        resources={n: parse_ptxas_log(log, n) for n in entries})

    # -- self checks ---------------------------------------------------------
    def _np_dtype(self):
        import numpy as np

        return np.float32 if self.dtype in ("float32", "fp32") else np.float64

    def validate(self, u_input=None, atol: float = 1e-10) -> bool:
        """Run the kernel once and compare with the stencil function evaluated
        by NumPy on the same data (launcher.py:76-132): ``temporal_steps``
        applications, compared on the interior shrunk by ``T * halo`` (the
        kernel's intermediate steps see zero halos, NumPy's keep the input's)."""
        import numpy as np
        import torch

        if self._ref_fns and (len(self._ref_fns) > 1 or len(self.inputs) > 1):
            return self._validate_multi(atol)
        if self._ref_fn is None:
            raise RuntimeError("No reference function available")
        hw, ndim, T = self.halo_widths, self.ndim, self.temporal_steps
        if u_input is None:
            base = 128 if ndim == 1 else 64
            u_np = np.random.rand(*tuple(base + 2 * T * h for h in hw)).astype(self._np_dtype())
        else:
            u_np = np.asarray(u_input, dtype=self._np_dtype())
        ref = u_np.copy()
        for _ in range(T):
            ref = _numpy_apply(ref, self._ref_fn, ndim, hw)
        launcher = getattr(self.load_module(), f"launch_{self.name}")
        u_gpu = torch.from_numpy(u_np).cuda()
        out = torch.zeros_like(u_gpu)
        launcher(u_gpu, out)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        inner = tuple(slice(T * h, s - T * h) for h, s in zip(hw, u_np.shape))
        max_diff = float(np.max(np.abs(ref[inner] - got[inner])))
        ok = bool(np.allclose(ref[inner], got[inner], atol=atol))
        print(f"Validation: max_diff={max_diff:.2e}, pass={ok}")
        return ok

    def _validate_multi(self, atol: float) -> bool:
        import inspect

        import numpy as np
        import torch

        from cutile.frontend.elementwise import array_aware

        hw = self.halo_widths
        base = 128 if self.ndim == 1 else 64
        shape = tuple(base + 2 * h for h in hw)
        dt = self._np_dtype()
        inputs = {n: (np.random.rand(*shape) + 0.5).astype(dt) for n in self.inputs}
        launcher = getattr(self.load_module(), f"launch_{self.name}")
        gin = [torch.from_numpy(inputs[n]).cuda() for n in self.inputs]
        gout = [torch.zeros(shape, dtype=gin[0].dtype, device="cuda") for _ in self._ref_fns]
        launcher(*gin, *gout)
        torch.cuda.synchronize()
        interior = tuple(slice(h, s - h) for h, s in zip(hw, shape))
        ok = True
        for fn, out in zip(self._ref_fns, gout):
            params = list(inspect.signature(fn).parameters)[: -self.ndim]
            args = [_Views(inputs.get(n, np.zeros(shape, dt)), hw) for n in params]
            ref = array_aware(fn)(*args, *([0] * self.ndim))
            got = out.cpu().numpy()[interior]
            max_diff = float(np.max(np.abs(ref - got)))
            good = bool(np.allclose(ref, got, atol=atol))
            print(f"Validation[{fn.__name__}]: max_diff={max_diff:.2e}, pass={good}")
            ok = ok and good
        return ok

    def benchmark(self, u_input=None, warmup: int = 5, iters: int = 20) -> dict:
        """CUDA-event timing of ``launch_<name>`` (launcher.py:171-231); bytes
        use the real element size."""
        import numpy as np
        import torch

        hw = self.halo_widths
        if u_input is None:
            base = 128 if self.ndim == 1 else 64
            u_np = np.random.rand(*tuple(base + 2 * h for h in hw)).astype(self._np_dtype())
        else:
            u_np = np.asarray(u_input, dtype=self._np_dtype())
        launcher = getattr(self.load_module(), f"launch_{self.name}")
        ins = [torch.from_numpy(u_np).cuda() for _ in range(max(1, len(self.inputs)))]
        outs = [torch.zeros_like(ins[0]) for _ in range(max(1, len(self.outputs) or 1))]
        for _ in range(warmup):
            launcher(*ins, *outs)
        torch.cuda.synchronize()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        for _ in range(iters):
            launcher(*ins, *outs)
        end.record()
        end.synchronize()
        ms = start.elapsed_time(end) / iters
        npts = math.prod(s - 2 * h for h, s in zip(hw, u_np.shape))
        bytes_pt = (len(ins) + len(outs)) * u_np.itemsize
        return {"time_ms": ms, "gpoints_per_s": npts * self.temporal_steps / ms * 1e-6,
                "gbytes_per_s": npts * bytes_pt / ms * 1e-6}


class _Views:
    """Offset subscripts -> shifted interior views (what ``u[i+1, j]`` means
    when a stencil body runs on whole arrays)."""

    def __init__(self, data, halo):
        self._data = data
        self._halo = halo

    def __getitem__(self, key):
        if not isinstance(key, tuple):
            key = (key,)
        sl = tuple(slice(h + k, n - h + k) for k, h, n in zip(key, self._halo, self._data.shape))
        return self._data[sl]


def _numpy_apply(u, fn, ndim, halo):
    from cutile.frontend.elementwise import array_aware

    res = array_aware(fn)(_Views(u, halo), *([0] * ndim))
    out = u.copy()
    out[tuple(slice(h, s - h) for h, s in zip(halo, u.shape))] = res
    return out


# --------------------------------------------------------------------------- #
# compile()
# --------------------------------------------------------------------------- #


def pad_inner_halo(halo_widths: tuple[int, ...], dtype_bytes: int,
                   align_bytes: int = 128) -> tuple[int, ...]:
    """Round the innermost halo up to a multiple of ``align_bytes``
    (launcher.py:257-273): 16 float64 / 32 float32 elements."""
    if not halo_widths:
        return halo_widths
    align = max(1, align_bytes // dtype_bytes)
    inner = -(-halo_widths[-1] // align) * align
    return tuple(halo_widths[:-1]) + (inner,)


def _num_inputs(ir) -> int:
    from cutile.dialects.cutile_stencil.dialect import FuncOp

    for op in ir.body.block.ops:
        if isinstance(op, FuncOp):
            n_scalars = len(op.scalar_names.data) if op.scalar_names is not None else 0
            return len(op.body.blocks[0].args) - n_scalars
    return 1


def _input_names(ir) -> tuple:
    from cutile.lowering.stencil_to_target import _arg_names, _func_and_block

    f, b = _func_and_block(ir)
    return tuple(_arg_names(f, b))


def _precision(precision, dtype):
    """(dtype, kahan) for a ``precision`` request."""
    if precision is None:
        return dtype, False
    if precision == "fp64":
        return "float64", False
    if precision == "fp32":
        return "float32", False
    if precision == "fp32_kahan":
        return "float32", True
    raise ValueError(f"precision must be fp64, fp32 or fp32_kahan, got {precision!r}")


def _plan_from(tile_sizes, kernel_hints, ndim, base_plan):
    from cutile.passes.tiling import EnginePlan

    p = base_plan
    if tile_sizes is not None:
        # a caller's tile keeps one row per thread unless it asks for more
        p = replace(p, rpy=1)
        t = tuple(tile_sizes)
        if ndim == 3:
            p = replace(p, rows=t[0], tile_y=t[1], tile_x=t[2])
        elif ndim == 2:
            p = replace(p, rows=t[0], tile_x=t[1])
        else:
            p = replace(p, tile_x=t[0])
    if kernel_hints:
        kw = {}
        for k in ("threads", "stages", "zchunk", "waves", "vec"):
            if k in kernel_hints:
                kw[k] = int(kernel_hints[k])
        # "rows_per_thread" is the documented hint; "rpy" is the key
        # EnginePlan.hints() writes (autotune results, caches), read back
        # the same way so a tuned plan round-trips through compile()
        for key in ("rpy", "rows_per_thread"):
            if key in kernel_hints:
                kw["rpy"] = int(kernel_hints[key])
        occ = kernel_hints.get("min_blocks", kernel_hints.get("occupancy"))
        if occ is not None:
            kw["occupancy"] = int(occ)
        p = replace(p, **kw)
    assert isinstance(p, EnginePlan)
    return p


# The generated module's program lines.  An ahead-of-time build rewrites the
# two ``None`` lines to name the cubin beside the module and its hash.
_CUBIN_LINE = "CUBIN = None"
_CUBIN_HASH_LINE = "CUBIN_SHA256 = None"


def _program_lines(e) -> None:
    e.line(_CUBIN_LINE)
    e.line(_CUBIN_HASH_LINE)
    e.line("_PROGRAM = StencilProgram(CUDA_SOURCE, SPEC, cubin=CUBIN, cubin_sha256=CUBIN_SHA256)")


def generate_module_code(name: str, cuda_source: str, spec: dict, *, fused_outputs=None) -> str:
    """Python launcher module around ``cuda_source`` (the ``code`` of a result)."""
    from cutile.lowering.emitter import CodeEmitter

    e = CodeEmitter()
    e.line(f'"""B200 stencil module for {name} (generated)."""')
    e.blank()
    e.line("import os")
    e.blank()
    e.line("from cutile.runtime.module import StencilProgram")
    e.blank()
    e.line("CUDA_SOURCE = r'''" + cuda_source + "'''")
    e.blank()
    e.line(f"SPEC = {spec!r}")
    e.line("SPEC['halo'] = tuple(SPEC['halo'])")
    _program_lines(e)
    inputs = spec["input_names"]
    outs = spec["output_params"]
    scal = spec.get("scalars", [])
    kw = (", *, " + ", ".join(scal)) if scal else ""
    sc = ("{" + ", ".join(f"{n!r}: {n}" for n in scal) + "}") if scal else "None"
    e.blank()
    e.blank()
    args = ", ".join(inputs + outs)
    e.line(f"def launch_{name}({args}, stream=None{kw}):")
    with e.indent():
        e.line(f'"""{spec["temporal_steps"]} step(s) of {name}; writes the interior of the output(s)."""')
        e.line(f"_PROGRAM.launch(({', '.join(inputs)},), ({', '.join(outs)},), stream, scalars={sc})")
    if spec.get("boundary") is not None:
        e.blank()
        e.blank()
        e.line(f"def apply_boundary_{name}(u, stream=None):")
        with e.indent():
            e.line('"""Apply boundary conditions to halo cells (in place)."""')
            e.line("_PROGRAM.apply_boundary(u, stream)")
        e.blank()
        e.blank()
        e.line(f"def step_{name}({args}, stream=None{kw}):")
        with e.indent():
            e.line('"""One step with the boundary condition fused into the staging."""')
            e.line(f"_PROGRAM.step(({', '.join(inputs)},), ({', '.join(outs)},), stream, scalars={sc})")
    if spec.get("layout") == "bricked":
        bs = spec["brick_size"]
        e.blank()
        e.blank()
        e.line(f"def to_bricks(flat_array, brick_size={bs}, stream=None):")
        with e.indent():
            e.line('"""Bricked copy of a flat device array (one kernel launch)."""')
            e.line("return _PROGRAM.to_bricks(flat_array, brick_size, stream)")
        e.blank()
        e.blank()
        e.line(f"def from_bricks(bricked, original_shape, brick_size={bs}, stream=None):")
        with e.indent():
            e.line('"""Flat array of ``original_shape`` from its bricked form."""')
            e.line("return _PROGRAM.from_bricks(bricked, original_shape, brick_size, stream)")
        e.blank()
        e.blank()
        e.line(f"def launch_{name}_bricked({args}, brick_size={bs}, stream=None{kw}):")
        with e.indent():
            e.line('"""Bricked launch on flat arrays: the inputs are bricked, the bricked '
                   'kernel runs, and')
            e.line('the whole output is written back (interior = result, halo = 0)."""')
            e.line(f"_PROGRAM.launch_bricked(({', '.join(inputs)},), ({', '.join(outs)},), "
                   f"brick_size, stream, scalars={sc})")
        e.blank()
        e.blank()
        e.line(f"def launch_{name}_on_bricks({args}, shape, stream=None{kw}, halo=None):")
        with e.indent():
            e.line('"""The bricked kernel on fields already stored as bricks of a ``shape`` '
                   'array')
            e.line('(``halo``: the arrays\' halo widths, default ``halo_widths``)."""')
            e.line(f"_PROGRAM.launch_on_bricks(({', '.join(inputs)},), ({', '.join(outs)},), "
                   f"shape, stream, scalars={sc}, halo=halo)")
    e.blank()
    e.blank()
    e.line("def program():")
    with e.indent():
        e.line('"""The StencilProgram behind this module."""')
        e.line("return _PROGRAM")
    return e.render()


def chain_tile_3d(dtype_bytes: int, T: int) -> dict:
    """Default column tile and block size of a 3-D chain of T steps.

    Measured on B200, 7-point Laplacian 512^3, eight waves, GPts/s counting
    every step (plan sweeps over 4..32 x 32..128 tiles and 64..512 threads):
    FP64 T=2 8 x 128 / 256 threads 366 (16 x 64: 356; the single-step 4 x 128
    default 200); FP64 T=4 16 x 64 / 512 threads 246 (8 x 64 / 256: 159);
    FP32 T=2 8 x 128 / 128 threads 661 (/ 256: 622); FP32 T=4 32 x 64 / 512
    threads 445 (8 x 128 / 256: 282); FP32 T=8 16 x 32 / 128 threads 137
    (8 x 64: 122).  Past T=2 the rings leave one block per SM, and the
    tallest tile that fits, with a thread per unit, beats smaller tiles at
    higher occupancy: every stage recomputes 2(T - s) r halo rows per tile.
    ``fit_plan`` shrinks the tile of wider footprints until it fits."""
    if T == 2:
        return (dict(tile_y=8, tile_x=128, threads=256) if dtype_bytes == 8 else
                dict(tile_y=8, tile_x=128, threads=128))
    if T <= 4:
        return (dict(tile_y=16, tile_x=64, threads=512) if dtype_bytes == 8 else
                dict(tile_y=32, tile_x=64, threads=512))
    return (dict(tile_y=8, tile_x=32, threads=128) if dtype_bytes == 8 else
            dict(tile_y=16, tile_x=32, threads=128))


def chain_tile_2d(dtype_bytes: int, T: int) -> dict:
    """Default chunk (rows x columns) and block size of a 2-D chain of T steps.

    Measured on B200, 5-point heat 4096^2, GPts/s counting every step (plan
    sweeps over 4..32 rows, 64..256 columns, 128..512 threads; differences
    under 5 % are kept at the simpler plan): FP64 T=2 8 x 64 / 128 threads
    368, T=3 4 x 128 / 128 351 (/ 256: 328), T=4 4 x 128 / 256 302, T=5 259,
    T=8 176; FP32 T=2 8 x 128 / 128 581 (8 x 64: 516), T=3 8 x 128 / 256
    513 (4 x 128: 486), T=4 4 x 128 455, T=5 389, T=8 8 x 128 / 256 287
    (4 x 128: 271)."""
    if dtype_bytes == 8:
        if T == 2:
            return dict(rows=8, tile_x=64, threads=128)
        return dict(rows=4, tile_x=128, threads=128 if T == 3 else 256)
    if T == 2:
        return dict(rows=8, tile_x=128, threads=128)
    if T == 3 or T >= 8:
        return dict(rows=8, tile_x=128, threads=256)
    return dict(rows=4, tile_x=128, threads=256)


def _rpy_keeps_registers(stencil_fn, plan, stencil_halo, halo_widths, dtype, dtype_bytes,
                         num_inputs, T, body_ops, kahan) -> bool:
    """Whether the rows-per-thread default compiles without spills for this
    body.  Dense boxes whose terms the DSL orders irregularly keep many strips
    live at once; ptxas' report of the NVRTC build (cached, so the module
    load reuses it) decides.  Without a working NVRTC the plan is kept."""
    from cutile.lowering.stencil_to_target import lower_to_target_ir
    from cutile.lowering.target_to_cuda import emit_cuda
    from cutile.passes.tiling import fit_plan
    from cutile.runtime import native
    from cutile.runtime.regcheck import parse_ptxas_log

    p = fit_plan(plan, stencil_halo, dtype_bytes, num_inputs, body_ops)
    target = lower_to_target_ir(stencil_fn._ir.clone(), p.tile_sizes(), halo_widths,
                                temporal_steps=T, kernel_hints=p.hints(), dtype=dtype,
                                kahan=kahan)
    try:
        _, log = native.compile_source(emit_cuda(target))
    except Exception:  # noqa: BLE001 - no NVRTC here: keep the measured default
        return True
    res = parse_ptxas_log(log, f"{stencil_fn._fn.__name__}_tma")
    return res is None or not res.spills


def _analysis_of(clone) -> tuple:
    halo_widths, tile_sizes, temporal_steps = (1,), (256,), 1
    analysis, occupancy, num_loads = {}, None, 0
    body_ops = 0
    from cutile.passes.tiling import unique_access_count

    for op in clone.walk():
        if isinstance(op, ApplyOp):
            a = op.attributes
            if "halo_widths" in a:
                halo_widths = tuple(x.data for x in a["halo_widths"])
            if "tile_sizes" in a:
                tile_sizes = tuple(x.data for x in a["tile_sizes"])
            if "temporal_steps" in a:
                temporal_steps = a["temporal_steps"].data
            if "occupancy" in a:
                occupancy = a["occupancy"].data
            num_loads = unique_access_count(op)
            body_ops = sum(1 for _ in op.region.walk())
            for key in ("flops", "unique_loads", "arithmetic_intensity", "bound"):
                if key in a:
                    analysis[key] = a[key].data
            break
    analysis["body_ops"] = body_ops
    return halo_widths, tile_sizes, temporal_steps, analysis, occupancy, num_loads


def compile(stencil_fn, domain: tuple[int, ...] | None = None, hw=None,
            pipeline: Pipeline | None = None, temporal_blocking: bool = True,
            autotune: bool = True, num_gpus: int = 1, split_axis: int = 0, overlap: bool = True,
            layout: str | None = None, brick_size: int = 32, align_halo: bool = True,
            occupancy: int | None = None, select: str | None = None, *,
            temporal_steps: int | None = None, tile_sizes: tuple[int, ...] | None = None,
            kernel_hints: dict | None = None, dtype: str | None = None,
            precision: str | None = None, reduce: str | None = None) -> CompileResult:
    """Compile a ``@stencil`` function for the B200 engine (launcher.py:342-602).

    ``precision`` (extension): ``"fp64"``, ``"fp32"`` or ``"fp32_kahan"`` --
    the last stores fields in FP32 and applies the body, which must read
    ``u + increment``, as a Kahan-compensated update with a compensation field
    (``launch_<name>(u_in, c_in, u_out, c_out)``).  ``reduce="max"``
    (extension) compiles a pointwise body whose values are max-reduced per
    grid into a device scalar (``reduce_<name>(inputs..., out=None)``)."""
    if reduce is not None:
        return _compile_reduction(stencil_fn, reduce, dtype=dtype, precision=precision,
                                  align_halo=align_halo)
    from cutile.lowering.stencil_to_target import lower_to_target_ir
    from cutile.lowering.target_to_cuda import emit_cuda
    from cutile.passes.tiling import default_engine_plan, fit_plan

    if num_gpus != 1:
        raise NotImplementedError("multi-GPU domain decomposition is not part of the B200 backend")
    ir = stencil_fn._ir
    name = stencil_fn._fn.__name__
    dtype, kahan = _precision(precision, dtype or getattr(stencil_fn, "_dtype", "float64"))
    dtype_bytes = 4 if dtype in ("float32", "fp32") else 8
    if hw is not None:
        dtype_bytes = hw.dtype_bytes
    clone = ir.clone()
    if pipeline is None:
        shared_mem = 49152 if hw is None else hw.shared_mem_bytes
        pipeline = Pipeline.single_gpu(shared_mem_bytes=shared_mem, dtype_bytes=dtype_bytes,
                                       max_temporal_steps=8 if temporal_blocking else 1)
    pipeline.run(clone)
    halo_widths, _ref_tile, T, analysis, pass_occ, num_loads = _analysis_of(clone)
    if not temporal_blocking:
        T = 1
    num_inputs = _num_inputs(ir)
    stencil_halo = halo_widths
    if align_halo and layout != "bricked":
        halo_widths = pad_inner_halo(halo_widths, dtype_bytes)

    plan = default_engine_plan(len(stencil_halo), num_loads, dtype_bytes, stencil_halo, num_inputs,
                               _yields(ir))
    resources = None
    if autotune and domain is not None:
        from cutile.runtime.autotune import autotune as _autotune

        res = _autotune(stencil_fn, domain, hw=hw, dtype=dtype)
        if res.plan is not None:
            plan = res.plan
        T = res.temporal_steps
    if kahan:
        num_inputs += 1  # the compensation field
    n_out = _yields(ir) * (2 if kahan else 1)
    if temporal_steps is not None:
        T = int(temporal_steps)
        if T > 1 and num_inputs != n_out:
            # a chain feeds output field f into input field f of the next
            # step (an extension: the reference chains one field only)
            raise NotImplementedError("temporal blocking needs one output per input field "
                                      "(output f feeds input f of the next step)")
    elif num_inputs != 1 or _yields(ir) > 1:
        # The reference's T-launch loop chains one field only
        # (stencil_to_target.py:796-800), so a multi-field stencil cannot run
        # blocked there either; it advances one step per launch.
        T = 1
    plan = replace(plan, temporal=T, rpy=plan.rpy if T == 1 else 1)
    hinted_rpy = bool(kernel_hints) and ("rows_per_thread" in kernel_hints or "rpy" in kernel_hints)
    if plan.rpy > 1 and tile_sizes is None and not hinted_rpy and not _rpy_keeps_registers(
            stencil_fn, plan, stencil_halo, halo_widths, dtype, dtype_bytes, num_inputs, T,
            analysis.get("body_ops", 0), kahan):
        # the default rows-per-thread plan would spill this body's strips:
        # one row per thread over the wide tile instead
        plan = replace(plan, rpy=1, rows=1, tile_y=4, tile_x=64)
    if T > 1 and len(stencil_halo) == 3 and tile_sizes is None and not plan.rpy > 1:
        plan = replace(plan, rows=1, **chain_tile_3d(dtype_bytes, T))
    elif T > 1 and len(stencil_halo) == 2 and tile_sizes is None:
        plan = replace(plan, **chain_tile_2d(dtype_bytes, T))
    if layout == "bricked" and len(stencil_halo) == 3 and tile_sizes is None:
        # one Z row per chunk, so that the bricked kernel can stage bricks
        # with tensor copies (target_to_cuda.brick_tma_eligible)
        plan = replace(plan, rows=1)
    plan = _plan_from(tile_sizes, kernel_hints, len(stencil_halo), plan)
    if occupancy is not None:
        plan = replace(plan, occupancy=int(occupancy))
    plan = fit_plan(plan, stencil_halo, dtype_bytes, num_inputs, analysis.get("body_ops", 0))
    if layout == "bricked" and plan.vec != 16 // dtype_bytes:
        raise ValueError("bricked kernels keep one 16-byte vector per unit")
    verify_engine_plan(clone, plan, stencil_halo, dtype_bytes, num_inputs)
    hints = plan.hints()
    if occupancy is not None:
        hints["occupancy"] = occupancy

    boundary_spec = None
    if getattr(stencil_fn, "_boundary", None) is not None:
        b = stencil_fn._boundary
        boundary_spec = {"type": b} if isinstance(b, str) else (
            dict(b) if isinstance(b, dict) else b.to_dict())
        if "bc_type" in boundary_spec and "type" not in boundary_spec:
            boundary_spec["type"] = boundary_spec.pop("bc_type")
    target = lower_to_target_ir(ir.clone(), plan.tile_sizes(), halo_widths, temporal_steps=T,
                                boundary_spec=boundary_spec, kernel_hints=hints, dtype=dtype,
                                kahan=kahan)
    cuda = emit_cuda(target)
    kernels = {"main": name}
    if boundary_spec is not None:
        bc_plan = fit_plan(replace(plan, temporal=1), stencil_halo, dtype_bytes, num_inputs,
                           analysis.get("body_ops", 0),
                           periodic=boundary_spec.get("type") == "periodic")
        verify_engine_plan(clone, bc_plan, stencil_halo, dtype_bytes, num_inputs,
                           periodic=boundary_spec.get("type") == "periodic")
        bc_target = lower_to_target_ir(ir.clone(), bc_plan.tile_sizes(), halo_widths,
                                       temporal_steps=1, boundary_spec=boundary_spec,
                                       kernel_hints=bc_plan.hints(), dtype=dtype,
                                       boundary_mode=boundary_spec.get("type", "dirichlet"),
                                       kahan=kahan)
        _rename_kernel(bc_target, f"{name}_bc")
        cuda += "\n" + emit_cuda(bc_target, preamble=False)
        kernels["fused_bc"] = f"{name}_bc"
    if layout == "bricked":
        # the same stencil reading and writing fields stored as bricks
        bk_target = lower_to_target_ir(ir.clone(), plan.tile_sizes(), halo_widths,
                                       temporal_steps=T, kernel_hints=hints, dtype=dtype,
                                       kahan=kahan, layout="bricked", brick_size=int(brick_size))
        _rename_kernel(bk_target, f"{name}_bk")
        cuda += "\n" + emit_cuda(bk_target, preamble=False)
        kernels["bricked"] = f"{name}_bk"
    in_names = _input_names(ir)
    n_fields = num_inputs - (1 if kahan else 0)
    multi = n_fields > 1
    names = ([n for n in "uvwxyz"][:n_fields] if n_fields <= 6 else
             [f"arr{i}" for i in range(n_fields)]) if multi else ["u_in"]
    n_out = _kernel_outputs(target)
    outs = ["u_out"] if n_out == 1 else [f"out{k}" for k in range(n_out)]
    if kahan:
        names = names + ["c_in"]
        outs = ["u_out", "c_out"]
    spec = {
        "name": name, "ndim": len(stencil_halo), "dtype": dtype, "halo": list(halo_widths),
        "stencil_halo": list(stencil_halo), "inputs": num_inputs, "outputs": len(outs),
        "temporal_steps": T, "boundary": boundary_spec, "kernels": kernels,
        "input_names": names, "output_params": outs, "zchunk": plan.zchunk,
        "precision": precision or ("fp32" if dtype == "float32" else "fp64"),
        "scalars": _scalar_names(ir),
        "layout": layout or "flat", "brick_size": int(brick_size) if layout == "bricked" else 0,
    }
    code = generate_module_code(name, cuda, spec)
    return CompileResult(
        name=name, code=code, ndim=stencil_fn._ndim or len(halo_widths),
        halo_widths=tuple(halo_widths), tile_sizes=plan.tile_sizes(), temporal_steps=T,
        analysis=analysis, stencil_halo=tuple(stencil_halo), kernel_hints=hints,
        resources=resources, inputs=in_names + (("c_in",) if kahan else ()), cuda_source=cuda,
        dtype=dtype,
        boundary=boundary_spec, layout=layout or "flat", brick_size=brick_size if layout == "bricked" else 0,
        _ref_fn=stencil_fn._fn, _ref_fns=[stencil_fn._fn])


def _yields(ir) -> int:
    from cutile.dialects.cutile_stencil.dialect import YieldOp
    from cutile.lowering.stencil_to_target import _func_and_block

    _, b = _func_and_block(ir)
    for op in b.ops:
        if isinstance(op, YieldOp):
            return len(op.operands)
    return 1


def _kernel_outputs(target) -> int:
    from cutile.dialects.cutile_target import KernelOp

    for op in target.body.block.ops:
        if isinstance(op, KernelOp):
            return sum(max(1, sum(1 for x in prog if x.data.startswith("return")))
                       for prog in op.ssa_body.data)
    return 1


def _scalar_names(ir) -> list:
    from cutile.lowering.stencil_to_target import _func_and_block

    f, _ = _func_and_block(ir)
    return [a.data for a in f.scalar_names.data] if f.scalar_names is not None else []


def _rename_kernel(target, new_name: str) -> None:
    from cutile.dialects.cutile_target import KernelOp
    from cutile.ir.core import StringAttr

    for op in target.body.block.ops:
        if isinstance(op, KernelOp):
            op.properties["kernel_name"] = StringAttr(new_name)


# --------------------------------------------------------------------------- #
# compile_fused()
# --------------------------------------------------------------------------- #


def compile_fused(stencil_fns: list, domain: tuple[int, ...] | None = None, hw=None,
                  tile_sizes: tuple[int, ...] | None = None,
                  halo_widths: tuple[int, ...] | None = None, temporal_steps: int = 1,
                  occupancy: int | None = None, align_halo: bool = True,
                  select: str | None = None, *, kernel_hints: dict | None = None,
                  dtype: str | None = None, boundary=None,
                  precision: str | None = None) -> CompileResult:
    """Several stencils over one domain in one multi-output kernel
    (launcher.py:610-728): each distinct (field, offset) is staged once and
    every output is stored.  ``boundary`` (extension) adds a ``step_<name>``
    with that boundary condition fused into the staging of all inputs."""
    from cutile.lowering.stencil_to_target import extract_fused_meta, lower_fused_to_target_ir
    from cutile.lowering.target_to_cuda import emit_cuda
    from cutile.passes.tiling import default_engine_plan, fit_plan

    if not stencil_fns:
        raise ValueError("At least one stencil function is required")
    if temporal_steps != 1:
        raise NotImplementedError(
            "temporal blocking of fused kernels is not supported (temporal_steps must be 1)")
    modules = [fn._ir for fn in stencil_fns]
    dtype, kahan = _precision(precision, dtype or getattr(stencil_fns[0], "_dtype", "float64"))
    meta = extract_fused_meta(modules, dtype=dtype)
    if kahan:
        from cutile.lowering.stencil_to_target import apply_kahan

        apply_kahan(meta)
    ndim = meta.ndim
    dtype_bytes = 4 if dtype in ("float32", "fp32") else 8
    if hw is not None:
        dtype_bytes = hw.dtype_bytes
    if halo_widths is None:
        per = []
        for m in modules:
            c = m.clone()
            Pipeline.single_gpu(dtype_bytes=dtype_bytes, max_temporal_steps=1).run(c)
            per.append(_analysis_of(c)[0])
        halo_widths = tuple(max(hs) for hs in zip(*per)) if per else (1,) * ndim
    stencil_halo = tuple(halo_widths)
    if align_halo:
        halo_widths = pad_inner_halo(tuple(halo_widths), dtype_bytes)
    num_loads = len(meta.accesses)
    plan = default_engine_plan(ndim, num_loads, dtype_bytes, stencil_halo, meta.num_inputs,
                               meta.num_outputs)
    plan = _plan_from(tile_sizes, kernel_hints, ndim, plan)
    if occupancy is not None:
        plan = replace(plan, occupancy=int(occupancy))
    body_ops = sum(sum(1 for _ in m.walk()) for m in modules)
    plan = fit_plan(plan, stencil_halo, dtype_bytes, meta.num_inputs, body_ops)
    for m in modules:
        c = m.clone()
        Pipeline.single_gpu(dtype_bytes=dtype_bytes, max_temporal_steps=1).run(c)
        verify_engine_plan(c, plan, stencil_halo, dtype_bytes, meta.num_inputs,
                           periodic=boundary == "periodic")
    hints = plan.hints()
    if occupancy is not None:
        hints["occupancy"] = occupancy
    target = lower_fused_to_target_ir(modules, plan.tile_sizes(), tuple(halo_widths), hints,
                                      dtype=dtype, kahan=kahan)
    cuda = emit_cuda(target)
    kernels = {"main": meta.name}
    bspec = None
    if boundary is not None:
        bspec = {"type": boundary} if isinstance(boundary, str) else (
            dict(boundary) if isinstance(boundary, dict) else boundary.to_dict())
        bc_hints = hints
        if bspec["type"] == "periodic":
            # the wrap buffer enlarges shared memory: refit the launch bound
            bc_hints = fit_plan(plan, stencil_halo, dtype_bytes, meta.num_inputs, body_ops,
                                periodic=True).hints()
            if occupancy is not None:
                bc_hints["occupancy"] = occupancy
        bc_target = lower_fused_to_target_ir(modules, plan.tile_sizes(), tuple(halo_widths),
                                             bc_hints, dtype=dtype, boundary_mode=bspec["type"],
                                             kahan=kahan)
        _rename_kernel(bc_target, f"{meta.name}_bc")
        cuda += "\n" + emit_cuda(bc_target, preamble=False)
        kernels["fused_bc"] = f"{meta.name}_bc"
    spec = {
        "name": meta.name, "ndim": ndim, "dtype": dtype, "halo": list(halo_widths),
        "stencil_halo": list(stencil_halo), "inputs": meta.num_inputs,
        "outputs": meta.num_outputs, "temporal_steps": 1, "boundary": bspec, "kernels": kernels,
        "input_names": list(meta.input_names), "output_params": meta.output_params(),
        "zchunk": plan.zchunk, "precision": precision or ("fp32" if dtype == "float32" else "fp64"),
    }
    code = generate_module_code(meta.name, cuda, spec)
    return CompileResult(
        name=meta.name, code=code, ndim=ndim, halo_widths=tuple(halo_widths),
        tile_sizes=plan.tile_sizes(), temporal_steps=1, analysis={"unique_loads": num_loads},
        stencil_halo=stencil_halo, kernel_hints=hints, resources=None,
        inputs=tuple(meta.input_names),
        outputs=tuple(meta.output_names) + (tuple(f"{n}_c" for n in meta.output_names) if kahan
                                            else ()), cuda_source=cuda,
        dtype=dtype, boundary=bspec, _ref_fns=[fn._fn for fn in stencil_fns],
        _ref_inputs=meta.stencil_inputs)


__all__ = ["compile", "compile_fused", "CompileResult", "pad_inner_halo",
           "generate_module_code"]


# --------------------------------------------------------------------------- #
# Kernel variants (Runge-Kutta stages, reductions) of one stencil
# --------------------------------------------------------------------------- #


def build_variants(stencil_fn, variants: dict, *, dtype: str | None = None,
                   precision: str | None = None, align_halo: bool = True,
                   tile_sizes=None, kernel_hints=None, boundary=None):
    """Lower several kernel variants of one stencil into one CUDA unit.

    ``variants`` maps a kernel name to options for ``lower_to_target_ir``
    (``rk=``, ``reduce_max=``, ``boundary_mode=``).  Returns
    ``(cuda_source, info)`` with the halo (padded and stencil), the engine plan
    and, per kernel, its input and output counts.
    """
    from cutile.lowering.stencil_to_target import lower_to_target_ir
    from cutile.lowering.target_to_cuda import emit_cuda, engine_params
    from cutile.passes.tiling import default_engine_plan, fit_plan

    ir = stencil_fn._ir
    dtype, _ = _precision(precision, dtype or getattr(stencil_fn, "_dtype", "float64"))
    dtype_bytes = 4 if dtype == "float32" else 8
    clone = ir.clone()
    Pipeline.single_gpu(dtype_bytes=dtype_bytes, max_temporal_steps=1).run(clone)
    stencil_halo, _t, _T, analysis, _o, num_loads = _analysis_of(clone)
    halo_widths = pad_inner_halo(stencil_halo, dtype_bytes) if align_halo else stencil_halo
    n_fields = _num_inputs(ir)
    parts = []
    info = {"halo": tuple(halo_widths), "stencil_halo": tuple(stencil_halo), "dtype": dtype,
            "kernels": {}, "scalars": _scalar_names(ir), "analysis": analysis}
    bspec = None
    if boundary is not None:
        bspec = {"type": boundary} if isinstance(boundary, str) else dict(boundary)
    first = True
    for kname, opts in variants.items():
        opts = dict(opts)
        extra_in = 0
        if opts.get("rk") is not None:
            rk = opts["rk"]
            m = _yields(ir)
            extra_in = ((m if rk["a"] != 0.0 and not rk.get("same_base") else 0)
                        + (m if rk.get("w") is not None else 0))
        plan = default_engine_plan(len(stencil_halo), num_loads, dtype_bytes, stencil_halo,
                                   n_fields + extra_in, _yields(ir))
        if len(stencil_halo) == 2 and tile_sizes is None and analysis.get("body_ops", 0) > 120:
            # long 2-D flux bodies (issue-bound): 64-wide chunks; measured on
            # the 256-grid shallow-water RK2 batch, 6.82 ms per step against
            # 7.42 for 128-wide (4 instead of 2 blocks per SM)
            plan = replace(plan, tile_x=64)
        bmode = opts.pop("boundary_mode", "none")
        plan = fit_plan(_plan_from(tile_sizes, kernel_hints, len(stencil_halo), plan),
                        stencil_halo, dtype_bytes, n_fields + extra_in,
                        analysis.get("body_ops", 0), periodic=bmode == "periodic")
        verify_engine_plan(clone, plan, stencil_halo, dtype_bytes, n_fields + extra_in,
                           periodic=bmode == "periodic")
        target = lower_to_target_ir(ir.clone(), plan.tile_sizes(), tuple(halo_widths),
                                    kernel_hints=plan.hints(), dtype=dtype, name=kname,
                                    boundary_spec=bspec, boundary_mode=bmode, **opts)
        parts.append(emit_cuda(target, preamble=first))
        first = False
        from cutile.dialects.cutile_target import KernelOp

        kop = next(op for op in target.body.block.ops if isinstance(op, KernelOp))
        ep = engine_params(kop)
        info["kernels"][kname] = {"inputs": ep["NIN"], "outputs": 0 if ep["REDUCE"] else ep["NOUT"],
                                  "plan": plan}
    return "\n".join(parts), info


def _compile_reduction(stencil_fn, reduce: str, *, dtype=None, precision=None,
                       align_halo=True) -> CompileResult:
    from cutile.lowering.emitter import CodeEmitter

    if reduce != "max":
        raise ValueError("only reduce='max' is supported (non-negative values, NaN propagates)")
    name = stencil_fn._fn.__name__
    cuda, info = build_variants(stencil_fn, {name: {"reduce_max": True}}, dtype=dtype,
                                precision=precision, align_halo=align_halo)
    n_in = info["kernels"][name]["inputs"]
    names = [f"u{k}" for k in range(n_in)] if n_in > 1 else ["u_in"]
    spec = {"name": name, "ndim": len(info["halo"]), "dtype": info["dtype"],
            "halo": list(info["halo"]), "stencil_halo": list(info["stencil_halo"]),
            "inputs": n_in, "outputs": 0, "temporal_steps": 1, "boundary": None,
            "kernels": {"main": name}, "input_names": names, "output_params": [],
            "zchunk": 0, "scalars": info["scalars"], "reduce": "max"}
    e = CodeEmitter()
    e.line(f'"""Per-grid max of {name} over the interior (generated)."""')
    e.blank()
    e.line("import os")
    e.blank()
    e.line("from cutile.runtime.module import StencilProgram")
    e.blank()
    e.line("CUDA_SOURCE = r\'\'\'" + cuda + "\'\'\'")
    e.line(f"SPEC = {spec!r}")
    e.line("SPEC['halo'] = tuple(SPEC['halo'])")
    _program_lines(e)
    e.blank()
    e.blank()
    e.line(f"def reduce_{name}({', '.join(names)}, out=None, stream=None, **scalars):")
    with e.indent():
        e.line('"""Max over the interior into the device float64 ``out`` (returned);'
               ' the value is max(out, ...) when ``out`` is given."""')
        e.line(f"return _PROGRAM.reduce(({', '.join(names)},), out, stream, scalars)")
    e.blank()
    e.blank()
    e.line("def program():")
    with e.indent():
        e.line("return _PROGRAM")
    return CompileResult(name=name, code=e.render(), ndim=len(info["halo"]),
                         halo_widths=tuple(info["halo"]), tile_sizes=(), temporal_steps=1,
                         analysis=info["analysis"], stencil_halo=tuple(info["stencil_halo"]),
                         inputs=_input_names(stencil_fn._ir), cuda_source=cuda,
                         dtype=info["dtype"], _ref_fn=stencil_fn._fn, _ref_fns=[stencil_fn._fn])
