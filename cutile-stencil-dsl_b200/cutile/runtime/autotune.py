"""Empirical autotuner over the B200 engine's plan space.

The reference (runtime/autotune.py:88-309) times cuTile tile shapes and
temporal depths on the GPU and caches the winner per stencil name and GPU.
Here the search is over the engine plan -- rows per streaming step, tile
(Y, X), threads, chunks in flight, work items per resident block, temporal
depth -- and the cache is keyed by what decides the best plan: the stencil's
footprint (per-dimension radius, distinct loads, fields in and out), the
dtype, the dimensionality and the grid-size class (log2 of the interior
points), plus the GPU name.  Every candidate goes through ``fit_plan`` (box,
shared-memory and register limits), is built with NVRTC, and runs on a
synthetic grid of the requested domain; GPoints/s counts the steps a launch
advances.  The cache is a JSON file in the package's build directory, so a
tuned plan travels with the tree.
"""

from __future__ import annotations

import json
import math
import os
import threading
from dataclasses import asdict, dataclass, field, replace

_CACHE_VERSION = "b200-v1"
_lock = threading.Lock()


@dataclass
class AutotuneResult:
    tile_sizes: tuple
    temporal_steps: int
    throughput_gpoints: float
    bandwidth_gbs: float
    time_ms: float = 0.0
    kernel_hints: dict = field(default_factory=dict)
    plan: object = None
    candidates: int = 0


def cache_path() -> str:
    from cutile.runtime.native import default_cache_dir

    return os.path.join(os.path.dirname(default_cache_dir()), "autotune.json")


def _footprint(stencil_fn, dtype_bytes: int):
    from cutile.runtime.launcher import Pipeline, _analysis_of, _num_inputs, _yields

    clone = stencil_fn._ir.clone()
    Pipeline.single_gpu(dtype_bytes=dtype_bytes, max_temporal_steps=1).run(clone)
    halo, _t, _T, analysis, _o, num_loads = _analysis_of(clone)
    return {"radius": list(halo), "loads": num_loads, "inputs": _num_inputs(stencil_fn._ir),
            "outputs": _yields(stencil_fn._ir), "body_ops": analysis.get("body_ops", 0)}


def cache_key(fp: dict, dtype: str, domain, gpu: str) -> str:
    pts = 1
    for n in domain:
        pts *= int(n)
    size_class = int(round(math.log2(max(1, pts))))
    return (f"{_CACHE_VERSION}|{gpu}|{dtype}|nd{len(domain)}|r{fp['radius']}|l{fp['loads']}|"
            f"i{fp['inputs']}o{fp['outputs']}|b{fp['body_ops']}|s{size_class}")


def _load(key: str):
    try:
        with open(cache_path()) as f:
            return json.load(f).get(key)
    except (OSError, ValueError):
        return None


def _save(key: str, entry: dict) -> None:
    path = cache_path()
    with _lock:
        try:
            with open(path) as f:
                data = json.load(f)
        except (OSError, ValueError):
            data = {}
        data[key] = entry
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + f".{os.getpid()}.tmp"
        with open(tmp, "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)
        os.replace(tmp, path)


def candidates(ndim: int, dtype_bytes: int, radius, num_inputs: int, num_loads: int,
               body_ops: int, single_field: bool, max_candidates: int = 30,
               num_outputs: int = 1) -> list:
    """Distinct fitted plans around the default one, most promising first."""
    from cutile.passes.tiling import EnginePlan, default_engine_plan, fit_plan

    vec = 16 // dtype_bytes
    base = default_engine_plan(ndim, num_loads, dtype_bytes, tuple(radius), num_inputs,
                               num_outputs)
    raw = [base]
    depths = (1, 2) if single_field else (1,)
    if ndim == 3:
        shapes = [(1, 4, 128), (1, 8, 128), (1, 2, 128), (1, 16, 64), (1, 8, 64), (1, 4, 64),
                  (2, 4, 128), (1, 16, 128), (1, 32, 32)]
        for (rows, ty, tx) in shapes:
            for nt in (128, 256):
                for T in depths:
                    raw.append(EnginePlan(3, rows=rows, tile_y=ty, tile_x=tx, vec=vec, threads=nt,
                                          stages=1, zchunk=0, temporal=T))
    elif ndim == 2:
        for rows in (4, 8, 16):
            for tx in (64, 128):
                for nt in (128, 256):
                    for T in (depths + ((4,) if single_field else ())):
                        raw.append(EnginePlan(2, rows=rows, tile_y=1, tile_x=tx, vec=vec,
                                              threads=nt, stages=1, zchunk=0, temporal=T))
    else:
        for tx in (64, 128):
            for nt in (64, 128, 256):
                for T in (depths + ((4, 8) if single_field else ())):
                    raw.append(EnginePlan(1, rows=1, tile_y=1, tile_x=tx, vec=vec, threads=nt,
                                          stages=0, zchunk=0, temporal=T))
    out, seen = [], set()
    for p in raw:
        try:
            f = fit_plan(p, tuple(radius), dtype_bytes, num_inputs, body_ops)
        except ValueError:
            continue
        if f.rows < radius[0] if ndim > 1 else False:
            continue
        key = (f.rows, f.tile_y, f.tile_x, f.threads, f.stages, f.temporal, f.min_blocks, f.rpy)
        if key in seen:
            continue
        seen.add(key)
        out.append(f)
    return out[:max_candidates]


def probe_hints(p) -> dict:
    """The kernel hints that make ``compile(tile_sizes=p.tile_sizes(), ...)``
    build exactly the candidate plan ``p`` (rows per thread included), so the
    plan that is timed is the plan that is returned."""
    return {"threads": p.threads, "stages": p.stages, "zchunk": p.zchunk,
            "min_blocks": p.min_blocks, "waves": p.waves, "rows_per_thread": p.rpy}


def _gpu_name() -> str:
    try:
        import torch

        return torch.cuda.get_device_name()
    except Exception:  # noqa: BLE001 - no device: the key says so
        return "unknown"


def autotune(stencil_fn, domain=None, hw=None, *, dtype: str | None = None,
             max_candidates: int = 30, warmup: int = 3, iters: int = 10,
             verbose: bool = False, use_cache: bool = True) -> AutotuneResult:
    """Time candidate plans of ``stencil_fn`` on a synthetic ``domain``
    (interior extents) and return the fastest; cached per footprint, dtype,
    dimensionality, size class and GPU."""
    import numpy as np
    import torch

    from cutile.runtime.launcher import compile as stencil_compile
    from cutile.runtime.regcheck import Config, Resources, select_fastest

    if domain is None:
        raise ValueError("autotune needs the domain (interior extents) to time on")
    dtype = dtype or getattr(stencil_fn, "_dtype", "float64") or "float64"
    if dtype in ("fp32",):
        dtype = "float32"
    dtype_bytes = 4 if dtype == "float32" else 8
    if hw is not None:
        dtype_bytes = hw.dtype_bytes
    fp = _footprint(stencil_fn, dtype_bytes)
    ndim = len(domain)
    gpu = _gpu_name()
    key = cache_key(fp, dtype, domain, gpu)
    if use_cache:
        hit = _load(key)
        if hit is not None:
            from cutile.passes.tiling import EnginePlan

            plan = EnginePlan(**hit["plan"])
            return AutotuneResult(tuple(hit["tile_sizes"]), hit["temporal_steps"],
                                  hit["gpoints"], hit["gbs"], hit["ms"], hit["hints"], plan,
                                  hit.get("candidates", 0))
    single = fp["inputs"] == 1 and fp["outputs"] == 1
    plans = candidates(ndim, dtype_bytes, fp["radius"], fp["inputs"], fp["loads"],
                       fp["body_ops"], single, max_candidates, fp["outputs"])
    if not torch.cuda.is_available():
        raise RuntimeError("autotune times candidates on the GPU; no CUDA device is visible")
    pts = 1
    for n in domain:
        pts *= int(n)
    results = {}

    def probe(cfg: Config):
        p = plans[cfg.kernel_hints["_index"]]
        hints = probe_hints(p)
        try:
            r = stencil_compile(stencil_fn, tile_sizes=p.tile_sizes(), kernel_hints=hints,
                                temporal_steps=p.temporal, dtype=dtype, autotune=False,
                                align_halo=True)
        except (ValueError, NotImplementedError):
            return None
        halo = r.halo_widths
        shape = tuple(int(n) + 2 * h for n, h in zip(domain, halo))
        tdt = torch.float64 if dtype == "float64" else torch.float32
        rng = np.random.default_rng(0)
        prog = r.load_module().program()
        ins = []
        for _ in range(prog.spec["inputs"]):
            a = torch.zeros(shape, dtype=tdt, device="cuda")
            inner = tuple(slice(h, s - h) for h, s in zip(halo, shape))
            a[inner] = torch.from_numpy(rng.random(tuple(domain)).astype(np.float64)).to(
                device="cuda", dtype=tdt)
            ins.append(a)
        outs = [torch.zeros_like(ins[0]) for _ in range(prog.spec["outputs"])]
        try:
            for _ in range(warmup):
                prog.launch(ins, outs)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(iters):
                prog.launch(ins, outs)
            e1.record()
            e1.synchronize()
        except Exception:  # noqa: BLE001 - a candidate that cannot launch is skipped
            return None
        ms = e0.elapsed_time(e1) / iters
        results[cfg.kernel_hints["_index"]] = (prog.spec["inputs"] + prog.spec["outputs"], ms)
        res = prog.kernel("main").resources()
        if verbose:
            print(f"autotune {p.tile_sizes()} t{p.threads} T{p.temporal}: {ms * 1e3:.1f} us, "
                  f"{pts * p.temporal / ms / 1e6:.1f} GPts/s")
        # rank by time per step
        return Resources(registers=res["registers"], stack_bytes=res["local_bytes"],
                         ms=ms / p.temporal, spill_bytes=res["local_bytes"])

    cfgs = [Config(tile_sizes=p.tile_sizes(), kernel_hints={"_index": k}, temporal_steps=p.temporal)
            for k, p in enumerate(plans)]
    best = select_fastest(cfgs, probe)
    k = best.kernel_hints["_index"]
    if k not in results:
        raise RuntimeError("autotune: no candidate could be timed")
    plan = plans[k]
    nfields, ms = results[k]
    nbytes = nfields * dtype_bytes * pts
    out = AutotuneResult(tile_sizes=plan.tile_sizes(), temporal_steps=plan.temporal,
                         throughput_gpoints=pts * plan.temporal / ms / 1e6,
                         bandwidth_gbs=nbytes / ms / 1e6, time_ms=ms,
                         kernel_hints=plan.hints(), plan=plan, candidates=len(plans))
    if use_cache:
        _save(key, {"plan": asdict(plan), "tile_sizes": list(plan.tile_sizes()),
                    "temporal_steps": plan.temporal, "gpoints": out.throughput_gpoints,
                    "gbs": out.bandwidth_gbs, "ms": ms, "hints": out.kernel_hints,
                    "candidates": len(plans)})
    return out


__all__ = ["AutotuneResult", "autotune", "candidates", "cache_key", "cache_path"]
