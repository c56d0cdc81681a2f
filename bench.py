"""Benchmark: 3-D 7-point Laplacian, 512^3 interior, FP64, on one B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--dtype float64|float32] [--temporal T]

A *step* is one sweep of the stencil over the 512^3 grid (``launch_lap7``
with ping-pong buffers), inputs resident in HBM.  ``value`` is GPoints/s =
interior points x steps / device time (CUDA events on the launching stream,
max over ranks).  Arrays (1.15 GB each) are far larger than the 126 MB L2,
so no flush is needed between sweeps.

``e2e`` times the configured solve through the public API with host buffers:
per step, the initial field is copied from pinned host memory, 50 sweeps run
through ``launch_lap7`` and the result is read back; consecutive solves are
pipelined over two buffer pairs so copies overlap sweeps.

Other workloads (``--workload``): ``gray_scott`` (4096^2 fused Gray-Scott,
FP64/FP32/Kahan), ``sw_batch`` (256 batched shallow-water RK2 solves),
``serve`` (continuous-batching server on a Poisson request stream), ``wide``
(125/27-point boxes and an eight-in/five-out fused update).

``--impl reference`` times the reference's CPU algorithm (the NumPy
restatement in oracle/, the reference's own NumPy executor cannot travel)
on all host cores, on a bounded z-slab sample of the same grid.

With N > 1 (torchrun), every rank runs its own independent 512^3 solve
("replicas only": the path has no data exchange); ``value`` is the sum.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (os.path.join(ROOT, "cutile-stencil-dsl_b200"), ROOT, os.path.join(ROOT, "tests")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

N_INTERIOR = 512
SOLVE_STEPS = 50
METRIC = "GPts/s (3-D 7-pt 512^3 sweep)"


def _peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _max_over_ranks(value: float) -> float:
    """The largest ``value`` over all ranks (the process group's backend
    decides the device: CUDA for NCCL, host for gloo)."""
    import torch

    if not torch.distributed.is_initialized() or torch.distributed.get_world_size() == 1:
        return float(value)
    dev = "cuda" if torch.distributed.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def _dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.device_index = device_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device_index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    mx = float(parts[2])
                except ValueError:
                    continue
                for n, v in zip(names, parts[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def _compile(dtype: str, temporal: int, layout: str = "flat", brick: int = 8):
    import stencil_defs as D
    from cutile import compile as stencil_compile
    from cutile import stencil

    fn = stencil(ndim=3, order=2, dtype=dtype)(D.lap7)
    if layout == "bricked":
        return stencil_compile(fn, temporal_blocking=temporal > 1,
                               temporal_steps=temporal if temporal > 1 else None,
                               layout="bricked", brick_size=brick)
    return stencil_compile(fn, temporal_blocking=temporal > 1,
                           temporal_steps=temporal if temporal > 1 else None)


def _init_field(shape, halo, dtype, rank: int):
    import numpy as np

    u = np.zeros(shape, dtype=dtype)
    inner = tuple(slice(h, s - h) for h, s in zip(halo, shape))
    rng = np.random.default_rng(1 + rank)
    u[inner] = rng.standard_normal(tuple(s - 2 * h for h, s in zip(halo, shape))).astype(dtype)
    return u


def run_ours(args) -> dict:
    import numpy as np
    import torch

    world, rank, local = _dist()
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist

        dist.init_process_group("nccl", init_method="env://")
    np_dtype = np.float64 if args.dtype == "float64" else np.float32
    r = _compile(args.dtype, args.temporal, args.layout, args.brick)
    T = r.temporal_steps
    halo = r.halo_widths
    if args.layout == "bricked":
        # a zero halo of whole bricks (the stencil still reads one cell of
        # it): the interior starts on a brick, so the TMA staging's column
        # tiles (which start on a brick) hold interior points only
        halo = tuple(-(-h // args.brick) * args.brick for h in halo)
    shape = tuple(N_INTERIOR + 2 * h for h in halo)
    npts = N_INTERIOR ** 3
    u0 = _init_field(shape, halo, np_dtype, rank)
    mod = r.load_module()
    a = torch.from_numpy(u0).cuda()
    if args.layout == "bricked":
        # fields resident as bricks: the bricked kernel reads and writes them
        a = mod.to_bricks(a)
        b = torch.zeros_like(a)

        def launch(x, y):
            mod.launch_lap7_on_bricks(x, y, shape, halo=halo)
    else:
        launch = mod.launch_lap7
        b = torch.zeros_like(a)
    stream = torch.cuda.current_stream()

    # warm-up (JIT load, occupancy, clocks)
    for _ in range(args.warmup):
        launch(a, b)
        a, b = b, a
    torch.cuda.synchronize()

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        barrier()
        ev0.record(stream)
        for _ in range(args.steps):
            launch(a, b)
            a, b = b, a
        ev1.record(stream)
        barrier()
    ms = ev0.elapsed_time(ev1)
    if world > 1:
        ms = _max_over_ranks(ms)
    clocks = clk.summary()
    ms_per_step = ms / args.steps
    gpts = npts * T * args.steps / (ms / 1e3) / 1e9 * world
    itemsize = np.dtype(np_dtype).itemsize
    alg_bytes = 2 * itemsize * npts  # one read + one write per point per launch
    achieved = alg_bytes / (ms_per_step / 1e3) / 1e9
    peak, peak_kind = _peaks()

    # end-to-end: pinned host field -> device, 50-sweep solve, result -> host
    # (bricked: the host holds the field in bricked form).  Solves run as a
    # pipeline over three device buffer pairs on three streams, so one solve's
    # upload, another's sweeps and a third's download run at once (two copy
    # engines, one compute stream); with two pairs an upload waited for the
    # download of the solve before last and the copies could not both run
    # all the time.
    if args.layout == "bricked":
        host_in = mod.to_bricks(torch.from_numpy(u0).cuda()).cpu().pin_memory()
    else:
        host_in = torch.from_numpy(u0).pin_memory()
    npairs = 3
    host_outs = [torch.empty_like(host_in).pin_memory() for _ in range(npairs)]
    pairs = [(a, b)] + [(torch.empty_like(a), torch.empty_like(a)) for _ in range(npairs - 1)]
    s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()
    ev = {k: [torch.cuda.Event() for _ in range(npairs)] for k in ("h2d", "comp", "d2h")}
    e2e_steps = 32
    sweeps = max(1, SOLVE_STEPS // T)

    def solve(k):
        p = k % npairs
        x, y = pairs[p]
        if k >= npairs:                 # the pair's previous solve is read out
            s_in.wait_event(ev["d2h"][p])
        with torch.cuda.stream(s_in):
            x.copy_(host_in, non_blocking=True)
            ev["h2d"][p].record(s_in)
        stream.wait_event(ev["h2d"][p])
        with torch.cuda.stream(stream):
            for _ in range(sweeps):
                launch(x, y)
                x, y = y, x
            ev["comp"][p].record(stream)
        s_out.wait_event(ev["comp"][p])
        with torch.cuda.stream(s_out):
            host_outs[p].copy_(x, non_blocking=True)
            ev["d2h"][p].record(s_out)

    solve(0)
    torch.cuda.synchronize()
    barrier()
    t0 = time.perf_counter()
    for k in range(1, e2e_steps + 1):
        solve(k)
    torch.cuda.synchronize()
    e2e_ms = (time.perf_counter() - t0) * 1e3 / e2e_steps
    barrier()
    if world > 1:
        e2e_ms = _max_over_ranks(e2e_ms)
    e2e_gpts = npts * T * sweeps / (e2e_ms / 1e3) / 1e9 * world
    a, b = pairs[0]

    traffic = _profiled_traffic(args.dtype, T, args.layout)
    cpu = cpu_baseline(np_dtype) if (rank == 0 and world == 1 and not args.no_cpu) else None
    line = {
        "metric": METRIC, "value": round(gpts, 3), "unit": "GPts/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 5),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.dtype == "float64" else "f32", "data": "synthetic",
        "config": {"workload": f"3-D 7-point Laplacian u + 0.1*(sum6 - 6u), {N_INTERIOR}^3 interior, "
                               f"{args.dtype}, zero Dirichlet halo 1 ("
                               + (f"stored as a zero halo of one brick, {halo[0]} cells, per side"
                                  if args.layout == "bricked" else
                                  f"innermost padded to {halo[-1]} as compile() aligns")
                               + "), N(0,1) seed 1, one sweep per step",
                   "grid": list(shape), "temporal_steps": T, "tile": list(r.tile_sizes),
                   "layout": args.layout if args.layout == "flat" else f"bricked {args.brick}^3",
                   "l2": "arrays 1.15 GB >> 126 MB L2, no flush needed",
                   "parallelism": f"replicas{world}"},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                     "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": traffic,
                     "peak_kind": peak_kind,
                     "algorithmic_bytes_per_launch": alg_bytes},
        "e2e": {"value": round(e2e_gpts, 3), "unit": "GPts/s",
                "h2d_bytes_per_step": int(u0.nbytes), "d2h_bytes_per_step": int(u0.nbytes),
                "step": f"H2D of the field, {sweeps} launches of launch_lap7 ({SOLVE_STEPS} steps),"
                        f" D2H of the result; {e2e_steps} consecutive solves pipelined over "
                        f"{npairs} buffer pairs (copies on two streams overlap the sweeps), wall "
                        f"time per solve"},
        "gpu_launches": args.steps,
        "clocks": clocks,
        "cpu_baseline": cpu,
    }
    if world > 1:
        torch.distributed.destroy_process_group()
    return line if rank == 0 else None


def _profiled_traffic(dtype: str, T: int, layout: str = "flat"):
    """DRAM bytes per launch from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "lap7_512_traffic.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        d = json.load(f)
    return d.get(f"{dtype}_T{T}" + ("_bricked" if layout == "bricked" else ""))


def _slab_job(args):
    """One worker: time ``steps`` oracle sweeps of a z-slab (seeded)."""
    nz, dtype_name, steps, seed = args
    import numpy as np

    import stencil_defs as D
    from oracle import stencil_oracle as O

    dt = np.dtype(dtype_name)
    shape = (nz + 2, N_INTERIOR + 2, N_INTERIOR + 2)
    u = _init_field(shape, (1, 1, 1), dt, seed)
    t0 = time.perf_counter()
    for _ in range(steps):
        u = O.apply_stencil(u, D.lap7, 3, (1, 1, 1))
    return time.perf_counter() - t0, nz * N_INTERIOR * N_INTERIOR * steps


def cpu_baseline(np_dtype, cores: int = 1, planes: int = 96, steps: int = 20) -> dict:
    """The oracle (NumPy restatement of reference/stencil_ref.apply_stencil)
    on z-slabs of the 512^2 cross-section, ``cores`` worker processes."""
    import multiprocessing as mp

    import numpy as np

    name = np.dtype(np_dtype).name
    if cores == 1:
        secs, pts = _slab_job((planes, name, steps, 0))
        total_pts, wall = pts, secs
    else:
        ctx = mp.get_context("spawn")
        with ctx.Pool(cores) as pool:
            pool.map(_slab_job, [(2, name, 1, k) for k in range(cores)])  # warm the workers
            t0 = time.perf_counter()
            res = pool.map(_slab_job, [(planes, name, steps, k) for k in range(cores)])
            wall = time.perf_counter() - t0
        total_pts = sum(p for _, p in res)
    return {"value": round(total_pts / wall / 1e9, 5), "unit": "GPts/s", "cores": cores,
            "kind": "port",
            "sample": f"{cores} x {steps} sweeps of a {planes}x512x512 z-slab "
                      f"({name}, oracle apply_stencil, wall {wall:.1f} s)"}


def run_reference(args) -> dict | None:
    import numpy as np

    world, rank, _ = _dist()
    if rank != 0:
        return None
    np_dtype = np.float64 if args.dtype == "float64" else np.float32
    cores = os.cpu_count() or 1
    vals = []
    for k in range(args.warmup + args.steps):
        cb = cpu_baseline(np_dtype, cores=cores, planes=8, steps=1)
        if k >= args.warmup:
            vals.append(cb["value"])
    value = statistics.median(vals)
    cb["value"] = value
    return {
        "metric": METRIC, "value": value, "unit": "GPts/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(N_INTERIOR ** 3 / (value * 1e9) * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.dtype == "float64" else "f32", "data": "synthetic",
        "impl": "reference",
        "config": {"workload": f"3-D 7-point Laplacian, {N_INTERIOR}^3, {args.dtype}, CPU NumPy "
                               f"oracle on {cores} processes, z-slab samples"},
        "cpu_baseline": cb,
        "e2e": {"value": value, "unit": "GPts/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


# ---------------------------------------------------------------------------
# Batched shallow water: 256 independent 2-D grids, RK2, CFL 0.4, reflective
# ---------------------------------------------------------------------------
SW_GRIDS = 256
SW_STEPS = 200
SW_METRIC = "solves/s (256 batched 2-D shallow-water RK2 solves, 200 steps each)"
SW_BC_ODD = (0, 2, 1)   # hu flips sign across x walls (dim 1), hv across y walls (dim 0)


SW_FIXED_N = 0          # > 0: every grid n x n (small profiling cases)
SW_ZCHUNK = 0           # > 0: rows per batched work item (0: the kernels' default)


def _sw_workload(seed: int = 3):
    """Sizes log-uniform in [64, 2048] and the h-bump initial states (seeded)."""
    import numpy as np

    import stencil_defs as D

    rng = np.random.default_rng(seed)
    sizes = [int(x) for x in np.rint(np.exp(rng.uniform(np.log(64), np.log(2048), SW_GRIDS)))]
    if SW_FIXED_N > 0:
        sizes = [SW_FIXED_N] * SW_GRIDS
    init = [D.sw_init(N, rng, halo=(1, 1), dtype="float64") for N in sizes]
    return sizes, init


def _sw_programs(dtype: str):
    import stencil_defs as D
    from cutile import RKIntegrator, stencil
    from cutile import compile as stencil_compile

    rk = RKIntegrator(stencil(ndim=2, dtype=dtype)(D.sw_rhs), "rk2").compile(
        boundary="reflecting", align_halo=False)
    speed = stencil_compile(stencil(ndim=2, dtype=dtype)(D.sw_speed), reduce="max",
                            align_halo=False)
    return rk, speed


def _sw_batch(dtype: str, sizes, init, device):
    """Row-pitched packed fields, an RKBatch with per-grid CFL dt, and a
    device copy of the initial state for resets."""
    import numpy as np
    import torch

    from cutile.runtime.rk_runtime import RKBatch, pack_grids

    rk, speed = _sw_programs(dtype)
    tdt = torch.float64 if dtype == "float64" else torch.float32
    flat, states = pack_grids([a[0].shape for a in init], 3, tdt, device)
    for st, fields in zip(states, init):
        for dst, src in zip(st, fields):
            dst.copy_(torch.from_numpy(np.ascontiguousarray(src, dtype=np.dtype(dtype))))
    dx = [1.0 / N for N in sizes]
    batch = RKBatch(rk, states, [{"dx": d} for d in dx],
                    cfl=(speed.load_module().program(), dx, 0.4), bc_odd=SW_BC_ODD,
                    zchunk=SW_ZCHUNK or None)
    return batch, flat, flat.clone(), states, (rk, speed)


def _sw_cpu_job(args):
    """One worker: oracle RK2 + CFL steps of one seeded grid; returns
    (seconds, point-steps)."""
    n, steps, seed = args
    import numpy as np

    import stencil_defs as D
    from oracle import stencil_oracle as O

    rng = np.random.default_rng(seed)
    st = tuple(a.astype(np.float32) for a in D.sw_init(n, rng, halo=(1, 1), dtype="float64"))
    names = ["h", "hu", "hv"]
    odd = {1: (1,), 2: (0,)}
    t0 = time.perf_counter()
    for _ in range(steps):
        dt = O.cfl_dt(D.sw_speed, st, names, 2, (1, 1), 0.4, 1.0 / n)
        st = O.rk_step(D.sw_rhs, names, st, "rk2", dt, 2, (1, 1), {"dx": 1.0 / n},
                       "reflecting", odd)
    return time.perf_counter() - t0, n * n * steps


def sw_cpu_baseline(total_point_steps: float, cores: int, n: int = 256, steps: int = 4) -> dict:
    """The oracle (NumPy restatement of the reference's RK stepping around
    apply_stencil) on ``cores`` worker processes, each a seeded n^2 grid;
    solves/s extrapolated from the measured point-steps/s."""
    import multiprocessing as mp

    if cores == 1:
        secs, pts = _sw_cpu_job((n, steps, 0))
        rate, wall = pts / secs, secs
    else:
        ctx = mp.get_context("spawn")
        with ctx.Pool(cores) as pool:
            pool.map(_sw_cpu_job, [(64, 1, k) for k in range(cores)])
            t0 = time.perf_counter()
            res = pool.map(_sw_cpu_job, [(n, steps, k) for k in range(cores)])
            wall = time.perf_counter() - t0
        rate = sum(p for _, p in res) / wall
    solves = SW_GRIDS * rate / total_point_steps
    return {"value": solves, "unit": "solves/s", "cores": cores, "kind": "port",
            "sample": f"{cores} x {steps} RK2+CFL steps of a {n}^2 float32 grid (oracle rk_step, "
                      f"wall {wall:.1f} s), {rate / 1e6:.2f} M point-steps/s extrapolated to the "
                      f"workload's {total_point_steps:.3g} point-steps"}


def run_sw_batch(args) -> dict | None:
    import numpy as np
    import torch

    world, rank, local = _dist()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        torch.distributed.init_process_group("nccl", init_method="env://")
    sizes, init = _sw_workload(seed=3 + rank)
    pts = sum(N * N for N in sizes)
    stream = torch.cuda.current_stream()

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    def timed(fn, steps):
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        barrier()
        ev0.record(stream)
        for _ in range(steps):
            fn()
        ev1.record(stream)
        barrier()
        ms = ev0.elapsed_time(ev1)
        if world > 1:
            ms = _max_over_ranks(ms)
        return ms / steps

    runs = {}
    for dtype in (("float32", "float64") if args.compare else ("float32",)):
        batch, flat, flat0, states, _ = _sw_batch(dtype, sizes, init, dev)
        graph = batch.capture(SW_STEPS)

        def solve_set(flat=flat, flat0=flat0, graph=graph):
            flat.copy_(flat0)
            graph.replay()

        for _ in range(args.warmup):
            solve_set()
        torch.cuda.synchronize()
        if dtype == "float32":
            with ClockSampler(local) as clk:
                ms = timed(solve_set, args.steps)
            clocks = clk.summary()
        else:
            ms = timed(solve_set, max(1, args.steps // 2))
        solve_set()
        torch.cuda.synchronize()
        runs[dtype] = {"ms": ms, "batch": batch, "flat": flat, "flat0": flat0, "graph": graph,
                       "states": states}

    if not args.compare:
        ms32 = runs["float32"]["ms"]
        return {"metric": SW_METRIC, "value": round(SW_GRIDS * world / (ms32 / 1e3), 3),
                "unit": "solves/s", "ms_per_step": round(ms32, 3), "n_gpus": world,
                "config": {"workload": f"{SW_GRIDS} grids, fixed n={SW_FIXED_N}, "
                                       f"{SW_STEPS} RK2 steps (profiling case, no comparison)"},
                "gpu_launches": (1 + SW_STEPS * runs["float32"]["batch"].launches_per_step())
                * args.steps} if rank == 0 else None
    # relative L2 of the FP32 solves against the FP64 solves, per field, worst grid
    rel = [0.0, 0.0, 0.0]
    rel_state = 0.0      # the (h, hu, hv) state vector of a grid
    for a, b in zip(runs["float32"]["states"], runs["float64"]["states"]):
        num = den = 0.0
        for f in range(3):
            ia, ib = a[f][1:-1, 1:-1].double(), b[f][1:-1, 1:-1]
            d2 = float(torch.sum((ia - ib) ** 2))
            n2 = float(torch.sum(ib ** 2))
            num, den = num + d2, den + n2
            if n2 > 0:
                rel[f] = max(rel[f], (d2 / n2) ** 0.5)
        rel_state = max(rel_state, (num / den) ** 0.5)
    ms64 = runs.pop("float64")["ms"]
    torch.cuda.empty_cache()

    # the plain FP64 path: every grid on its own through the drop-in API
    # (one reduction, one dt update and one launch per RK stage, per grid,
    # eagerly), timed on a bounded number of steps and scaled to 200
    rk64, speed64 = _sw_programs("float64")
    prog = rk64.load_module().program()
    prog.bc_odd = SW_BC_ODD
    sp = speed64.load_module().program()
    st64 = [tuple(torch.from_numpy(a).to(dev) for a in g) for g in init]
    n = len(st64)
    smax = torch.zeros(n, dtype=torch.float64, device=dev)
    dts = torch.zeros(n, dtype=torch.float64, device=dev)
    scale = torch.tensor([1.0 / N for N in sizes], dtype=torch.float64, device=dev)
    from cutile.runtime import native

    def plain_step():
        for g, st in enumerate(st64):
            sp.reduce(list(st), out=smax[g])
            native.cfl_update(smax[g:g + 1], scale[g:g + 1], 0.4, dts[g:g + 1], 1e30, stream)
            prog.step(st, dts[g:g + 1], scalars={"dx": 1.0 / sizes[g]})

    plain_steps = 10
    plain_step()
    torch.cuda.synchronize()
    plain_ms = timed(plain_step, plain_steps) * SW_STEPS
    plain_launches = n * (2 + len(prog.table))

    ms32 = runs["float32"]["ms"]
    value = SW_GRIDS * world / (ms32 / 1e3)
    b32 = runs["float32"]["batch"]
    launches = 1 + SW_STEPS * b32.launches_per_step()

    # roofline of the FP32 batched step: algorithmic bytes per RK2 step =
    # 15 field transfers (stage 1: 3 in + 3 out; stage 2: 6 in + 3 out) plus
    # the CFL reduction's 3 reads, 4 B each, per interior point
    alg_bytes = 18 * 4 * pts
    step_ms = ms32 / SW_STEPS
    achieved = alg_bytes / (step_ms / 1e3) / 1e9
    peak, peak_kind = _peaks()

    # end-to-end: pinned host state -> device, 200 graph steps, result -> host
    flat, graph = runs["float32"]["flat"], runs["float32"]["graph"]
    host_in = runs["float32"]["flat0"].cpu().pin_memory()
    host_out = torch.empty_like(host_in).pin_memory()

    def e2e_set():
        flat.copy_(host_in, non_blocking=True)
        graph.replay()
        host_out.copy_(flat, non_blocking=True)

    e2e_set()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e2e_ms = timed(e2e_set, 2)
    e2e_ms = max(e2e_ms, (time.perf_counter() - t0) * 1e3 / 2)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = sw_cpu_baseline(float(pts) * SW_STEPS, os.cpu_count() or 1)
    line = {
        "metric": SW_METRIC, "value": round(value, 3), "unit": "solves/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms32, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 (FP64 RK combination)", "data": "synthetic",
        "config": {"workload": "256 shallow-water grids (h, hu, hv; Rusanov fluxes; g=9.81), N "
                               "log-uniform in [64, 2048] (seed 3), h = 1 + 0.1 Gaussian bump, "
                               "RK2 with FP64 stage combination, CFL 0.4 per grid on the device, "
                               "reflective walls fused into staging; one step = reset from the "
                               "resident initial state + 200 RK2 steps replayed from one CUDA "
                               "graph (one persistent launch per stage over all grids)",
                   "grids": SW_GRIDS, "interior_points": pts, "rk_steps": SW_STEPS,
                   "l2": f"fields {flat.numel() * 4 / 1e9:.2f} GB >> 126 MB L2, no flush",
                   "parallelism": f"replicas{world}"},
        "comparison": {
            "fp64_batched_solves_s": round(SW_GRIDS * world / (ms64 / 1e3), 3),
            "fp64_plain_solves_s": round(SW_GRIDS * world / (plain_ms / 1e3), 3),
            "speedup_vs_fp64_plain": round(plain_ms / ms32, 3),
            "speedup_vs_fp64_batched": round(ms64 / ms32, 3),
            "fp64_plain": f"per grid and step: reduce + dt update + {len(prog.table)} stage "
                          f"launches through the drop-in API ({plain_launches} launches per "
                          f"step), eager; timed over {plain_steps} steps, scaled to "
                          f"{SW_STEPS}",
            "rel_l2_fp32_vs_fp64": {"state": rel_state, "h": rel[0], "hu": rel[1],
                                    "hv": rel[2],
                                    "over": "interiors after 200 steps, worst grid; 'state' "
                                            "is the (h, hu, hv) vector"},
        },
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                     "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": None,
                     "peak_kind": peak_kind, "kernel": "whole RK2 step (4 launches)",
                     "algorithmic_bytes_per_step": alg_bytes},
        "e2e": {"value": round(SW_GRIDS * world / (e2e_ms / 1e3), 3), "unit": "solves/s",
                "h2d_bytes_per_step": int(host_in.numel() * 4),
                "d2h_bytes_per_step": int(host_out.numel() * 4),
                "step": "H2D of all fields, 200-step graph replay, D2H of all fields"},
        "gpu_launches": launches * args.steps,
        "clocks": clocks,
        "cpu_baseline": cpu,
    }
    del runs
    if world > 1:
        torch.distributed.destroy_process_group()
    return line if rank == 0 else None


# ---------------------------------------------------------------------------
# Gray-Scott: 4096^2 periodic, fused u/v kernel, FP64 vs FP32 vs FP32+Kahan
# ---------------------------------------------------------------------------
GS_N = 4096
GS_STEPS = 10000
GS_METRIC = "GPts/s (2-D Gray-Scott 4096^2 periodic, fused u/v step, FP32 + Kahan)"


def _gs_fused(precision: str):
    import cutile
    import stencil_defs as D
    from cutile import stencil

    return cutile.compile_fused([stencil(ndim=2)(D.gs_u), stencil(ndim=2)(D.gs_v)],
                                precision=precision, boundary="periodic")


def _gs_cpu_job(args):
    n, steps, seed = args
    import numpy as np

    import stencil_defs as D
    from oracle import stencil_oracle as O

    u, v = D.gray_scott_init(n, seed=seed, halo=(1, 1))
    t0 = time.perf_counter()
    for _ in range(steps):
        u, v = (O.stencil_with_boundary([u, v], D.gs_u, 2, (1, 1), "periodic"),
                O.stencil_with_boundary([u, v], D.gs_v, 2, (1, 1), "periodic"))
    return time.perf_counter() - t0, n * n * steps


def gs_cpu_baseline(cores: int, n: int = 1024, steps: int = 3) -> dict:
    """The oracle (NumPy restatement of apply_boundary + apply_stencil for
    both fields) on ``cores`` processes, each a seeded n^2 periodic grid."""
    import multiprocessing as mp

    if cores == 1:
        secs, pts = _gs_cpu_job((n, steps, 2))
        rate, wall = pts / secs, secs
    else:
        ctx = mp.get_context("spawn")
        with ctx.Pool(cores) as pool:
            pool.map(_gs_cpu_job, [(64, 1, k) for k in range(cores)])
            t0 = time.perf_counter()
            res = pool.map(_gs_cpu_job, [(n, steps, 2 + k) for k in range(cores)])
            wall = time.perf_counter() - t0
        rate = sum(p for _, p in res) / wall
    return {"value": round(rate / 1e9, 5), "unit": "GPts/s", "cores": cores, "kind": "port",
            "sample": f"{cores} x {steps} fused u/v steps of a {n}^2 periodic float64 grid "
                      f"(oracle stencil_with_boundary, wall {wall:.1f} s)"}


def run_gray_scott(args) -> dict | None:
    import numpy as np
    import torch

    import stencil_defs as D

    world, rank, local = _dist()
    torch.cuda.set_device(local)
    if world > 1:
        torch.distributed.init_process_group("nccl", init_method="env://")
    stream = torch.cuda.current_stream()
    steps = args.steps

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    runs = {}
    for prec in ("fp64", "fp32", "fp32_kahan"):
        r = _gs_fused(prec)
        h = r.halo_widths
        dtype = "float64" if prec == "fp64" else "float32"
        u0, v0 = D.gray_scott_init(GS_N, seed=2 + rank, halo=h, dtype=dtype)
        step = getattr(r.load_module(), f"step_{r.name}")
        a = [torch.from_numpy(u0).cuda(), torch.from_numpy(v0).cuda()]
        b = [torch.zeros_like(a[0]), torch.zeros_like(a[1])]
        kahan = prec == "fp32_kahan"
        ca = [torch.zeros_like(a[0]), torch.zeros_like(a[1])] if kahan else []
        cb = [torch.zeros_like(a[0]), torch.zeros_like(a[1])] if kahan else []
        init = [x.clone() for x in a]
        # the time loop is replayed from a CUDA graph of `chunk` fused steps
        # (ping-pong, so the state returns to `a` after each replay)
        prog = r.load_module().program()
        chunk = 100 if steps % 100 == 0 else (2 if steps % 2 == 0 else 0)
        graph = prog.capture_steps(a + ca, b + cb, chunk, boundary=True) if chunk else None

        def run(n):
            nonlocal a, b, ca, cb
            if graph is not None and n % chunk == 0:
                for _ in range(n // chunk):
                    graph.replay()
                return
            for _ in range(n):
                if kahan:
                    step(*a, *ca, *b, *cb)
                    ca, cb = cb, ca
                else:
                    step(*a, *b)
                a, b = b, a

        run(chunk if graph is not None else args.warmup)
        for x, y in zip(a, init):
            x.copy_(y)
        for c in ca:
            c.zero_()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        if prec == "fp32_kahan":
            clk = ClockSampler(local).__enter__()
        barrier()
        ev0.record(stream)
        run(steps)
        ev1.record(stream)
        barrier()
        if prec == "fp32_kahan":
            clk.__exit__(None, None, None)
            clocks = clk.summary()
        ms = ev0.elapsed_time(ev1)
        if world > 1:
            ms = _max_over_ranks(ms)
        inner = tuple(slice(x, sz - x) for x, sz in zip(h, u0.shape))
        runs[prec] = {"ms": ms, "u": a[0][inner].double(), "v": a[1][inner].double(),
                      "itemsize": np.dtype(dtype).itemsize, "h": h, "step": step,
                      "state": (a, ca), "init": init, "graph": graph, "chunk": chunk}

    def rel(x, y):
        return float(torch.linalg.norm(x - y) / torch.linalg.norm(y))

    ref = runs["fp64"]
    err = {p: {"u": rel(runs[p]["u"], ref["u"]), "v": rel(runs[p]["v"], ref["v"])}
           for p in ("fp32", "fp32_kahan")}
    npts = GS_N * GS_N
    gpts = {p: npts * steps / (runs[p]["ms"] / 1e3) / 1e9 * world for p in runs}
    k = runs["fp32_kahan"]
    ms_step = k["ms"] / steps
    # algorithmic bytes per launch: u, v, c_u, c_v read once and written once
    alg_bytes = 8 * 4 * npts
    achieved = alg_bytes / (ms_step / 1e3) / 1e9
    peak, peak_kind = _peaks()

    # end-to-end through the public step function: pinned host u, v (and
    # zero compensation) -> device, the whole solve, u, v -> host
    (a, ca), init = k["state"], k["init"]
    host_in = [x.cpu().pin_memory() for x in init]
    host_out = [torch.empty_like(x).pin_memory() for x in host_in]
    e2e_steps = min(steps, 1000)
    step = k["step"]
    graph, chunk = k["graph"], k["chunk"]
    b = [torch.zeros_like(a[0]), torch.zeros_like(a[1])]
    cb = [torch.zeros_like(a[0]), torch.zeros_like(a[1])]
    barrier()
    t0 = time.perf_counter()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for x, y in zip(a, host_in):
        x.copy_(y, non_blocking=True)
    for c in ca:
        c.zero_()
    if graph is not None and e2e_steps % chunk == 0:
        for _ in range(e2e_steps // chunk):
            graph.replay()
    else:
        for _ in range(e2e_steps):
            step(*a, *ca, *b, *cb)
            a, b, ca, cb = b, a, cb, ca
    for x, y in zip(host_out, a):
        x.copy_(y, non_blocking=True)
    e1.record(stream)
    barrier()
    e2e_ms = max(e0.elapsed_time(e1), (time.perf_counter() - t0) * 1e3)
    e2e = npts * e2e_steps / (e2e_ms / 1e3) / 1e9 * world

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = gs_cpu_baseline(os.cpu_count() or 1)
    line = {
        "metric": GS_METRIC, "value": round(gpts["fp32_kahan"], 3), "unit": "GPts/s",
        "n_gpus": world, "steps": steps, "warmup": args.warmup, "ms_per_step": round(ms_step, 5),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 + f32 compensation", "data": "synthetic",
        "config": {"workload": f"Gray-Scott u/v, Du=0.16 Dv=0.08 F=0.037 k=0.06 dt=1, {GS_N}^2 "
                               f"periodic (fused into staging), u=1 v=0 plus 20 noisy 32^2 "
                               f"squares (seed 2); one step = one compile_fused launch of both "
                               f"fields with Kahan-compensated updates; {steps} steps from the "
                               f"initial state",
                   "l2": "fields 4 x 67 MB + outputs > 126 MB L2",
                   "parallelism": f"replicas{world}"},
        "comparison": {
            "fp64_gpts": round(gpts["fp64"], 3), "fp32_gpts": round(gpts["fp32"], 3),
            "fp32_kahan_gpts": round(gpts["fp32_kahan"], 3),
            "rel_l2_vs_fp64_after_steps": err,
            "oracle": "the GPU FP64 path, bit-exact to the NumPy oracle on 50-step runs of "
                      "the same stencils (parity tests)"},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": None, "peak_kind": peak_kind,
                     "kernel": "fused u/v Kahan step",
                     "algorithmic_bytes_per_launch": alg_bytes},
        "e2e": {"value": round(e2e, 3), "unit": "GPts/s",
                "h2d_bytes_per_step": int(sum(x.numel() * 4 for x in host_in)),
                "d2h_bytes_per_step": int(sum(x.numel() * 4 for x in host_out)),
                "step": f"H2D of u, v; {e2e_steps} Kahan steps (graph replays); D2H of u, v"},
        "gpu_launches": steps,
        "clocks": clocks,
        "cpu_baseline": cpu,
    }
    if world > 1:
        torch.distributed.destroy_process_group()
    return line if rank == 0 else None


# ---------------------------------------------------------------------------
# Small-step heat diffusion: where the compensated FP32 update pays
# ---------------------------------------------------------------------------
HEAT_METRIC = "GPts/s (2-D heat, small step, FP32 + Kahan)"


def run_heat_kahan(args) -> dict | None:
    """2-D heat u += 0.02 * lap(u), 4096^2, zero Dirichlet halo, u = 1 + 0.1
    * Gaussian bump: every update is ~1e-8..1e-4 of u, below FP32's rounding
    of u in most of the field.  FP64, FP32 and FP32+Kahan run the same steps
    from the same start; the line reports the Kahan kernel's throughput and
    each FP32 mode's relative L2 error against FP64."""
    import numpy as np
    import torch

    import cutile
    import stencil_defs as D
    from cutile import stencil

    world, rank, local = _dist()
    torch.cuda.set_device(local)
    n, steps = GS_N, args.steps
    chain = 4
    steps = max(chain, steps // chain * chain)
    stream = torch.cuda.current_stream()
    runs = {}
    # (name, precision, steps per launch): the chained runs keep the field
    # (and for Kahan its compensation) in shared memory for `chain` steps
    for name, prec, T in (("fp64", "fp64", 1), ("fp32", "fp32", 1), ("fp32_kahan", "fp32_kahan", 1),
                          ("fp64_T4", "fp64", chain), ("fp32_kahan_T4", "fp32_kahan", chain)):
        dt = "float64" if prec == "fp64" else "float32"
        r = cutile.compile(stencil(ndim=2, dtype=dt)(D.heat_small_dt), precision=prec,
                           temporal_steps=T, temporal_blocking=T > 1)
        assert r.temporal_steps == T
        h = r.halo_widths
        u0 = D.heat_bump_init(n, halo=h, dtype=dt)
        launch = getattr(r.load_module(), f"launch_{r.name}")
        a = torch.from_numpy(u0).cuda()
        b = torch.zeros_like(a)
        ca, cb = torch.zeros_like(a), torch.zeros_like(a)
        kahan = prec == "fp32_kahan"
        for _ in range(args.warmup):
            launch(a, ca, b, cb) if kahan else launch(a, b)
        a.copy_(torch.from_numpy(u0))
        ca.zero_()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        clk = ClockSampler(local).__enter__() if name == "fp32_kahan" else None
        e0.record(stream)
        for _ in range(steps // T):
            if kahan:
                launch(a, ca, b, cb)
                ca, cb = cb, ca
            else:
                launch(a, b)
            a, b = b, a
        e1.record(stream)
        torch.cuda.synchronize()
        clocks = None
        if clk is not None:
            clk.__exit__(None, None, None)
            clocks = clk.summary()
        inner = tuple(slice(x, sz - x) for x, sz in zip(h, u0.shape))
        runs[name] = {"ms": e0.elapsed_time(e1), "u": a[inner].double(), "clocks": clocks, "T": T}
        del a, b, ca, cb

    def rel(x, y):
        return float(torch.linalg.norm(x - y) / torch.linalg.norm(y))

    ref = runs["fp64"]["u"]
    err = {p: rel(runs[p]["u"], ref) for p in ("fp32", "fp32_kahan", "fp32_kahan_T4", "fp64_T4")}
    npts = n * n
    gpts = {p: npts * steps / (runs[p]["ms"] / 1e3) / 1e9 for p in runs}
    best = "fp32_kahan"
    ms_launch = runs[best]["ms"] / steps
    alg = 4 * 4 * npts     # u, c read and written once per launch, FP32
    peak, peak_kind = _peaks()
    line = {
        "metric": HEAT_METRIC, "value": round(gpts[best], 3), "unit": "GPts/s",
        "n_gpus": 1, "steps": steps, "warmup": args.warmup,
        "ms_per_step": round(runs[best]["ms"] / steps, 5),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 + f32 compensation", "data": "synthetic",
        "config": {"workload": f"2-D heat u + 0.02*(N+S+W+E-4u), {n}^2, zero Dirichlet halo, "
                               f"u = 1 + 0.1*Gaussian bump (width 0.08); {steps} steps from the "
                               f"initial state; value: FP32+Kahan one step per launch, compared "
                               f"with FP64 / FP32 and with FP64 and FP32+Kahan at {chain} steps "
                               f"chained per launch (u and its compensation kept in shared "
                               f"memory); the 4096^2 fields partly stay in the 126 MB L2 between "
                               f"steps, which the one-step runs profit from",
                   "temporal_steps": 1},
        "comparison": {**{f"{p}_gpts": round(gpts[p], 3) for p in runs},
                       "rel_l2_vs_fp64_after_steps": err,
                       "bytes_per_point_step": {"fp64": 16, "fp32": 8, "fp32_kahan": 32,
                                                "fp64_T4": 16 / chain, "fp32_kahan_T4": 32 / chain}},
        "roofline": {"bound": "hbm", "achieved": round(alg / (ms_launch / 1e3) / 1e9, 1),
                     "peak": peak, "unit": "GB/s",
                     "frac": round(alg / (ms_launch / 1e3) / 1e9 / peak, 4), "traffic": None,
                     "peak_kind": peak_kind, "algorithmic_bytes_per_launch": alg,
                     "kernel": "Kahan heat step, one step per launch"},
        "gpu_launches": steps, "clocks": runs[best]["clocks"], "cpu_baseline": None,
    }
    return line if rank == 0 else None


def run_gs_reference(args) -> dict | None:
    world, rank, _ = _dist()
    if rank != 0:
        return None
    cores = os.cpu_count() or 1
    vals = []
    for k in range(args.warmup + args.steps):
        cb = gs_cpu_baseline(cores, n=512, steps=1)
        if k >= args.warmup:
            vals.append(cb["value"])
    value = statistics.median(vals)
    cb["value"] = value
    return {
        "metric": GS_METRIC, "value": value, "unit": "GPts/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(GS_N * GS_N / (value * 1e9) * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic", "impl": "reference",
        "config": {"workload": f"Gray-Scott {GS_N}^2 periodic fused u/v step, CPU NumPy oracle "
                               f"on {cores} processes, 512^2 samples"},
        "cpu_baseline": cb,
        "e2e": {"value": value, "unit": "GPts/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


# ---------------------------------------------------------------------------
# Serving: Poisson stream of mixed solves, continuous batching, 150 GB budget
# ---------------------------------------------------------------------------
SERVE_REQUESTS = 2000
SERVE_RATE = 2000.0
SERVE_BUDGET = 150e9
SERVE_METRIC = "solves/s (continuous-batching server, Poisson 2000 req/s mixed stencil solves)"


def _serve_workload(n: int, rate: float = SERVE_RATE, seed: int = 4, host_init: bool = False):
    """Seeded request stream: kinds uniform over heat 5-pt / upwind advection /
    leapfrog wave / 3-D 7-pt, N log-uniform (2-D 64..4096, 3-D 32..256),
    steps log-uniform 10..1000, float32/float64 50/50, Uniform[0,1) interiors."""
    import numpy as np

    import stencil_defs as D
    from cutile.runtime.serving import SolveRequest

    rng = np.random.default_rng(seed)
    names = list(D.SERVE_KINDS)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, n))
    kind_idx = rng.integers(0, len(names), n)
    n2 = np.exp(rng.uniform(np.log(64), np.log(4096), n))
    n3 = np.exp(rng.uniform(np.log(32), np.log(256), n))
    steps = np.rint(np.exp(rng.uniform(np.log(10), np.log(1000), n))).astype(int)
    dts = rng.integers(0, 2, n)
    reqs = []
    for i in range(n):
        kind = names[int(kind_idx[i])]
        ndim, nstate = D.SERVE_KINDS[kind][1], D.SERVE_KINDS[kind][2]
        m = int(round(n3[i] if ndim == 3 else n2[i]))
        shape = (m + 2,) * ndim
        dtype = ("float32", "float64")[int(dts[i])]
        init = None
        if host_init:
            r = np.random.default_rng(4000 + i)
            u = np.zeros(shape, dtype=dtype)
            u[(slice(1, -1),) * ndim] = r.random((m,) * ndim, dtype=np.float64).astype(dtype)
            init = (u,) * nstate
        reqs.append(SolveRequest(kind, dtype, shape, int(steps[i]), arrival=float(arrivals[i]),
                                 init=init, seed=4000 + i, rid=i))
    return reqs


def _serve_point_steps(reqs) -> float:
    tot = 0.0
    for r in reqs:
        pts = 1
        for x in r.shape:
            pts *= x - 2
        tot += pts * r.steps
    return tot


def _timeline(trace, parts: int = 10):
    """Iterations and mean active solves in each tenth of the run."""
    if not trace:
        return []
    end = trace[-1][0]
    out = []
    for k in range(parts):
        lo, hi = end * k / parts, end * (k + 1) / parts
        seg = [t for t in trace if lo <= t[0] < hi or (k == parts - 1 and t[0] == end)]
        out.append([round(hi, 2), len(seg),
                    round(sum(t[1] for t in seg) / len(seg), 1) if seg else 0])
    return out


def run_serve(args) -> dict | None:
    import numpy as np
    import torch

    import stencil_defs as D
    from cutile.runtime.serving import StencilServer, percentile

    world, rank, local = _dist()
    torch.cuda.set_device(local)
    if world > 1:
        torch.distributed.init_process_group("nccl", init_method="env://")
    kinds = D.serving_kinds()
    server = StencilServer(kinds, budget_bytes=SERVE_BUDGET)
    # warm-up: every (kind, dtype) program loaded and launched
    warm = _serve_workload(8 * max(1, args.warmup), seed=99)
    for r in warm:
        r.steps = 3
        r.shape = tuple(min(x, 66) for x in r.shape)
    server.run(warm, realtime=False, keep_state=False)
    torch.cuda.synchronize()

    reqs = _serve_workload(SERVE_REQUESTS, seed=4 + rank)
    server.stats = type(server.stats)()
    if world > 1:
        torch.distributed.barrier()
    with ClockSampler(local) as clk:
        res = server.run(reqs, realtime=True, keep_state=False)
        torch.cuda.synchronize()
    clocks = clk.summary()
    st = server.stats
    server.stats = type(st)()
    done = [r for r in res if r.error is None]
    lat = [r.latency * 1e3 for r in done]
    span = max(r.completed for r in done) - min(r.arrival for r in reqs)
    solves_s = len(done) / span
    if world > 1:
        solves_s = len(done) * world / _max_over_ranks(span)
    gpts = _serve_point_steps([r for r in reqs]) / span / 1e9

    # the same mix at an arrival rate the server sustains (half its measured
    # throughput), so that p50/p99 describe the server rather than a queue
    # that grows for the whole run
    sus_rate = max(50.0, 0.5 * solves_s)
    sus_reqs = _serve_workload(max(200, SERVE_REQUESTS // 2), rate=sus_rate, seed=40 + rank)
    sus_res = server.run(sus_reqs, realtime=True, keep_state=False)
    torch.cuda.synchronize()
    server.stats = type(server.stats)()
    sus_done = [r for r in sus_res if r.error is None]
    sus_lat = [r.latency * 1e3 for r in sus_done]
    sus_span = max(r.completed for r in sus_done) - min(r.arrival for r in sus_reqs)
    sustained = {"rate_req_s": round(sus_rate, 1), "requests": len(sus_reqs),
                 "solves_s": round(len(sus_done) / sus_span, 3),
                 "latency_ms": {"p50": round(percentile(sus_lat, 50), 3),
                                "p99": round(percentile(sus_lat, 99), 3),
                                "mean": round(float(np.mean(sus_lat)), 3)},
                 "note": "Poisson arrivals at half the throughput measured under the "
                         f"{SERVE_RATE:.0f} req/s stream (seed 40), same request mix"}

    # each request alone on the plain path (drop-in launch per step), sampled
    rng = np.random.default_rng(7)
    sample = sorted(rng.choice(len(reqs), size=min(64, len(reqs)), replace=False).tolist())
    alone_ms = []
    for i in sample:
        _, ms = server.run_alone(reqs[i])
        alone_ms.append(ms)
    alone_mean = float(np.mean(alone_ms))
    # sequential FIFO on the plain path: request k completes after the
    # alone times of requests 0..k (sample mean), or its arrival, whichever
    # is later
    seq_lat, t_free = [], 0.0
    for r in reqs:
        start = max(t_free, r.arrival)
        t_free = start + alone_mean / 1e3
        seq_lat.append((t_free - r.arrival) * 1e3)

    # end to end: the first 200 requests with host-side initial fields
    # (copied in at admission) and every result read back to the host
    e2e_reqs = _serve_workload(200, seed=4 + rank, host_init=True)
    for r in e2e_reqs:
        r.init = tuple(torch.from_numpy(a).pin_memory() for a in r.init)
    h2d = sum(a.numel() * a.element_size() for r in e2e_reqs for a in r.init)
    host_out = [tuple(torch.empty(r.shape, dtype=getattr(torch, r.dtype), pin_memory=True)
                      for _ in range(D.SERVE_KINDS[r.kind][2])) for r in e2e_reqs]
    t0 = time.perf_counter()
    eres = server.run(e2e_reqs, realtime=True, keep_state=True)
    for r, o in zip(eres, host_out):
        for dst, src in zip(o, r.state):
            dst.copy_(src, non_blocking=True)
    torch.cuda.synchronize()
    e2e_span = time.perf_counter() - t0
    d2h = sum(t.numel() * t.element_size() for o in host_out for t in o)
    del eres, host_out

    line = {
        "metric": SERVE_METRIC, "value": round(solves_s, 3), "unit": "solves/s",
        "n_gpus": world, "steps": len(reqs), "warmup": args.warmup,
        "ms_per_step": round(span * 1e3 / len(reqs), 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32/f64 mix", "data": "synthetic",
        "config": {"workload": f"{len(reqs)} requests, Poisson arrivals at {SERVE_RATE:.0f}/s "
                               f"(seed 4): heat 5-pt, upwind advection (1, 0.5), leapfrog wave "
                               f"c=1, 3-D 7-pt; 2-D N log-uniform 64..4096, 3-D 32..256; steps "
                               f"log-uniform 10..1000; float32/float64 50/50; Uniform[0,1) "
                               f"interiors generated on the device; zero Dirichlet halo; "
                               f"HBM admission budget {SERVE_BUDGET / 1e9:.0f} GB; a step is one "
                               f"request",
                   "l2": "working set >> 126 MB L2",
                   "parallelism": f"replicas{world}"},
        "latency_ms": {"p50": round(percentile(lat, 50), 3), "p99": round(percentile(lat, 99), 3),
                       "mean": round(float(np.mean(lat)), 3)},
        "comparison": {
            "sustained_rate": sustained,
            "alone_plain_solves_s": round(1e3 / alone_mean, 3),
            "speedup_vs_alone_plain": round(solves_s / (1e3 / alone_mean), 3),
            "alone_sequential_latency_ms": {"p50": round(percentile(seq_lat, 50), 3),
                                            "p99": round(percentile(seq_lat, 99), 3)},
            "alone": f"each request by itself, one launch_<name> per step on C-contiguous "
                     f"fields, device time of {len(sample)} sampled requests (mean "
                     f"{alone_mean:.3f} ms); sequential latencies assume FIFO on one GPU",
            "gpts_served": round(gpts, 3),
            "server": {"iterations": st.iterations, "launches": st.launches,
                       "host_issue_s": round(st.host_s, 3), "gpu_wait_s": round(st.wait_s, 3),
                       "admit_s": round(st.admit_s, 3), "timeline": _timeline(st.trace),
                       "max_active": st.max_active, "peak_gb": round(st.peak_bytes / 1e9, 3),
                       "rejected": st.rejected, "wall_s": round(st.wall, 3)},
        },
        "roofline": None,
        "e2e": {"value": round(len(e2e_reqs) / e2e_span, 3), "unit": "solves/s",
                "h2d_bytes_per_step": int(h2d / len(e2e_reqs)),
                "d2h_bytes_per_step": int(d2h / len(e2e_reqs)),
                "step": "one request: pinned host fields copied in at admission, result read "
                        "back after the run (first 200 requests of the stream)"},
        "gpu_launches": st.launches,
        "clocks": clocks,
        "cpu_baseline": None,
    }
    if world > 1:
        torch.distributed.destroy_process_group()
    return line if rank == 0 else None


# ---------------------------------------------------------------------------
# Wide tier: 27- and 125-point boxes at 512^3, eight-in/five-out fused update
# ---------------------------------------------------------------------------
WIDE_METRIC = "GPts/s (3-D 125-point box 512^3 sweep, FP64)"


def _time_launches(launch, steps: int, warmup: int) -> float:
    import torch

    for _ in range(warmup):
        launch()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        launch()
    e1.record()
    e1.synchronize()
    return e0.elapsed_time(e1) / steps


def _wide_cpu_job(args):
    """The oracle on a slab of the reference's box125 (radius 2) or box27."""
    radius, nz, steps = args
    import numpy as np

    import ref_corpus
    from oracle import stencil_oracle as O

    key = "wide_stencils/box125" if radius == 2 else "wide_stencils/box27"
    entries, _ = ref_corpus.load()
    with tempfile.TemporaryDirectory() as tmp:
        fn = ref_corpus.build(tmp, key, entries[key])
    u = np.random.default_rng(1).standard_normal((nz + 2 * radius, 512 + 2 * radius,
                                                  512 + 2 * radius))
    t0 = time.perf_counter()
    for _ in range(steps):
        O.apply_stencil(u, fn, 3, (radius,) * 3)
    return time.perf_counter() - t0, nz * 512 * 512 * steps


def run_wide(args) -> dict | None:
    import numpy as np
    import torch

    import wide_defs as W
    from cutile import compile as stencil_compile
    from cutile import compile_fused, stencil

    import ref_corpus

    world, rank, local = _dist()
    torch.cuda.set_device(local)
    res = {}
    nb = N_INTERIOR
    entries, _ = ref_corpus.load()
    with ClockSampler(local) as clk, tempfile.TemporaryDirectory() as tmp:
        # the reference's own published wide-tier stencils (its
        # tests/wide_stencils.py box125 and box27, README benchmark set),
        # loaded from the parity corpus fixture
        for name in ("box125", "box27"):
            key = f"wide_stencils/{name}"
            r = stencil_compile(ref_corpus.build(tmp, key, entries[key]), temporal_blocking=False)
            h = r.halo_widths
            shape = tuple(nb + 2 * x for x in h)
            a = torch.zeros(shape, dtype=torch.float64, device="cuda")
            inner = tuple(slice(x, s - x) for x, s in zip(h, shape))
            a[inner] = torch.randn((nb,) * 3, dtype=torch.float64, device="cuda")
            b = torch.zeros_like(a)
            launch = getattr(r.load_module(), f"launch_{r.name}")
            ms = _time_launches(lambda: launch(a, b), args.steps, args.warmup)
            res[name] = {"ms": ms, "gpts": nb ** 3 / ms / 1e6, "tile": list(r.tile_sizes),
                         "hints": r.kernel_hints}
            del a, b
        n = 320
        rc = compile_fused([stencil(ndim=3)(f) for f in W.CNS_MEMBERS], temporal_steps=1)
        h = rc.halo_widths
        fields = W.cns_init(n, halo=h)
        ins = [torch.from_numpy(fields[k]).cuda() for k in rc.inputs]
        outs = [torch.zeros_like(ins[0]) for _ in W.CNS_MEMBERS]
        launch = getattr(rc.load_module(), f"launch_{rc.name}")
        ms = _time_launches(lambda: launch(*ins, *outs), max(3, args.steps // 2), args.warmup)
        res["cns"] = {"ms": ms, "gpts": n ** 3 / ms / 1e6, "tile": list(rc.tile_sizes)}
    clocks = clk.summary()
    peak, peak_kind = _peaks()
    box = res["box125"]
    alg = 2 * 8 * nb ** 3
    achieved = alg / (box["ms"] / 1e3) / 1e9
    cpu = None
    if rank == 0 and not args.no_cpu:
        secs, pts = _wide_cpu_job((2, 8, 1))
        cpu = {"value": round(pts / secs / 1e9, 6), "unit": "GPts/s", "cores": 1, "kind": "port",
               "sample": f"1 sweep of an 8x512x512 slab, oracle apply_stencil, {secs:.1f} s"}
    cns_bytes = (8 + 5) * 8 * n ** 3
    line = {
        "metric": WIDE_METRIC, "value": round(box["gpts"], 3), "unit": "GPts/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(box["ms"], 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": f"the reference's box125 (tests/wide_stencils.py: 125 loads, "
                               f"coefficients by distance class, terms grouped by class), {nb}^3 "
                               f"interior, FP64, halo (2, 2, 16), N(0,1) interior; one sweep per "
                               f"step",
                   "tile": box["tile"], "hints": box["hints"], "parallelism": f"replicas{world}",
                   "l2": "arrays >> 126 MB L2"},
        "comparison": {
            "box27_gpts": round(res["box27"]["gpts"], 3),
            "box27_hbm_frac": round(2 * 8 * nb ** 3 / (res["box27"]["ms"] / 1e3) / 1e9 / peak, 4),
            "box27_tile": res["box27"]["tile"], "box27_hints": res["box27"]["hints"],
            "cns_8in_5out_gpts": round(res["cns"]["gpts"], 3),
            "cns_hbm_frac": round(cns_bytes / (res["cns"]["ms"] / 1e3) / 1e9 / peak, 4),
            "cns": f"compile_fused of 5 members over 8 fields, {n}^3 FP64, "
                   f"{cns_bytes / 1e9:.2f} GB algorithmic per launch"},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": None, "peak_kind": peak_kind,
                     "algorithmic_bytes_per_launch": alg},
        "e2e": None, "gpu_launches": args.steps, "clocks": clocks, "cpu_baseline": cpu,
    }
    return line if rank == 0 else None


def run_sw_reference(args) -> dict | None:
    world, rank, _ = _dist()
    if rank != 0:
        return None
    sizes, _ = _sw_workload()
    pts = float(sum(N * N for N in sizes)) * SW_STEPS
    cores = os.cpu_count() or 1
    vals = []
    for k in range(args.warmup + args.steps):
        cb = sw_cpu_baseline(pts, cores, n=128, steps=2)
        if k >= args.warmup:
            vals.append(cb["value"])
    value = statistics.median(vals)
    cb["value"] = value
    return {
        "metric": SW_METRIC, "value": value, "unit": "solves/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(SW_GRIDS / value * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic", "impl": "reference",
        "config": {"workload": f"256 shallow-water grids, RK2 + CFL, CPU NumPy oracle on {cores} "
                               f"processes, sampled grids extrapolated"},
        "cpu_baseline": cb,
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


# Secondary workloads the default run reports beside the headline: each runs
# as its own `bench.py` process (its own memory, its own clock samples) and
# contributes a compact summary of its JSON line under "secondary".
SECONDARY = (
    ("lap7_fp32", ["--dtype", "float32", "--steps", "100"]),
    ("lap7_fp64_T2", ["--temporal", "2", "--steps", "50"]),
    ("lap7_fp64_T4", ["--temporal", "4", "--steps", "25"]),
    ("lap7_fp64_T8", ["--temporal", "8", "--steps", "10"]),
    ("lap7_fp32_T2", ["--dtype", "float32", "--temporal", "2", "--steps", "50"]),
    ("lap7_fp32_T4", ["--dtype", "float32", "--temporal", "4", "--steps", "25"]),
    ("lap7_fp32_T8", ["--dtype", "float32", "--temporal", "8", "--steps", "10"]),
    ("lap7_fp64_bricked8", ["--layout", "bricked", "--steps", "50"]),
    ("gray_scott_4096_kahan", ["--workload", "gray_scott", "--steps", "1000"]),
    ("heat_4096_small_step_kahan", ["--workload", "heat_kahan", "--steps", "2000"]),
    ("sw_batch_256", ["--workload", "sw_batch"]),
    ("wide", ["--workload", "wide"]),
    ("serve", ["--workload", "serve"]),
)
_SUMMARY_KEYS = ("metric", "value", "unit", "steps", "ms_per_step", "dtype", "latency_ms",
                 "comparison")


def _summary(line: dict) -> dict:
    """The figures of a workload line worth carrying beside the headline."""
    out = {k: line[k] for k in _SUMMARY_KEYS if k in line}
    server = (out.get("comparison") or {}).get("server")
    if isinstance(server, dict):
        out["comparison"] = dict(out["comparison"],
                                 server={k: v for k, v in server.items() if k != "timeline"})
    cfg = line.get("config") or {}
    out["workload"] = cfg.get("workload")
    for k in ("temporal_steps", "tile", "layout"):
        if k in cfg:
            out[k] = cfg[k]
    rf = line.get("roofline")
    if rf:
        out["roofline"] = {k: rf.get(k) for k in ("bound", "achieved", "peak", "unit", "frac",
                                                 "traffic", "algorithmic_bytes_per_launch")
                           if k in rf}
    if line.get("e2e"):
        out["e2e"] = {"value": line["e2e"].get("value"), "unit": line["e2e"].get("unit")}
    if line.get("clocks"):
        c = line["clocks"]
        out["clocks"] = {k: c.get(k) for k in ("sm_mhz", "sm_max_mhz", "reasons")}
    if line.get("gpu_launches") is not None:
        out["gpu_launches"] = line["gpu_launches"]
    return out


def run_secondary(budget_s: float = 600.0) -> dict:
    """Run each secondary workload in a child process and summarise it."""
    res = {}
    t_end = time.monotonic() + budget_s
    for name, extra in SECONDARY:
        left = t_end - time.monotonic()
        if left < 30:
            res[name] = {"skipped": "secondary time budget spent"}
            continue
        t0 = time.monotonic()
        try:
            p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--no-cpu"] + extra,
                               capture_output=True, text=True, timeout=min(left, 300))
        except subprocess.TimeoutExpired:
            res[name] = {"error": "timed out"}
            continue
        lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
        if p.returncode != 0 or not lines:
            tail = (p.stderr or p.stdout).strip().splitlines()[-1:] or [""]
            res[name] = {"error": f"rc={p.returncode}: {tail[0][:200]}"}
            continue
        res[name] = _summary(json.loads(lines[-1]))
        res[name]["wall_s"] = round(time.monotonic() - t0, 1)
    return res


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--dtype", choices=("float64", "float32"), default="float64")
    ap.add_argument("--temporal", type=int, default=1)
    ap.add_argument("--layout", choices=("flat", "bricked"), default="flat",
                    help="lap7: fields in flat or bricked layout (resident as bricks)")
    ap.add_argument("--brick", type=int, default=8, help="lap7 bricked: brick size")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--n", type=int, default=512, help="interior extent per dimension")
    ap.add_argument("--gs-n", type=int, default=4096, help="gray_scott: interior extent")
    ap.add_argument("--serve-requests", type=int, default=2000,
                    help="serve: number of requests in the stream")
    ap.add_argument("--workload", choices=("lap7", "sw_batch", "gray_scott", "serve", "wide",
                                           "heat_kahan"),
                    default="lap7",
                    help="lap7: 3-D 7-point 512^3 sweeps; sw_batch: 256 batched shallow-water "
                         "solves; gray_scott: 4096^2 fused Gray-Scott, FP64/FP32/Kahan")
    ap.add_argument("--sw-grids", type=int, default=256, help="sw_batch: number of grids")
    ap.add_argument("--sw-n", type=int, default=0,
                    help="sw_batch: fixed grid size (0 = log-uniform in [64, 2048])")
    ap.add_argument("--sw-steps", type=int, default=200, help="sw_batch: RK2 steps per solve")
    ap.add_argument("--sw-zchunk", type=int, default=0,
                    help="sw_batch: rows per work item (0: the kernels' default)")
    ap.add_argument("--no-compare", dest="compare", action="store_false",
                    help="sw_batch: time the FP32 batch only (profiling cases)")
    ap.add_argument("--no-secondary", dest="secondary", action="store_false",
                    help="default run: skip the secondary workloads summarised under "
                         "'secondary' (each runs as its own process after the headline)")
    args = ap.parse_args()
    args.steps_given = args.steps
    if args.steps is None:
        args.steps = 50
    global N_INTERIOR, SW_GRIDS, SW_FIXED_N, SW_STEPS, SW_ZCHUNK
    N_INTERIOR = args.n
    SW_GRIDS, SW_FIXED_N, SW_STEPS = args.sw_grids, args.sw_n, args.sw_steps
    SW_ZCHUNK = args.sw_zchunk
    global SERVE_REQUESTS, GS_N
    SERVE_REQUESTS = args.serve_requests
    GS_N = args.gs_n
    if args.warmup < 3:
        args.warmup = 3
    if args.workload == "wide":
        if args.impl == "reference":
            line = {"impl": "reference", "unavailable": "the wide tier is timed against the oracle "
                    "in its own line's cpu_baseline"}
        else:
            line = run_wide(args)
    elif args.workload == "serve":
        if args.impl == "reference":
            line = {"impl": "reference", "unavailable": "the reference has no serving layer "
                    "(one launch per grid); the plain-path comparison is in the serve line"}
        else:
            line = run_serve(args)
    elif args.workload == "heat_kahan":
        if args.impl == "reference":
            line = {"impl": "reference", "unavailable": "accuracy comparison of the GPU precision "
                    "modes; its CPU side is the oracle's float32 Kahan step in the parity tests"}
        else:
            if args.steps_given is None:
                args.steps = 2000
            line = run_heat_kahan(args)
    elif args.workload == "gray_scott":
        if args.steps_given is None:
            args.steps = GS_STEPS if args.impl == "ours" else 3
        line = run_gs_reference(args) if args.impl == "reference" else run_gray_scott(args)
    elif args.workload == "sw_batch":
        if args.steps_given is None:
            args.steps = 3
        line = run_sw_reference(args) if args.impl == "reference" else run_sw_batch(args)
    else:
        line = run_reference(args) if args.impl == "reference" else run_ours(args)
        default_run = (args.impl == "ours" and args.workload == "lap7" and args.dtype == "float64"
                       and args.temporal == 1 and args.layout == "flat" and args.n == 512)
        if (line is not None and default_run and args.secondary and line.get("n_gpus") == 1
                and not args.no_cpu):
            # the headline is complete (its timed region is over); the
            # other configurations follow, each in its own process
            line["secondary"] = run_secondary()
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
