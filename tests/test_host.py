"""Host-side logic without a GPU: the C ABI exports every declared entry
point, the frontend and passes produce the reference's attributes, the
planner respects the B200 limits, the emitter's kernels compile with NVRTC
(no device needed), and the launcher's layout/halo rules match the
reference's (tests/test_perf_layout.py, test_normalize_and_analysis.py,
test_dialects.py in the reference are the models)."""

import ctypes
import os
import re

import numpy as np
import pytest

import stencil_defs as D

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


# --------------------------------------------------------------------------- #
# C ABI
# --------------------------------------------------------------------------- #

def _declared_symbols():
    text = open(os.path.join(ROOT, "include", "csd.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(csd_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_entry_point():
    from cutile.runtime import native

    lib = native.library()
    names = _declared_symbols()
    assert len(names) >= 18
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_host_only_entry_points_answer_without_a_gpu():
    from cutile.runtime import native

    lib = native.library()
    assert lib.csd_version() > 0
    assert native.grid_size() % 64 == 0
    shp = (ctypes.c_longlong * 3)(10, 17, 33)
    assert lib.csd_bricked_elems(shp, 3, 8) == 16 * 24 * 40
    assert native.bricked_shape((10, 17, 33), 8) == (2, 3, 5, 8, 8, 8)


# --------------------------------------------------------------------------- #
# Frontend, dialects, passes
# --------------------------------------------------------------------------- #

def _heat2d():
    from cutile import stencil

    return stencil(ndim=2, order=2)(D.heat2d)


def test_heat2d_analysis_attributes():
    from cutile.dialects.stencil import ApplyOp
    from cutile.runtime.pipeline import Pipeline

    m = _heat2d()._ir.clone()
    Pipeline.single_gpu().run(m)
    ap = next(op for op in m.walk() if isinstance(op, ApplyOp))
    assert [a.data for a in ap.attributes["halo_widths"].data] == [1, 1]
    assert ap.attributes["flops"].data == 4          # 3 adds + 1 multiply
    assert ap.attributes["unique_loads"].data == 4
    assert abs(ap.attributes["arithmetic_intensity"].value.data - 4.0 / 40) < 1e-12
    assert ap.attributes["bound"].data == "memory"


def test_lap7_roofline_counts():
    from cutile import stencil
    from cutile.dialects.stencil import ApplyOp
    from cutile.runtime.pipeline import Pipeline

    m = stencil(ndim=3)(D.lap7)._ir.clone()
    Pipeline.single_gpu().run(m)
    ap = next(op for op in m.walk() if isinstance(op, ApplyOp))
    assert ap.attributes["flops"].data == 9
    assert ap.attributes["unique_loads"].data == 7
    assert abs(ap.attributes["arithmetic_intensity"].value.data - 9.0 / 64) < 1e-12


@pytest.mark.parametrize("fn,ndim,T", [(D.heat2d, 2, 5), (D.heat1d, 1, 8), (D.lap7, 3, 1)])
def test_default_temporal_depth_is_the_references(fn, ndim, T):
    from cutile import compile as stencil_compile
    from cutile import stencil

    r = stencil_compile(stencil(ndim=ndim)(fn))
    assert r.temporal_steps == T


def test_boundary_attribute_validation():
    from cutile.dialects.cutile_stencil.dialect import BoundaryAttr

    assert BoundaryAttr("dirichlet", 0.5).has_value
    assert not BoundaryAttr("periodic").has_value
    with pytest.raises(ValueError):
        BoundaryAttr("sideways")


def test_parser_dedups_accesses_and_names_fields():
    from cutile import stencil
    from cutile.dialects.cutile_stencil.dialect import AccessOp, FuncOp

    def f(u, v, i, j):
        return u[i, j] + u[i, j] + v[i + 1, j] * u[i, j]

    ir = stencil(ndim=2)(f)._ir
    func = next(op for op in ir.walk() if isinstance(op, FuncOp))
    accesses = [op for op in ir.walk() if isinstance(op, AccessOp)]
    assert [a.data for a in func.arg_names.data] == ["u", "v"]
    assert sorted(tuple(a.offset.offsets) for a in accesses) == [(0, 0), (1, 0)]


def test_parser_rejects_unsupported_syntax():
    from cutile import stencil

    def bad(u, i, j):
        return u[i * 2, j]

    with pytest.raises(Exception):
        stencil(ndim=2)(bad)


# --------------------------------------------------------------------------- #
# Launcher layout rules (reference test_perf_layout.py)
# --------------------------------------------------------------------------- #

def test_aligned_inner_halo():
    from cutile import compile as stencil_compile
    from cutile import stencil
    from cutile.runtime.launcher import pad_inner_halo

    r = stencil_compile(stencil(ndim=3)(D.lap7), temporal_blocking=False)
    assert r.halo_widths == (1, 1, 16) and r.stencil_halo == (1, 1, 1)
    r = stencil_compile(stencil(ndim=1)(D.lap4_1d), temporal_blocking=False)
    assert r.halo_widths == (16,) and r.stencil_halo == (2,)
    r = stencil_compile(stencil(ndim=3)(D.lap7), temporal_blocking=False, align_halo=False)
    assert r.halo_widths == (1, 1, 1)
    assert pad_inner_halo((1, 1), 4) == (1, 32)
    r = stencil_compile(stencil(ndim=3)(D.lap7), layout="bricked", brick_size=8,
                        temporal_blocking=False)
    assert r.halo_widths == (1, 1, 1)


def test_fit_tiles_and_grid_order():
    from cutile.lowering.stencil_to_target import fit_tiles, grid_order

    assert fit_tiles((1, 1, 512), (66, 66, 96), (1, 1, 16)) == (1, 1, 64)
    assert fit_tiles((1, 1, 512), (258, 258, 544), (1, 1, 16)) == (1, 1, 512)
    assert fit_tiles((4, 256), (6, 132), (1, 16)) == (4, 128)
    assert grid_order(3) == (1, 0, 2) and grid_order(2) == (0, 1) and grid_order(1) == (0,)


# --------------------------------------------------------------------------- #
# Engine planning and code generation
# --------------------------------------------------------------------------- #

@pytest.mark.parametrize("ndim,dtype_bytes,radius,nin", [
    (3, 8, (1, 1, 1), 1), (3, 4, (1, 1, 1), 1), (2, 8, (1, 1), 2), (2, 4, (2, 2), 6),
    (1, 8, (4,), 1), (3, 8, (2, 2, 2), 3)])
def test_plans_fit_the_b200_limits(ndim, dtype_bytes, radius, nin):
    from cutile.passes.tiling import (B200_SMEM_PER_BLOCK, default_engine_plan,
                                      engine_geometry, radius3)

    p = default_engine_plan(ndim, 7, dtype_bytes, radius, nin)
    g = engine_geometry(p, radius3(ndim, radius), dtype_bytes, nin)
    assert g["box_w"] <= 256 and g["box_h"] <= 256
    assert g["smem_bytes"] <= B200_SMEM_PER_BLOCK
    assert (g["box_w"] * dtype_bytes) % 16 == 0


def test_emitted_kernel_keeps_term_order_and_exact_constants():
    from cutile import compile as stencil_compile
    from cutile import stencil

    r = stencil_compile(stencil(ndim=3)(D.lap7), temporal_blocking=False)
    src = r.cuda_source
    # 0.1 as its exact binary64 value, additions in DSL order, no contraction
    assert "0x1.999999999999ap-4" in src
    assert "fma(" not in src
    adds = re.findall(r"__dadd_rn\((\w+), (\w+)\)", src)
    # first addition: the z-1 and z+1 neighbours of point 0, in that order
    assert adds[0] == ("q_L1_0", "q_L2_0")
    assert "t.template strip<0, -1, 0, 0, 0>" in src.split("st1 =")[1].split(";")[0]
    assert "q_L1_0 = st1.v[0];" in src and "q_L2_0 = st2.v[0];" in src


def test_shifted_values_are_computed_once_per_position():
    """A thread's neighbouring points share X-shifted subexpressions: the
    shallow-water body's velocity hu/h and wave speed sqrt(g h) at the east,
    centre and west cells of 4 points cover 6 positions, not 12."""
    from cutile import compile as stencil_compile
    from cutile import stencil

    r = stencil_compile(stencil(ndim=2, dtype="float32")(D.sw_rhs), temporal_blocking=False,
                        align_halo=False)
    body = r.cuda_source.split("struct Body_")[1].split("};")[0]
    sqrts = re.findall(r"csd::sqrt_rn\(", body)
    # centre/east/west: positions -1..4 (6); north and south: 4 each
    assert len(sqrts) == 6 + 4 + 4
    # every output of every point is stored once
    for f in range(3):
        for k in range(4):
            assert body.count(f"o.v[{f}][{k}] = ") == 1


def test_generated_kernels_compile_with_nvrtc_without_spills():
    from cutile import compile as stencil_compile
    from cutile import compile_fused, stencil
    from cutile.runtime.native import compile_source

    results = [
        stencil_compile(stencil(ndim=3)(D.lap7), temporal_blocking=False),
        stencil_compile(stencil(ndim=2, boundary="periodic")(D.heat2d)),
        compile_fused([stencil(ndim=2)(D.gs_u), stencil(ndim=2)(D.gs_v)], precision="fp32_kahan"),
        stencil_compile(stencil(ndim=3, dtype="float32")(D.lap7), layout="bricked", brick_size=8),
    ]
    for r in results:
        path, log = compile_source(r.cuda_source, ["-Xptxas=-v"])
        assert os.path.exists(path)
        blocks = re.split(r"Compiling entry function '", log)[1:]
        assert blocks, log
        for blk in blocks:
            name = blk.split("'", 1)[0]
            m = re.search(r"Function properties for " + name + r"\n.*?(\d+) bytes spill stores",
                          blk, re.S)
            assert m, blk
            sp = int(m.group(1))
            # fused-boundary variants run at the 64-register occupancy floor
            # and may keep a word or two on the stack
            assert sp <= (16 if name.endswith(("_bc_tma", "_bc_ldg")) else 0), (name, log)


def test_module_entry_points():
    from cutile import compile as stencil_compile
    from cutile import stencil

    r = stencil_compile(stencil(ndim=2, boundary="reflecting")(D.heat2d), layout="bricked",
                        brick_size=8)
    mod = r.load_module()
    for name in ("launch_heat2d", "apply_boundary_heat2d", "step_heat2d", "to_bricks",
                 "from_bricks", "launch_heat2d_bricked", "launch_heat2d_on_bricks", "program"):
        assert hasattr(mod, name), name


def test_rk_tables_are_consistent_methods():
    from cutile.runtime.rk_integrator import stage_table

    for method, stages in (("euler", 1), ("rk2", 2), ("rk4", 4), ("ssprk3", 3)):
        t = stage_table(method)
        assert len(t) == stages
        # every method but Euler writes the state in its last stage
        assert (t[-1][7] == "u") == (method != "euler")


def test_pack_grids_rows_are_aligned_for_tma():
    import torch

    from cutile.runtime.rk_runtime import pack_grids

    flat, grids = pack_grids([(66, 66), (5, 7, 9), (130,)], 3, torch.float32, "cpu")
    for g in grids:
        for t in g:
            assert (t.storage_offset() * 4) % 256 == 0
            if t.dim() > 1:
                assert (t.stride(-2) * 4) % 128 == 0
            assert t.stride(-1) == 1
    # views do not overlap
    ends = sorted((t.storage_offset(), t.storage_offset() + t.stride(0) * t.shape[0])
                  for g in grids for t in g)
    assert all(a[1] <= b[0] for a, b in zip(ends, ends[1:]))


def test_autotune_candidates_fit_and_are_distinct():
    from cutile.passes.tiling import B200_SMEM_PER_BLOCK, engine_geometry, radius3
    from cutile.runtime.autotune import cache_key, candidates

    for ndim, db, radius, nin, single in ((3, 8, (1, 1, 1), 1, True), (3, 4, (2, 2, 2), 1, True),
                                          (2, 8, (1, 1), 3, False), (1, 4, (4,), 1, True)):
        plans = candidates(ndim, db, radius, nin, 7, 20, single)
        assert 1 < len(plans) <= 30
        keys = {(p.rows, p.tile_y, p.tile_x, p.threads, p.stages, p.temporal, p.min_blocks)
                for p in plans}
        assert len(keys) == len(plans)
        for p in plans:
            g = engine_geometry(p, radius3(ndim, radius), db, nin)
            assert g["smem_bytes"] <= B200_SMEM_PER_BLOCK and g["box_w"] <= 256
            assert single or p.temporal == 1
    fp = {"radius": [1, 1, 1], "loads": 7, "inputs": 1, "outputs": 1, "body_ops": 20}
    assert cache_key(fp, "float64", (512,) * 3, "B200") == cache_key(fp, "float64", (512,) * 3, "B200")
    assert cache_key(fp, "float64", (512,) * 3, "B200") != cache_key(fp, "float32", (512,) * 3, "B200")
    assert cache_key(fp, "float64", (512,) * 3, "B200") != cache_key(fp, "float64", (128,) * 3, "B200")


def test_regcheck_selection_rules():
    from cutile.runtime.regcheck import (Config, Resources, parse_ptxas_log, register_budget,
                                         select_config, select_fastest)

    assert register_budget(occupancy=4) == 128 and register_budget(2) == 256
    cfgs = [Config((1, 4, 128), {"k": 0}), Config((1, 8, 64), {"k": 1}), Config((1, 2, 32), {"k": 2})]
    res = {0: Resources(200, 0), 1: Resources(90, 0), 2: Resources(60, 0)}
    assert select_config(cfgs, lambda c: res[c.kernel_hints["k"]], max_registers=128) is cfgs[1]
    spill = {0: Resources(128, 64, spill_bytes=64), 1: Resources(128, 32, spill_bytes=32),
             2: Resources(255, 8, spill_bytes=8)}
    assert select_config(cfgs, lambda c: spill[c.kernel_hints["k"]]) is cfgs[2]
    timed = {0: Resources(64, 0, ms=1.00), 1: Resources(64, 0, ms=0.99), 2: Resources(64, 0, ms=0.5)}
    assert select_fastest(cfgs, lambda c: timed[c.kernel_hints["k"]]) is cfgs[2]
    near = {0: Resources(64, 0, ms=1.02), 1: Resources(64, 0, ms=1.0), 2: Resources(64, 0, ms=1.5)}
    assert select_fastest(cfgs, lambda c: near[c.kernel_hints["k"]]) is cfgs[0]   # within 3 %
    log = ("ptxas info    : Compiling entry function 'k_tma' for 'sm_100a'\n"
           "ptxas info    : Function properties for k_tma\n"
           "ptxas         .     8 bytes stack frame, 4 bytes spill stores, 4 bytes spill loads\n"
           "ptxas info    : Used 96 registers, used 1 barriers, 128 bytes smem\n")
    r = parse_ptxas_log(log, "k_tma")
    assert r.registers == 96 and r.stack_bytes == 8 and r.spill_bytes == 4 and r.spills


def test_serving_descriptor_pool_reuses_and_grows():
    import torch

    from cutile.runtime import native
    from cutile.runtime.serving import SolveKind, StencilServer

    s = StencilServer([SolveKind("k", {}, 1)], device="cpu")
    gsz = native.grid_size()
    a = s._pool_alloc(2)
    s._pool[a * gsz:(a + 2) * gsz] = 7
    b = s._pool_alloc(3)
    assert b == a + 2
    s._pool_release(a, 2)
    assert s._pool_alloc(2) == a            # a freed block of the same size comes back
    blocks = [s._pool_alloc(3) for _ in range(200)]   # forces growth
    assert len(set(blocks)) == 200
    assert s._pool.numel() >= (max(blocks) + 3) * gsz
    assert bool((s._pool[a * gsz:(a + 2) * gsz] == 7).all())   # contents survive growth
    assert s._pool.dtype == torch.uint8


def test_occupancy_hint_reaches_the_launch_bound():
    from cutile import compile as stencil_compile
    from cutile import stencil

    fn = stencil(ndim=3)(D.lap7)
    for occ in (1, 2, 4):
        r = stencil_compile(fn, temporal_blocking=False, occupancy=occ)
        bounds = re.findall(r"__launch_bounds__\((\d+), (\d+)\)", r.cuda_source)
        assert bounds and all(int(b) == occ for _, b in bounds), (occ, bounds)
        assert r.kernel_hints["occupancy"] == occ
    # without a hint the planner derives it from shared memory and registers
    r = stencil_compile(fn, temporal_blocking=False)
    assert "occupancy" not in r.kernel_hints


@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_body_emission_is_well_formed_on_random_expressions(tmp_path, dtype):
    """The shift-shared body of every random expression defines each value
    once, before its first use, and stores every output of every point once."""
    import random_exprs

    import cutile

    vec = 2 if dtype == "float64" else 4
    for seed in range(40):
        ndim, nfields, radius, fields, idx, body = random_exprs.case(seed)
        fn = random_exprs.build(tmp_path, f"e{seed}_{dtype}", fields, idx, body, dtype=dtype)
        r = cutile.compile(fn, temporal_blocking=False, align_halo=bool(seed % 2))
        text = r.cuda_source.split("struct Body_")[1].split("\n};")[0]
        defined = set()
        for line in text.splitlines():
            m = re.match(r"\s*const (?:double|float|bool) (q_\w+) = (.*);$", line)
            if m:
                for used in re.findall(r"\bq_\w+", m.group(2)):
                    assert used in defined, (seed, line)
                assert m.group(1) not in defined, (seed, line)
                defined.add(m.group(1))
        for k in range(vec):
            assert len(re.findall(rf"o\.v\[0\]\[{k}\] = ", text)) == 1, seed


def test_rows_per_thread_plans():
    """Dense FP64 boxes default to several Y rows per thread (measured
    faster); temporal chains, caller tiles and other stencils keep one."""
    import wide_defs as W

    from dataclasses import replace

    from cutile import compile as stencil_compile
    from cutile import stencil
    from cutile.passes.tiling import EnginePlan, fit_plan

    r27 = stencil_compile(W.load_box("box27_plan", 1), temporal_blocking=False)
    assert r27.tile_sizes == (1, 16, 64) and r27.kernel_hints["rpy"] == 4
    assert ", 4, 2> Cfg_box27_plan_tma;" in r27.cuda_source   # RPY 4, VEC 2
    r125 = stencil_compile(W.load_box("box125_plan", 2), temporal_blocking=False)
    assert r125.tile_sizes == (2, 4, 128) and r125.kernel_hints["rpy"] == 2
    assert "rpy" not in stencil_compile(W.load_box("box27_plan", 1)).kernel_hints  # T = 2
    assert "rpy" not in stencil_compile(W.load_box("box27_plan", 1), temporal_blocking=False,
                                        tile_sizes=(1, 4, 64)).kernel_hints
    assert "rpy" not in stencil_compile(W.load_box("box27_f32", 1, dtype="float32"),
                                        temporal_blocking=False).kernel_hints
    assert "rpy" not in stencil_compile(stencil(ndim=3)(D.lap7), temporal_blocking=False).kernel_hints
    p = EnginePlan(3, rows=1, tile_y=8, tile_x=64, vec=2, threads=128, stages=1, zchunk=0, rpy=2)
    assert fit_plan(p, (1, 1, 1), 8, 1).units_per_step == 8 // 2 * 32
    with pytest.raises(ValueError):
        fit_plan(replace(p, temporal=2), (1, 1, 1), 8, 1)
    with pytest.raises(ValueError):
        fit_plan(replace(p, tile_y=6, rpy=4), (1, 1, 1), 8, 1)


# --------------------------------------------------------------------------- #
# Autotune plans round-trip through compile()
# --------------------------------------------------------------------------- #


def _box27():
    import wide_defs as W

    return W.load_box("box27_rt", 1)


def test_probe_compiles_the_candidate_plan():
    """Every autotune candidate, compiled with the hints its probe passes,
    gives a kernel of that plan (rows per thread included)."""
    import cutile
    from cutile.runtime import autotune as A

    fn = _box27()
    fp = A._footprint(fn, 8)
    plans = A.candidates(3, 8, fp["radius"], fp["inputs"], fp["loads"], fp["body_ops"],
                         True, 30, fp["outputs"])
    assert any(p.rpy > 1 for p in plans), "the rows-per-thread default is a candidate"
    for p in plans:
        r = cutile.compile(fn, tile_sizes=p.tile_sizes(), kernel_hints=A.probe_hints(p),
                           temporal_steps=p.temporal, autotune=False)
        assert r.tile_sizes == p.tile_sizes()
        assert r.kernel_hints == p.hints(), (p, r.kernel_hints)


def test_candidates_keep_plans_that_differ_only_in_rows_per_thread():
    from dataclasses import replace

    from cutile.passes.tiling import default_engine_plan

    base = default_engine_plan(3, 27, 8, (1, 1, 1), 1, 1)
    assert base.rpy == 4
    key = lambda f: (f.rows, f.tile_y, f.tile_x, f.threads, f.stages, f.temporal, f.min_blocks, f.rpy)
    assert key(base) != key(replace(base, rpy=1))


def test_autotuned_hints_round_trip_through_compile():
    """An AutotuneResult's (tile_sizes, kernel_hints) passed back to compile()
    rebuild its plan: the 'rpy' key written by EnginePlan.hints() is read."""
    import cutile
    from cutile.passes.tiling import default_engine_plan

    fn = _box27()
    plan = default_engine_plan(3, 27, 8, (1, 1, 1), 1, 1)
    r0 = cutile.compile(fn, temporal_blocking=False, autotune=False)
    assert r0.kernel_hints.get("rpy") == plan.rpy == 4
    r1 = cutile.compile(fn, tile_sizes=r0.tile_sizes, kernel_hints=r0.kernel_hints,
                        temporal_blocking=False, autotune=False)
    assert r1.kernel_hints == r0.kernel_hints and r1.tile_sizes == r0.tile_sizes


def test_tuple_returning_stencil_keeps_one_row_per_thread():
    """The rows-per-thread default is for one-input, one-output kernels; a
    wide single-input stencil with two outputs keeps one row."""
    import cutile
    from cutile import stencil

    def two(u, i, j, k):
        s = (u[i - 1, j, k] + u[i + 1, j, k] + u[i, j - 1, k] + u[i, j + 1, k] + u[i, j, k - 1]
             + u[i, j, k + 1] + u[i - 1, j - 1, k] + u[i + 1, j + 1, k] + u[i - 1, j, k - 1]
             + u[i + 1, j, k + 1] + u[i, j - 1, k - 1] + u[i, j + 1, k + 1] + u[i - 1, j + 1, k]
             + u[i + 1, j - 1, k] + u[i, j - 1, k + 1] + u[i, j + 1, k - 1] + u[i - 1, j, k + 1])
        return s, 0.5 * s

    import importlib.util
    import inspect
    import os
    import tempfile
    import textwrap

    src = "from cutile import stencil\n\n@stencil(ndim=3)\n" + textwrap.dedent(inspect.getsource(two))
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "two_out.py")
        open(path, "w").write(src)
        spec = importlib.util.spec_from_file_location("two_out", path)
        m = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(m)
        r = cutile.compile(m.two, temporal_blocking=False, autotune=False)
    assert "rpy" not in r.kernel_hints


def test_rows_per_thread_default_falls_back_when_it_would_spill():
    """The reference's box125 (46 irregularly ordered terms) spills at two
    rows per thread, so its default plan keeps one row; the regular 125-point
    box keeps the two-row plan."""
    import tempfile

    import cutile
    import ref_corpus as RC
    import wide_defs as W

    entries, _ = RC.load()
    with tempfile.TemporaryDirectory() as tmp:
        fn = RC.build(tmp, "wide_stencils/box125", entries["wide_stencils/box125"])
        r = cutile.compile(fn, temporal_blocking=False)
    assert "rpy" not in r.kernel_hints
    r2 = cutile.compile(W.load_box("regular_box125", 2), temporal_blocking=False)
    assert r2.kernel_hints.get("rpy") == 2


def test_body_unroll_choice():
    """Small bodies let the engine unroll a stage's units; wide ones (many
    strip groups, rows per thread, long bodies) keep the loop."""
    import re
    import tempfile

    import cutile
    import ref_corpus as RC
    from cutile import stencil

    def unroll(r):
        return {int(m) for m in re.findall(r"static constexpr int UNROLL = (\d+);", r.cuda_source)}

    assert unroll(cutile.compile(stencil(ndim=3, order=2)(D.lap7), temporal_blocking=False)) == {4}
    assert unroll(cutile.compile(stencil(ndim=2)(D.heat2d), temporal_blocking=False)) == {4}
    entries, _ = RC.load()
    with tempfile.TemporaryDirectory() as tmp:
        fn = RC.build(tmp, "wide_stencils/box125", entries["wide_stencils/box125"])
        assert unroll(cutile.compile(fn, temporal_blocking=False)) == {0}
    from cutile import RKIntegrator

    rk = RKIntegrator(stencil(ndim=2, dtype="float32")(D.sw_rhs), "rk2").compile(boundary="reflecting")
    assert unroll(rk) == {0}


def test_measured_default_plans_per_dtype_and_depth():
    """The plan tables: 2-D single steps (FP64 256 threads, FP32 128), 3-D
    chains by depth (tallest tile that fits, a thread per unit past T=2), 2-D
    chains by depth; what fit_plan returns for the 7-point and 5-point bodies."""
    import cutile
    from cutile import stencil

    def plan(fn, ndim, dt, T):
        kw = {"temporal_blocking": False} if T == 1 else {"temporal_steps": T}
        r = cutile.compile(stencil(ndim=ndim, dtype=dt)(fn), **kw)
        assert r.temporal_steps == T
        return r.tile_sizes, r.kernel_hints["threads"]

    assert plan(D.heat2d, 2, "float64", 1) == ((8, 128), 256)
    assert plan(D.heat2d, 2, "float32", 1) == ((8, 128), 128)
    assert plan(D.lap7, 3, "float64", 2) == ((1, 8, 128), 256)
    assert plan(D.lap7, 3, "float64", 4) == ((1, 16, 64), 512)
    assert plan(D.lap7, 3, "float64", 8) == ((1, 8, 32), 128)
    assert plan(D.lap7, 3, "float32", 2) == ((1, 8, 128), 128)
    assert plan(D.lap7, 3, "float32", 4) == ((1, 32, 64), 512)
    assert plan(D.lap7, 3, "float32", 8) == ((1, 16, 32), 128)
    assert plan(D.heat2d, 2, "float64", 2) == ((8, 64), 128)
    assert plan(D.heat2d, 2, "float64", 3) == ((4, 128), 128)
    assert plan(D.heat2d, 2, "float32", 2) == ((8, 128), 128)
    assert plan(D.heat2d, 2, "float32", 3) == ((8, 128), 256)
    assert plan(D.heat2d, 2, "float32", 8) == ((8, 128), 256)
    from cutile import compile_fused

    gs = [stencil(ndim=2)(D.gs_u), stencil(ndim=2)(D.gs_v)]
    r = compile_fused(gs, precision="fp64", boundary="periodic")
    assert (r.tile_sizes, r.kernel_hints["threads"]) == ((8, 64), 256)
    r = compile_fused(gs, precision="fp32", boundary="periodic")
    assert (r.tile_sizes, r.kernel_hints["threads"]) == ((8, 128), 256)


def test_wider_units_only_for_single_step_flat_one_row_kernels():
    import pytest as _pytest

    import cutile
    from cutile import stencil

    lap = stencil(ndim=3, order=2)(D.lap7)
    r = cutile.compile(lap, temporal_blocking=False, tile_sizes=(1, 4, 128),
                       kernel_hints={"vec": 4, "threads": 64})
    assert r.kernel_hints["vec"] == 4 and ", 1, 4> Cfg_lap7_tma;" in r.cuda_source
    with _pytest.raises(ValueError):
        cutile.compile(lap, temporal_steps=2, tile_sizes=(1, 8, 128), kernel_hints={"vec": 4})
    with _pytest.raises(ValueError):
        cutile.compile(lap, temporal_blocking=False, tile_sizes=(1, 4, 128),
                       kernel_hints={"vec": 3})
    with _pytest.raises(ValueError):
        cutile.compile(lap, temporal_blocking=False, layout="bricked", brick_size=8,
                       tile_sizes=(1, 4, 128), kernel_hints={"vec": 4})


def test_bricked_wrapper_takes_the_arrays_halo():
    """``launch_<name>_on_bricks`` passes a ``halo=`` override to the
    program (a halo of whole bricks starts the interior on a brick)."""
    import inspect

    import cutile
    from cutile import stencil

    r = cutile.compile(stencil(ndim=3)(D.lap7), layout="bricked", brick_size=8,
                       temporal_blocking=False)
    assert "def launch_lap7_on_bricks(u_in, u_out, shape, stream=None, halo=None):" in r.code
    assert "shape, stream, scalars=None, halo=halo)" in r.code
    from cutile.runtime.module import StencilProgram

    assert "halo" in inspect.signature(StencilProgram.launch_on_bricks).parameters
