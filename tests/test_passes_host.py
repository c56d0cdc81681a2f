"""Pass-level tests (the reference's own pass tests, tests/test_cutile_new.py:
437-519, plus the B200 engine constraints VerifyPass adds)."""

from dataclasses import replace

import pytest

import stencil_defs as D


def _heat2d():
    from cutile import stencil

    return stencil(ndim=2, order=2)(D.heat2d)


def _normalized(fn):
    from cutile.ir.core import Context
    from cutile.passes.normalize import NormalizePass

    ctx = Context()
    m = fn._ir.clone()
    NormalizePass().apply(ctx, m)
    return m, ctx


def _apply_attrs(module):
    from cutile.dialects.stencil import ApplyOp

    return next(op for op in module.walk() if isinstance(op, ApplyOp)).attributes


def test_fusion_pass_marks_group():
    from cutile.passes.fusion import FusionPass

    m, ctx = _normalized(_heat2d())
    FusionPass().apply(ctx, m)
    a = _apply_attrs(m)
    assert a["fusion_group"].data == 0 and a["fusion_outputs"].data == 1


def test_bricked_layout_pass():
    from cutile.passes.bricked import BrickedLayoutPass

    m, ctx = _normalized(_heat2d())
    BrickedLayoutPass(brick_size=64).apply(ctx, m)
    a = _apply_attrs(m)
    assert a["layout"].data == "bricked" and a["brick_size"].data == 64


def _through_tiling(fn):
    from cutile.runtime.pipeline import Pipeline

    m = fn._ir.clone()
    Pipeline.single_gpu().run(m)
    from cutile.ir.core import Context

    return m, Context()


def test_verify_pass_accepts_valid_ir():
    from cutile import stencil
    from cutile.passes.verify import VerifyPass

    m, ctx = _through_tiling(stencil(ndim=1, order=2)(D.heat1d))
    VerifyPass().apply(ctx, m)


def test_verify_pass_checks_power_of_2():
    from cutile.ir.core import ArrayAttr, IntAttr
    from cutile.passes.analysis.footprint import AnalysisPass
    from cutile.passes.verify import VerifyPass
    from cutile import stencil

    m, ctx = _normalized(stencil(ndim=1, order=2)(D.heat1d))
    AnalysisPass().apply(ctx, m)
    _apply_attrs(m)["tile_sizes"] = ArrayAttr([IntAttr(100)])
    with pytest.raises(ValueError, match="not a power of 2"):
        VerifyPass().apply(ctx, m)


def _lap7_plan():
    from cutile.passes.tiling import default_engine_plan, fit_plan

    return fit_plan(default_engine_plan(3, 7, 8, (1, 1, 1), 1), (1, 1, 1), 8, 1)


def _lap7_module():
    from cutile import stencil

    return _through_tiling(stencil(ndim=3, order=2)(D.lap7))[0]


def test_engine_plan_of_the_7_point_sweep_verifies():
    from cutile.passes.verify import verify_engine_plan

    m = _lap7_module()
    verify_engine_plan(m, _lap7_plan(), (1, 1, 1), 8, 1)
    a = _apply_attrs(m)
    assert [x.data for x in a["engine_tile"]] == list(_lap7_plan().tile_sizes())
    assert a["engine_smem"].data > 0


@pytest.mark.parametrize("change, match", [
    (dict(tile_x=512), "row width"),             # box row 512 + halo > 256
    (dict(tile_y=512), "tile height"),           # box height > 256
    (dict(tile_x=127), "vector"),                # not a whole number of 2-point vectors
    (dict(threads=100), "whole warps"),
    (dict(rpy=3, tile_y=4), "rows per thread"),
    (dict(rows=64, tile_y=64, tile_x=128), "shared memory"),
])
def test_engine_constraints_are_enforced(change, match):
    from cutile.passes.verify import verify_engine_plan

    with pytest.raises(ValueError, match=match):
        verify_engine_plan(_lap7_module(), replace(_lap7_plan(), **change), (1, 1, 1), 8, 1)


def test_box_row_must_be_whole_16_byte_units():
    from cutile.passes.verify import VerifyPass, attach_engine_plan
    from cutile.ir.core import Context

    m = _lap7_module()
    g = {"box_w": 131, "box_h": 6, "smem_bytes": 1000}
    attach_engine_plan(m, _lap7_plan(), g, 8)
    with pytest.raises(ValueError, match="16 bytes"):
        VerifyPass().apply(Context(), m)


def test_compile_paths_run_the_verifier(monkeypatch):
    """compile(), compile_fused() and the RK stage builds verify their plans."""
    import cutile
    from cutile import RKIntegrator, stencil
    from cutile.passes import verify as V
    from cutile.runtime import launcher as L

    calls = []
    real = V.verify_engine_plan

    def spy(*a, **k):
        calls.append(a[1])
        return real(*a, **k)

    monkeypatch.setattr(L, "verify_engine_plan", spy)
    cutile.compile(stencil(ndim=3, order=2)(D.lap7), temporal_blocking=False)
    assert len(calls) == 1
    cutile.compile_fused([stencil(ndim=2)(D.gs_u), stencil(ndim=2)(D.gs_v)], boundary="periodic")
    assert len(calls) == 3   # one per fused member
    RKIntegrator(stencil(ndim=2)(D.sw_rhs), "rk2").compile(boundary="reflecting")
    assert len(calls) > 3


def test_multi_field_temporal_chains_need_one_output_per_input():
    """A chain feeds output f into input f of the next step: the compensated
    (u, c) pair chains; two inputs feeding one output cannot."""
    import cutile
    from cutile import stencil

    r = cutile.compile(stencil(ndim=2, dtype="float32")(D.heat_small_dt), precision="fp32_kahan",
                       temporal_steps=4)
    assert r.temporal_steps == 4 and r.inputs == ("u", "c_in")
    with pytest.raises(NotImplementedError, match="one output per input"):
        cutile.compile(stencil(ndim=2)(D.leapfrog), temporal_steps=2)
    # without an explicit depth, multi-field stencils keep one step per launch
    assert cutile.compile(stencil(ndim=2, dtype="float32")(D.heat_small_dt),
                          precision="fp32_kahan").temporal_steps == 1


def test_chain_shared_memory_counts_every_field():
    from cutile.passes.tiling import EnginePlan, engine_geometry

    p = EnginePlan(2, rows=8, tile_y=1, tile_x=128, vec=4, threads=128, stages=1, zchunk=0,
                   temporal=4)
    one = engine_geometry(p, (1, 0, 1), 4, 1)["smem_bytes"]
    two = engine_geometry(p, (1, 0, 1), 4, 2)["smem_bytes"]
    assert two > 2 * one - 4096
