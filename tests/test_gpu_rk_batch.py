"""Runge-Kutta stages with fused FP64 combination, single grids and batches
of uneven grids (one persistent launch per stage), CFL steps, CUDA graphs."""

import numpy as np
import pytest

import stencil_defs as D
from oracle import stencil_oracle as O

pytestmark = pytest.mark.gpu


def _stencil(fn, ndim, **kw):
    from cutile import stencil

    return stencil(ndim=ndim, **kw)(fn)


def heat_op(u, i, j):
    return 0.25 * (u[i - 1, j] + u[i + 1, j] + u[i, j - 1] + u[i, j + 1] - 4.0 * u[i, j])


@pytest.mark.parametrize("method", ["euler", "rk2", "rk4", "ssprk3"])
def test_rk_single_grid_matches_oracle(method):
    import torch

    from cutile import RKIntegrator

    rk = RKIntegrator(_stencil(heat_op, 2), method).compile()
    h = rk.info["halo"]
    u0 = np.zeros((40 + 2 * h[0], 50 + 2 * h[1]))
    u0[h[0]:-h[0], h[1]:-h[1]] = np.random.default_rng(3).random((40, 50))
    step = getattr(rk.load_module(), f"rk_{method}_step")
    t = torch.from_numpy(u0).cuda()
    want = (u0,)
    for _ in range(3):
        step(t, 0.1)
        want = O.rk_step(heat_op, ["u"], want, method, 0.1, 2, h)
    torch.cuda.synchronize()
    inner = tuple(slice(x, s - x) for x, s in zip(h, u0.shape))
    assert np.array_equal(t.cpu().numpy()[inner], want[0][inner])


def _sw_setup(sizes, dtype="float32", seed=3):
    from cutile import RKIntegrator, compile as stencil_compile

    op = _stencil(D.sw_rhs, 2, dtype=dtype)
    rk = RKIntegrator(op, "rk2").compile(boundary="reflecting")
    speed = stencil_compile(_stencil(D.sw_speed, 2, dtype=dtype), reduce="max")
    rng = np.random.default_rng(seed)
    h = rk.info["halo"]
    grids = [D.sw_init(n, rng, halo=h, dtype=dtype) for n in sizes]
    return rk, speed, grids, h


ODD = {1: (1,), 2: (0,)}   # hu flips across x walls (dim 1), hv across y walls (dim 0)
BC_ODD = (0, 2, 1)


def test_sw_batch_rk2_cfl_bit_exact_with_oracle():
    import torch

    from cutile.runtime.rk_runtime import RKBatch

    sizes = [40, 65, 97]
    rk, speed, grids, h = _sw_setup(sizes)
    states = [tuple(torch.from_numpy(a).cuda() for a in g) for g in grids]
    dx = [1.0 / n for n in sizes]
    batch = RKBatch(rk, states, [{"dx": d} for d in dx],
                    cfl=(speed.load_module().program(), dx, 0.4), bc_odd=BC_ODD, zchunk=16)
    ref = [tuple(a.copy() for a in g) for g in grids]
    for _ in range(4):
        batch.step()
        for k, n in enumerate(sizes):
            dt = O.cfl_dt(D.sw_speed, ref[k], ["h", "hu", "hv"], 2, h, 0.4, dx[k])
            ref[k] = O.rk_step(D.sw_rhs, ["h", "hu", "hv"], ref[k], "rk2", dt, 2, h,
                               {"dx": dx[k]}, "reflecting", ODD)
    torch.cuda.synchronize()
    for k, n in enumerate(sizes):
        inner = tuple(slice(x, s - x) for x, s in zip(h, grids[k][0].shape))
        for f in range(3):
            got = states[k][f].cpu().numpy()[inner]
            assert np.array_equal(got, ref[k][f][inner]), (n, f)


def test_sw_batch_graph_replay_equals_eager():
    import torch

    from cutile.runtime.rk_runtime import RKBatch

    sizes = [64, 90, 128, 33]
    rk, speed, grids, h = _sw_setup(sizes, seed=4)
    dx = [1.0 / n for n in sizes]

    def make():
        st = [tuple(torch.from_numpy(a.copy()).cuda() for a in g) for g in grids]
        b = RKBatch(rk, st, [{"dx": d} for d in dx],
                    cfl=(speed.load_module().program(), dx, 0.4), bc_odd=BC_ODD)
        return st, b

    st_e, b_e = make()
    for _ in range(10):
        b_e.step()
    st_g, b_g = make()
    g = b_g.capture(10)
    g.replay()
    torch.cuda.synchronize()
    for a, b in zip(st_e, st_g):
        for x, y in zip(a, b):
            assert torch.equal(x, y)
    del g


def test_sw_fp32_vs_fp64_error_small():
    """FP32 fields with FP64 stage combination against the FP64 path."""
    import torch

    from cutile.runtime.rk_runtime import RKBatch

    sizes = [64, 128]
    steps = 50
    out = {}
    for dtype in ("float64", "float32"):
        rk, speed, grids, h = _sw_setup(sizes, dtype=dtype, seed=5)
        st = [tuple(torch.from_numpy(a).cuda() for a in g) for g in grids]
        dx = [1.0 / n for n in sizes]
        b = RKBatch(rk, st, [{"dx": d} for d in dx],
                    cfl=(speed.load_module().program(), dx, 0.4), bc_odd=BC_ODD)
        for _ in range(steps):
            b.step()
        torch.cuda.synchronize()
        out[dtype] = [(s[0].cpu().numpy().astype(np.float64), h) for s in st]
    for (a, ha), (b, hb) in zip(out["float32"], out["float64"]):
        ia = tuple(slice(x, s - x) for x, s in zip(ha, a.shape))
        ib = tuple(slice(x, s - x) for x, s in zip(hb, b.shape))
        rel = np.linalg.norm(a[ia] - b[ib]) / np.linalg.norm(b[ib])
        print("rel L2 fp32 vs fp64:", rel)
        assert rel < 1e-6


def test_sw_batch_row_pitched_equals_contiguous():
    """Packed row-pitched fields (TMA loader) give the same bits as separate
    C-contiguous fields (cp.async loader for odd row pitches)."""
    import torch

    from cutile.runtime.rk_runtime import RKBatch, pack_grids

    sizes = [40, 65, 97, 130]
    rk, speed, grids, h = _sw_setup(sizes, seed=6)
    dx = [1.0 / n for n in sizes]
    st_c = [tuple(torch.from_numpy(a.copy()).cuda() for a in g) for g in grids]
    _, st_p = pack_grids([g[0].shape for g in grids], 3, torch.float32, "cuda")
    for dst, g in zip(st_p, grids):
        for d, a in zip(dst, g):
            d.copy_(torch.from_numpy(a))
    out = []
    for st in (st_c, st_p):
        b = RKBatch(rk, st, [{"dx": d} for d in dx],
                    cfl=(speed.load_module().program(), dx, 0.4), bc_odd=BC_ODD)
        for _ in range(5):
            b.step()
        out.append(b)
    torch.cuda.synchronize()
    assert out[1].stage_launches[0].loader == 0   # TMA
    for a, b in zip(st_c, st_p):
        for x, y in zip(a, b):
            assert torch.equal(x, y)


@pytest.mark.parametrize("method", ["rk4", "ssprk3"])
def test_batch_of_other_methods_equals_single_grid_steps(method):
    """Batched stages of RK4 / SSPRK3 (accumulator and convex-combination
    forms) give each grid the bits of its own single-grid steps."""
    import torch

    from cutile import RKIntegrator
    from cutile.runtime.rk_runtime import RKBatch

    rk = RKIntegrator(_stencil(heat_op, 2), method).compile()
    h = rk.info["halo"]
    rng = np.random.default_rng(9)
    shapes = [(30, 41), (57, 33), (64, 64)]
    grids = []
    for n0, n1 in shapes:
        u = np.zeros((n0 + 2 * h[0], n1 + 2 * h[1]))
        u[h[0]:-h[0], h[1]:-h[1]] = rng.random((n0, n1))
        grids.append(u)
    batched = [(torch.from_numpy(u).cuda(),) for u in grids]
    b = RKBatch(rk, batched, dt=0.05)
    single = [torch.from_numpy(u).cuda() for u in grids]
    step = getattr(rk.load_module(), f"rk_{method}_step")
    for _ in range(4):
        b.step()
        for t in single:
            step(t, 0.05)
    torch.cuda.synchronize()
    for (x,), y in zip(batched, single):
        assert torch.equal(x, y)
