"""Parity at the benchmarked workload sizes, on the benchmark's own plans.

The small parity cases run other work splits than the full-size launches (one
work item per resident block, fused-boundary edge splits, batched work lists
over 256 uneven grids), so each benchmarked configuration is also checked at
its real size against the oracle:

* 3-D 7-point Laplacian, 512^3 interior, N(0,1) seed 1, FP64 and FP32, two
  sweeps through ping-pong buffers (compiled exactly as the benchmark does),
  and one four-step chained launch in each dtype;
* 2-D Gray-Scott 4096^2 periodic, fused two-output step in FP64 and the
  FP32 Kahan-compensated step, from the seeded 20-square start;
* 256 shallow-water grids, sizes log-uniform in 64..2048 (seed 3), FP32 with
  FP64 RK2 combination, reflective walls, per-grid CFL dt, two steps in one
  batch; every fourth grid plus the largest and smallest is replayed by the
  oracle (each grid is independent; the oracle needs ~40 s per step for all
  256 on one core).

All comparisons are bit-exact.
"""

import numpy as np
import pytest

import stencil_defs as D
from oracle import stencil_oracle as O

pytestmark = pytest.mark.gpu


def _torch():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch


@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_lap7_512_cubed_two_sweeps(dtype):
    import cutile
    from cutile import stencil

    torch = _torch()
    r = cutile.compile(stencil(ndim=3, order=2, dtype=dtype)(D.lap7), temporal_blocking=False)
    h = r.halo_widths
    n = 512
    shape = tuple(n + 2 * x for x in h)
    u = np.zeros(shape, dtype=dtype)
    inner = tuple(slice(x, s - x) for x, s in zip(h, shape))
    u[inner] = np.random.default_rng(1).standard_normal((n, n, n)).astype(dtype)
    launch = getattr(r.load_module(), f"launch_{r.name}")
    a = torch.from_numpy(u).cuda()
    b = torch.zeros_like(a)
    launch(a, b)
    launch(b, a)
    torch.cuda.synchronize()
    got = a.cpu().numpy()
    del a, b
    want = O.apply_stencil(u, D.lap7, 3, h)
    want = O.apply_stencil(want, D.lap7, 3, h)
    assert np.array_equal(got[inner], want[inner])
    from cutile.runtime import native

    assert native.error_word(reset=True) == 0


@pytest.mark.parametrize("dtype,T", [("float64", 4), ("float32", 4)])
def test_lap7_512_cubed_chain(dtype, T):
    """One temporally blocked launch at 512^3 on the default chain plan (the
    tallest tiles, one block per SM, eight waves of items)."""
    import cutile
    from cutile import stencil

    torch = _torch()
    r = cutile.compile(stencil(ndim=3, order=2, dtype=dtype)(D.lap7), temporal_steps=T)
    assert r.temporal_steps == T
    h = r.halo_widths
    n = 512
    shape = tuple(n + 2 * x for x in h)
    u = np.zeros(shape, dtype=dtype)
    inner = tuple(slice(x, s - x) for x, s in zip(h, shape))
    u[inner] = np.random.default_rng(1).standard_normal((n, n, n)).astype(dtype)
    a = torch.from_numpy(u).cuda()
    b = torch.zeros_like(a)
    getattr(r.load_module(), f"launch_{r.name}")(a, b)
    torch.cuda.synchronize()
    got = b.cpu().numpy()
    del a, b
    want = O.temporal_launch(u, np.zeros_like(u), D.lap7, 3, h, T)
    assert np.array_equal(got[inner], want[inner])


def _gs(precision):
    import cutile
    from cutile import stencil

    return cutile.compile_fused([stencil(ndim=2)(D.gs_u), stencil(ndim=2)(D.gs_v)],
                                precision=precision, boundary="periodic")


def test_gray_scott_4096_fp64_fused_periodic_steps():
    torch = _torch()
    r = _gs("fp64")
    h = r.halo_widths
    u, v = D.gray_scott_init(4096, seed=2, halo=h)
    step = getattr(r.load_module(), f"step_{r.name}")
    a = [torch.from_numpy(u).cuda(), torch.from_numpy(v).cuda()]
    b = [torch.zeros_like(a[0]), torch.zeros_like(a[1])]
    for _ in range(2):
        step(*a, *b)
        a, b = b, a
    torch.cuda.synchronize()
    cu, cv = u.copy(), v.copy()
    for _ in range(2):
        cu, cv = (O.stencil_with_boundary([cu, cv], D.gs_u, 2, h, "periodic"),
                  O.stencil_with_boundary([cu, cv], D.gs_v, 2, h, "periodic"))
    inner = tuple(slice(x, s - x) for x, s in zip(h, u.shape))
    assert np.array_equal(a[0].cpu().numpy()[inner], cu[inner])
    assert np.array_equal(a[1].cpu().numpy()[inner], cv[inner])


def test_gray_scott_4096_kahan_step():
    torch = _torch()
    r = _gs("fp32_kahan")
    h = r.halo_widths
    u, v = D.gray_scott_init(4096, seed=2, halo=h, dtype="float32")
    rng = np.random.default_rng(6)
    cu = (rng.standard_normal(u.shape) * 1e-8).astype(np.float32)
    cv = (rng.standard_normal(u.shape) * 1e-8).astype(np.float32)
    t = [torch.from_numpy(x).cuda() for x in (u, v, cu, cv)]
    outs = [torch.full_like(t[0], float("nan")) for _ in range(4)]
    getattr(r.load_module(), f"step_{r.name}")(*t, *outs)
    torch.cuda.synchronize()
    want = O.fused_kahan_step({"u": u, "v": v}, {"u": cu, "v": cv},
                              {"u": D.gs_u_incr, "v": D.gs_v_incr}, 2, h, boundary="periodic")
    inner = tuple(slice(x, s - x) for x, s in zip(h, u.shape))
    got = [o.cpu().numpy()[inner] for o in outs]
    assert np.array_equal(got[0], want["u"][0][inner])
    assert np.array_equal(got[1], want["v"][0][inner])
    assert np.array_equal(got[2], want["u"][1][inner])
    assert np.array_equal(got[3], want["v"][1][inner])


SW_ODD = {1: (1,), 2: (0,)}   # hu flips across x walls, hv across y walls
SW_BC_ODD = (0, 2, 1)


def test_shallow_water_256_grid_mix_two_rk2_steps():
    from cutile import RKIntegrator, stencil
    from cutile import compile as stencil_compile
    from cutile.runtime.rk_runtime import RKBatch, pack_grids

    torch = _torch()
    rng = np.random.default_rng(3)
    sizes = [int(x) for x in np.rint(np.exp(rng.uniform(np.log(64), np.log(2048), 256)))]
    init = [D.sw_init(n, rng, halo=(1, 1), dtype="float32") for n in sizes]
    rk = RKIntegrator(stencil(ndim=2, dtype="float32")(D.sw_rhs), "rk2").compile(
        boundary="reflecting", align_halo=False)
    speed = stencil_compile(stencil(ndim=2, dtype="float32")(D.sw_speed), reduce="max",
                            align_halo=False)
    h = rk.info["halo"]
    assert tuple(h) == (1, 1)
    flat, states = pack_grids([g[0].shape for g in init], 3, torch.float32, torch.device("cuda"))
    for st, fields in zip(states, init):
        for dst, src in zip(st, fields):
            dst.copy_(torch.from_numpy(src))
    dx = [1.0 / n for n in sizes]
    batch = RKBatch(rk, states, [{"dx": d} for d in dx],
                    cfl=(speed.load_module().program(), dx, 0.4), bc_odd=SW_BC_ODD)
    for _ in range(2):
        batch.step()
    torch.cuda.synchronize()
    order = np.argsort(sizes)
    check = sorted(set(range(0, 256, 4)) | {int(order[0]), int(order[-1])})
    names = ["h", "hu", "hv"]
    for k in check:
        ref = tuple(a.copy() for a in init[k])
        for _ in range(2):
            dt = O.cfl_dt(D.sw_speed, ref, names, 2, h, 0.4, dx[k])
            ref = O.rk_step(D.sw_rhs, names, ref, "rk2", dt, 2, h, {"dx": dx[k]}, "reflecting", SW_ODD)
        inner = tuple(slice(x, s - x) for x, s in zip(h, init[k][0].shape))
        for f in range(3):
            got = states[k][f].cpu().numpy()
            assert np.array_equal(got[inner], ref[f][inner]), (k, sizes[k], names[f])
