"""FP32 and Kahan-compensated FP32 modes (Gray-Scott, periodic, fused u/v)."""

import numpy as np
import pytest

import stencil_defs as D
from oracle import stencil_oracle as O

pytestmark = pytest.mark.gpu


def _fused(precision, boundary="periodic"):
    import cutile
    from cutile import stencil

    return cutile.compile_fused([stencil(ndim=2)(D.gs_u), stencil(ndim=2)(D.gs_v)],
                                precision=precision, boundary=boundary)


@pytest.mark.parametrize("n", [96, 700])
def test_kahan_step_bit_exact_against_numpy_float32(n):
    """n = 700 is wide enough for the fused-boundary work split."""
    import torch

    r = _fused("fp32_kahan")
    assert r.inputs == ("u", "v", "c_u", "c_v")
    h = r.halo_widths
    u, v = D.gray_scott_init(n, seed=5, halo=h, dtype="float32")
    rng = np.random.default_rng(6)
    cu = (rng.standard_normal(u.shape) * 1e-8).astype(np.float32)
    cv = (rng.standard_normal(u.shape) * 1e-8).astype(np.float32)
    t = [torch.from_numpy(a).cuda() for a in (u, v, cu, cv)]
    outs = [torch.full_like(t[0], float("nan")) for _ in range(4)]
    r.load_module().step_gs_u_gs_v(*t, *outs)
    torch.cuda.synchronize()
    want = O.fused_kahan_step({"u": u, "v": v}, {"u": cu, "v": cv},
                              {"u": D.gs_u_incr, "v": D.gs_v_incr}, 2, h, boundary="periodic")
    inner = tuple(slice(x, s - x) for x, s in zip(h, u.shape))
    got = [o.cpu().numpy()[inner] for o in outs]
    assert np.array_equal(got[0], want["u"][0][inner])
    assert np.array_equal(got[1], want["v"][0][inner])
    assert np.array_equal(got[2], want["u"][1][inner])
    assert np.array_equal(got[3], want["v"][1][inner])


def _run(r, u, v, steps, kahan=False):
    import torch

    mod = r.load_module()
    step = getattr(mod, f"step_{r.name}")
    a = [torch.from_numpy(u).cuda(), torch.from_numpy(v).cuda()]
    b = [torch.zeros_like(a[0]), torch.zeros_like(a[1])]
    if kahan:
        ca = [torch.zeros_like(a[0]), torch.zeros_like(a[1])]
        cb = [torch.zeros_like(a[0]), torch.zeros_like(a[1])]
    for _ in range(steps):
        if kahan:
            step(*a, *ca, *b, *cb)
            ca, cb = cb, ca
        else:
            step(*a, *b)
        a, b = b, a
    torch.cuda.synchronize()
    return [x.cpu().numpy().astype(np.float64) for x in a]


def test_fp64_gray_scott_matches_numpy_over_50_steps():
    r = _fused("fp64")
    h = r.halo_widths
    u, v = D.gray_scott_init(128, seed=2, halo=h)
    got = _run(r, u, v, 50)
    cu, cv = u.copy(), v.copy()
    for _ in range(50):
        o = O.stencil_with_boundary([cu, cv], D.gs_u, 2, h, "periodic")
        p = O.stencil_with_boundary([cu, cv], D.gs_v, 2, h, "periodic")
        cu, cv = o, p
    inner = tuple(slice(x, s - x) for x, s in zip(h, u.shape))
    assert np.array_equal(got[0][inner], cu[inner])
    assert np.array_equal(got[1][inner], cv[inner])


def test_kahan_error_against_fp64_is_reported():
    """Relative L2 of FP32 and FP32+Kahan against the FP64 run (GPU FP64 is
    bit-exact to NumPy, so it serves as the long-run oracle).  Gray-Scott
    amplifies state perturbations, so compensated summation (which removes
    the accumulation drift, not the FP32 state rounding) stays at the FP32
    level here; the bound is the FP32 one."""
    steps = 2000
    r64 = _fused("fp64")
    h = r64.halo_widths
    u, v = D.gray_scott_init(256, seed=2, halo=h)
    ref = _run(r64, u, v, steps)
    r32 = _fused("fp32")
    rk = _fused("fp32_kahan")
    h32 = r32.halo_widths
    u32, v32 = D.gray_scott_init(256, seed=2, halo=h32, dtype="float32")
    plain = _run(r32, u32, v32, steps)
    comp = _run(rk, u32, v32, steps, kahan=True)
    i64 = tuple(slice(x, s - x) for x, s in zip(h, u.shape))
    i32 = tuple(slice(x, s - x) for x, s in zip(h32, u32.shape))

    def rel(a, b):
        return float(np.linalg.norm(a - b) / np.linalg.norm(b))

    e_plain = rel(plain[0][i32], ref[0][i64])
    e_kahan = rel(comp[0][i32], ref[0][i64])
    print(f"rel L2 after {steps} steps: fp32 {e_plain:.3e}, fp32+kahan {e_kahan:.3e}")
    assert e_plain < 1e-4 and e_kahan < 1e-4


@pytest.mark.parametrize("precision", ["fp64", "fp32_kahan"])
def test_captured_time_loop_equals_eager_steps(precision):
    """A CUDA graph of ping-pong fused steps gives the eager loop's bits."""
    import torch

    r = _fused(precision)
    h = r.halo_widths
    dt = "float64" if precision == "fp64" else "float32"
    u, v = D.gray_scott_init(100, seed=3, halo=h, dtype=dt)
    prog = r.load_module().program()
    n = prog.spec["inputs"]

    def fresh():
        f = [torch.from_numpy(u).cuda(), torch.from_numpy(v).cuda()]
        f += [torch.zeros_like(f[0]) for _ in range(n - 2)]
        return f, [torch.zeros_like(f[0]) for _ in range(n)]

    a, b = fresh()
    graph = prog.capture_steps(a, b, 6, boundary=True)
    graph.replay()
    graph.replay()
    ea, eb = fresh()
    for _ in range(12):
        prog.step(ea, eb)
        ea, eb = eb, ea
    torch.cuda.synchronize()
    for x, y in zip(a, ea):
        assert torch.equal(x, y)


def _heat(precision):
    import cutile
    from cutile import stencil

    dt = "float64" if precision == "fp64" else "float32"
    return cutile.compile(stencil(ndim=2, dtype=dt)(D.heat_small_dt), precision=precision,
                          temporal_blocking=False)


def _heat_run(r, u, steps, kahan):
    import torch

    launch = getattr(r.load_module(), f"launch_{r.name}")
    a, b = torch.from_numpy(u).cuda(), torch.zeros(u.shape, dtype=torch.from_numpy(u).dtype,
                                                     device="cuda")
    ca, cb = torch.zeros_like(a), torch.zeros_like(a)
    for _ in range(steps):
        if kahan:
            launch(a, ca, b, cb)
            ca, cb = cb, ca
        else:
            launch(a, b)
        a, b = b, a
    torch.cuda.synchronize()
    return a.cpu().numpy().astype(np.float64), ca.cpu().numpy()


def test_kahan_heat_steps_bit_exact_against_numpy_float32():
    r = _heat("fp32_kahan")
    h = r.halo_widths
    u = D.heat_bump_init(200, halo=h, dtype="float32")
    got, gc = _heat_run(r, u, 5, True)
    want = u.copy()
    c = np.zeros_like(u)
    inner = tuple(slice(x, s - x) for x, s in zip(h, u.shape))
    for _ in range(5):
        inc = O.evaluate_ops({"u": want}, _increment_of_heat, 2, h, u.shape, np.float32)[0]
        nu, nc = O.kahan_update(want[inner], c[inner], inc)
        want[inner], c[inner] = nu, nc
    assert np.array_equal(got[inner].astype(np.float32), want[inner])
    assert np.array_equal(gc[inner], c[inner])


def _increment_of_heat(u, i, j):
    return D.KD_HEAT * (u[i - 1, j] + u[i + 1, j] + u[i, j - 1] + u[i, j + 1] - 4.0 * u[i, j])


def test_kahan_cuts_small_step_heat_error_against_fp64():
    """Small-step heat diffusion (each update ~1e-4 of u): FP32 updates lose
    the increments' low bits every step, the compensated update keeps them.
    After 10k steps on 256^2 the FP32+Kahan field is within 1e-6 (relative
    L2) of the FP64 field and at least 20x closer than plain FP32."""
    steps = 10000
    r64, r32, rk = _heat("fp64"), _heat("fp32"), _heat("fp32_kahan")
    h = r64.halo_widths
    ref, _ = _heat_run(r64, D.heat_bump_init(256, halo=h), steps, False)
    h32 = r32.halo_widths
    plain, _ = _heat_run(r32, D.heat_bump_init(256, halo=h32, dtype="float32"), steps, False)
    comp, _ = _heat_run(rk, D.heat_bump_init(256, halo=rk.halo_widths, dtype="float32"), steps,
                        True)
    i64 = tuple(slice(x, s - x) for x, s in zip(h, ref.shape))
    i32 = tuple(slice(x, s - x) for x, s in zip(h32, plain.shape))
    ik = tuple(slice(x, s - x) for x, s in zip(rk.halo_widths, comp.shape))

    def rel(a, b):
        return float(np.linalg.norm(a - b) / np.linalg.norm(b))

    e32, ek = rel(plain[i32], ref[i64]), rel(comp[ik], ref[i64])
    print(f"heat, {steps} steps: rel L2 vs FP64: fp32 {e32:.3e}, fp32+kahan {ek:.3e}")
    assert ek < 1e-6 and ek * 20 < e32


@pytest.mark.parametrize("T", [2, 4])
def test_kahan_temporal_chain_keeps_compensation_on_chip(T):
    """T compensated heat steps in one pass: u and its compensation both stay
    in shared memory between the chained steps (32 B per point per launch,
    so 32/T per step), bit-exact against T chained oracle Kahan steps; with
    a zero Dirichlet halo that also equals T separate single-step launches."""
    import torch

    import cutile
    from cutile import stencil

    fn = stencil(ndim=2, dtype="float32")(D.heat_small_dt)
    r = cutile.compile(fn, precision="fp32_kahan", temporal_steps=T)
    assert r.temporal_steps == T
    h = r.halo_widths
    u = D.heat_bump_init(300, halo=h, dtype="float32")
    c = (np.random.default_rng(9).standard_normal(u.shape) * 1e-9).astype(np.float32)
    inner = tuple(slice(x, s - x) for x, s in zip(h, u.shape))
    t = [torch.from_numpy(x).cuda() for x in (u, c)]
    outs = [torch.full_like(t[0], float("nan")) for _ in range(2)]
    getattr(r.load_module(), f"launch_{r.name}")(*t, *outs)
    torch.cuda.synchronize()
    want_u, want_c = O.kahan_temporal_launch(u, c, _increment_of_heat, 2, h, T)
    got_u, got_c = (o.cpu().numpy() for o in outs)
    assert np.array_equal(got_u[inner], want_u[inner])
    assert np.array_equal(got_c[inner], want_c[inner])
    # T single-step launches through zero-halo buffers give the same bits
    r1 = cutile.compile(fn, precision="fp32_kahan", temporal_blocking=False)
    launch1 = getattr(r1.load_module(), f"launch_{r1.name}")
    a = [torch.from_numpy(x).cuda() for x in (u, c)]
    for _ in range(T):
        b = [torch.zeros_like(a[0]), torch.zeros_like(a[0])]
        launch1(*a, *b)
        a = b
    torch.cuda.synchronize()
    assert np.array_equal(a[0].cpu().numpy()[inner], got_u[inner])
    assert np.array_equal(a[1].cpu().numpy()[inner], got_c[inner])
