"""GPU parity: the sm_100a kernels against the CPU oracle, bit for bit.

Every kernel here runs through the public path (``cutile.compile`` ->
``load_module().launch_<name>`` -> libcsd).  Outputs start as NaN so a write
outside the interior is caught (the halo must stay untouched).
"""

import numpy as np
import pytest

import random_exprs
import stencil_defs as D
from oracle import stencil_oracle as O

pytestmark = pytest.mark.gpu


def _torch():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch


def _stencil(fn, ndim, **kw):
    from cutile import stencil

    return stencil(ndim=ndim, **kw)(fn)


def _run(result, arrays, n_out=1, nan_out=True):
    torch = _torch()
    mod = result.load_module()
    launch = getattr(mod, f"launch_{result.name}")
    ins = [torch.from_numpy(a).cuda() for a in arrays]
    outs = [torch.full_like(ins[0], float("nan")) if nan_out else torch.zeros_like(ins[0])
            for _ in range(n_out)]
    launch(*ins, *outs)
    torch.cuda.synchronize()
    return [o.cpu().numpy() for o in outs]


def _interior(shape, halo):
    return tuple(slice(h, s - h) for h, s in zip(halo, shape))


def _check_halo_untouched(out, halo):
    mask = np.ones(out.shape, bool)
    mask[_interior(out.shape, halo)] = False
    assert np.all(np.isnan(out[mask])), "kernel wrote outside the interior"


def _error_word_clear():
    from cutile.runtime import native

    assert native.error_word(reset=True) == 0


SIZES = {1: (300,), 2: (45, 77), 3: (19, 14, 37)}


@pytest.mark.parametrize("align_halo", [True, False])
@pytest.mark.parametrize("name", sorted(D.CASES))
def test_named_cases_bit_exact(name, align_halo):
    import cutile

    fn, ndim, nin = D.CASES[name]
    r = cutile.compile(_stencil(fn, ndim), temporal_blocking=False, align_halo=align_halo)
    shape = tuple(s + 2 * h for s, h in zip(SIZES[ndim], r.halo_widths))
    rng = np.random.default_rng(hash(name) % 1000)
    ins = [rng.random(shape) + 0.25 for _ in range(nin)]
    (got,) = _run(r, ins)
    want = O.apply_multi(ins, fn, ndim, r.halo_widths)
    inner = _interior(shape, r.halo_widths)
    assert np.array_equal(got[inner], want[inner])
    _check_halo_untouched(got, r.halo_widths)
    _error_word_clear()


@pytest.mark.parametrize("seed", range(40))
def test_random_expressions_bit_exact(tmp_path, seed):
    import cutile

    ndim, nfields, radius, fields, idx, body = random_exprs.case(seed)
    fn = random_exprs.build(tmp_path, f"g{seed}", fields, idx, body)
    used = random_exprs.used_fields(body, fields)
    r = cutile.compile(fn, temporal_blocking=False, align_halo=bool(seed % 2))
    assert r.inputs == tuple(used)
    rng = np.random.default_rng(seed)
    shape = tuple(9 + 2 * h + seed % 5 for h in r.halo_widths)
    ins = {f: rng.random(shape) + 0.5 for f in used}
    (got,) = _run(r, [ins[f] for f in used])
    want = O.evaluate(ins, fn._fn, ndim, r.halo_widths, shape, np.float64)
    inner = _interior(shape, r.halo_widths)
    assert np.array_equal(got[inner], np.broadcast_to(want, got[inner].shape)), body


@pytest.mark.parametrize("loader", [0, 1])
def test_tma_and_cp_async_loaders_agree(loader):
    import cutile

    torch = _torch()
    r = cutile.compile(_stencil(D.lap7, 3), temporal_blocking=False, align_halo=False)
    rng = np.random.default_rng(3)
    u = rng.standard_normal((34, 18, 66))
    prog = r.load_module().program()
    tin = torch.from_numpy(u).cuda()
    tout = torch.full_like(tin, float("nan"))
    prog.launch((tin,), (tout,), loader=loader)
    torch.cuda.synchronize()
    got = tout.cpu().numpy()
    want = O.apply_stencil(u, D.lap7, 3, (1, 1, 1))
    assert np.array_equal(got[1:-1, 1:-1, 1:-1], want[1:-1, 1:-1, 1:-1])
    _check_halo_untouched(got, (1, 1, 1))


def test_unaligned_pitch_uses_cp_async_path():
    """FP32 rows of 514 elements (2056 B) cannot use TMA; results still exact."""
    import cutile

    r = cutile.compile(_stencil(D.lap7, 3, dtype="float32"), temporal_blocking=False,
                       align_halo=False)
    rng = np.random.default_rng(4)
    u = rng.standard_normal((20, 11, 514)).astype(np.float32)
    (got,) = _run(r, [u])
    want = O.apply_stencil(u, D.lap7, 3, (1, 1, 1))
    assert want.dtype == np.float32
    assert np.array_equal(got[1:-1, 1:-1, 1:-1], want[1:-1, 1:-1, 1:-1])


@pytest.mark.parametrize("zchunk", [1, 3, 64])
def test_work_item_chunking(zchunk):
    import cutile

    torch = _torch()
    r = cutile.compile(_stencil(D.lap7, 3), temporal_blocking=False, align_halo=False)
    u = np.random.default_rng(5).standard_normal((23, 13, 30))
    prog = r.load_module().program()
    tin = torch.from_numpy(u).cuda()
    tout = torch.full_like(tin, float("nan"))
    prog.launch((tin,), (tout,), zchunk=zchunk, grid=3)
    torch.cuda.synchronize()
    want = O.apply_stencil(u, D.lap7, 3, (1, 1, 1))
    assert np.array_equal(tout.cpu().numpy()[1:-1, 1:-1, 1:-1], want[1:-1, 1:-1, 1:-1])


def test_heat_1024_100_steps_ping_pong():
    """2-D heat 5-point FP64, 1024^2 interior, zero halo, seed 0, 100 steps."""
    import cutile

    torch = _torch()
    r = cutile.compile(_stencil(D.heat2d, 2), align_halo=False, temporal_blocking=False)
    u0 = np.zeros((1026, 1026))
    u0[1:-1, 1:-1] = np.random.default_rng(0).random((1024, 1024))
    launch = getattr(r.load_module(), "launch_heat2d")
    a = torch.from_numpy(u0).cuda()
    b = torch.zeros_like(a)
    for _ in range(100):
        launch(a, b)
        a, b = b, a
    torch.cuda.synchronize()
    want = O.time_march(u0, D.heat2d, 2, (1, 1), 100)[-1]
    assert np.array_equal(a.cpu().numpy(), want)


@pytest.mark.parametrize("name,ndim,T", [("heat2d", 2, None), ("heat1d", 1, None),
                                          ("lap7", 3, 2), ("lap7", 3, 3), ("lap7", 3, 4),
                                          ("lap7", 3, 8), ("heat2d", 2, 4), ("heat2d", 2, 8),
                                          ("lap4_1d", 1, 3), ("wave4", 2, 2), ("wave4", 2, 4)])
def test_temporal_blocking_matches_T_launches(name, ndim, T):
    import cutile

    fn = D.CASES[name][0]
    r = cutile.compile(_stencil(fn, ndim), temporal_steps=T, align_halo=False)
    assert r.temporal_steps >= 2
    sizes = {1: (401,), 2: (61, 90), 3: (21, 17, 46)}
    shape = tuple(s + 2 * h for s, h in zip(sizes[ndim], r.halo_widths))
    u = np.random.default_rng(7).standard_normal(shape)
    (got,) = _run(r, [u])
    want = O.temporal_launch(u, np.full(shape, np.nan), fn, ndim, r.halo_widths, r.temporal_steps)
    inner = _interior(shape, r.halo_widths)
    assert np.array_equal(got[inner], want[inner])
    _check_halo_untouched(got, r.halo_widths)


@pytest.mark.parametrize("kind", ["dirichlet", "neumann", "periodic", "reflecting"])
@pytest.mark.parametrize("ndim", [1, 2, 3])
def test_apply_boundary_matches_oracle(kind, ndim):
    import cutile

    torch = _torch()
    fn = {1: D.heat1d, 2: D.heat2d, 3: D.lap7}[ndim]
    bnd = {"type": kind, "value": 0.5} if kind == "dirichlet" else kind
    r = cutile.compile(_stencil(fn, ndim, boundary=bnd), temporal_blocking=False)
    shape = tuple(s + 2 * h for s, h in zip(SIZES[ndim], r.halo_widths))
    u = np.random.default_rng(8).standard_normal(shape)
    t = torch.from_numpy(u).cuda()
    getattr(r.load_module(), f"apply_boundary_{r.name}")(t)
    torch.cuda.synchronize()
    want = u.copy()
    O.apply_boundary(want, O.uniform_spec(kind, ndim, 0.5), r.halo_widths)
    assert np.array_equal(t.cpu().numpy(), want)


@pytest.mark.parametrize("kind", ["dirichlet", "neumann", "periodic", "reflecting"])
@pytest.mark.parametrize("name", ["heat2d", "lap7", "heat1d", "gs_u"])
def test_fused_boundary_step(kind, name):
    import cutile

    fn, ndim, nin = D.CASES[name]
    bnd = {"type": kind, "value": -0.25} if kind == "dirichlet" else kind
    r = cutile.compile(_stencil(fn, ndim, boundary=bnd), temporal_blocking=False,
                       align_halo=(name != "lap7"))
    shape = tuple(s + 2 * h for s, h in zip(SIZES[ndim], r.halo_widths))
    rng = np.random.default_rng(9)
    ins = [rng.random(shape) for _ in range(nin)]
    torch = _torch()
    tin = [torch.from_numpy(a).cuda() for a in ins]
    tout = torch.full_like(tin[0], float("nan"))
    getattr(r.load_module(), f"step_{r.name}")(*tin, tout)
    torch.cuda.synchronize()
    want = O.stencil_with_boundary(ins, fn, ndim, r.halo_widths, kind, -0.25)
    inner = _interior(shape, r.halo_widths)
    assert np.array_equal(tout.cpu().numpy()[inner], want[inner])
    for a, t in zip(ins, tin):  # inputs are not modified
        assert np.array_equal(t.cpu().numpy(), a)


@pytest.mark.parametrize("kind", ["dirichlet", "neumann", "periodic", "reflecting"])
@pytest.mark.parametrize("name,size", [("heat2d", (300, 700)), ("gs_u", (257, 1030)),
                                       ("lap7", (26, 14, 522))])
def test_fused_boundary_step_uneven_split(kind, name, size):
    """Grids wide enough for the fused-boundary work split (shorter X-edge
    items from the wave's spare slots, shorter first/last items)."""
    import cutile

    fn, ndim, nin = D.CASES[name]
    bnd = {"type": kind, "value": -0.25} if kind == "dirichlet" else kind
    r = cutile.compile(_stencil(fn, ndim, boundary=bnd), temporal_blocking=False)
    shape = tuple(s + 2 * h for s, h in zip(size, r.halo_widths))
    rng = np.random.default_rng(19)
    ins = [rng.random(shape) for _ in range(nin)]
    torch = _torch()
    tin = [torch.from_numpy(a).cuda() for a in ins]
    tout = torch.full_like(tin[0], float("nan"))
    getattr(r.load_module(), f"step_{r.name}")(*tin, tout)
    torch.cuda.synchronize()
    want = O.stencil_with_boundary(ins, fn, ndim, r.halo_widths, kind, -0.25)
    inner = _interior(shape, r.halo_widths)
    assert np.array_equal(tout.cpu().numpy()[inner], want[inner])


def test_compile_fused_gray_scott():
    import cutile

    a = _stencil(D.gs_u, 2)
    b = _stencil(D.gs_v, 2)
    r = cutile.compile_fused([a, b])
    assert r.inputs == ("u", "v") and r.outputs == ("gs_u", "gs_v")
    shape = (70 + 2, 50 + 2 * r.halo_widths[1])
    rng = np.random.default_rng(10)
    u, v = rng.random(shape), rng.random(shape)
    got = _run(r, [u, v], n_out=2)
    want = O.fused_apply({"u": u, "v": v}, [D.gs_u, D.gs_v], 2, r.halo_widths)
    inner = _interior(shape, r.halo_widths)
    for g, w in zip(got, want):
        assert np.array_equal(g[inner], w[inner])


def test_compile_fused_merges_inputs_by_name():
    import cutile

    def fa(u, v, i, j):
        return u[i + 1, j] + 0.3 * v[i, j]

    def fb(v, w, i, j):
        return 0.3 * v[i, j] - w[i, j - 1]

    r = cutile.compile_fused([_stencil(fa, 2), _stencil(fb, 2)])
    assert r.inputs == ("u", "v", "w")
    shape = (30, 40 + 2 * r.halo_widths[1])
    rng = np.random.default_rng(11)
    arrs = {n: rng.random(shape) for n in "uvw"}
    got = _run(r, [arrs[n] for n in "uvw"], n_out=2)
    want = O.fused_apply(arrs, [fa, fb], 2, r.halo_widths)
    inner = _interior(shape, r.halo_widths)
    for g, w in zip(got, want):
        assert np.array_equal(g[inner], w[inner])


@pytest.mark.parametrize("name", ["lap7", "heat2d", "cond3d", "clip1d", "gs_u"])
def test_float32_bit_exact_with_numpy_float32(name):
    import cutile

    fn, ndim, nin = D.CASES[name]
    r = cutile.compile(_stencil(fn, ndim, dtype="float32"), temporal_blocking=False)
    shape = tuple(s + 2 * h for s, h in zip(SIZES[ndim], r.halo_widths))
    rng = np.random.default_rng(12)
    ins = [(rng.random(shape) - 0.3).astype(np.float32) for _ in range(nin)]
    (got,) = _run(r, ins)
    want = O.apply_multi(ins, fn, ndim, r.halo_widths)
    assert want.dtype == np.float32
    inner = _interior(shape, r.halo_widths)
    assert np.array_equal(got[inner], want[inner])


def test_validate_and_benchmark_api():
    import cutile

    r = cutile.compile(_stencil(D.heat2d, 2))
    assert r.validate(atol=1e-12)
    b = r.benchmark(iters=3, warmup=1)
    assert b["time_ms"] > 0 and b["gpoints_per_s"] > 0


@pytest.mark.parametrize("dtype", ["float64", "float32"])
@pytest.mark.parametrize("T", [2, 4, 8])
def test_3d_chain_default_tiles_over_ragged_columns(dtype, T):
    """The 3-D chain defaults (tiles up to 32 x 64, up to 512 threads) over a
    grid of several ragged column tiles, both dtypes, bit-exact against T
    oracle steps."""
    import cutile

    r = cutile.compile(_stencil(D.lap7, 3, dtype=dtype), temporal_steps=T, align_halo=False)
    assert r.temporal_steps == T
    shape = tuple(s + 2 * h for s, h in zip((11, 37, 141), r.halo_widths))
    u = np.random.default_rng(13).standard_normal(shape).astype(dtype)
    (got,) = _run(r, [u])
    want = O.temporal_launch(u, np.full(shape, np.nan, dtype=dtype), D.lap7, 3, r.halo_widths, T)
    assert want.dtype == np.dtype(dtype)
    inner = _interior(shape, r.halo_widths)
    assert np.array_equal(got[inner], want[inner])
    _check_halo_untouched(got, r.halo_widths)


@pytest.mark.parametrize("dtype", ["float64", "float32"])
@pytest.mark.parametrize("T", [2, 3, 5, 8])
def test_2d_chain_default_chunks_over_ragged_columns(dtype, T):
    """The 2-D chain defaults per depth and dtype (4 or 8 rows by 64 or 128
    columns, 128 or 256 threads) over several ragged column tiles."""
    import cutile

    r = cutile.compile(_stencil(D.heat2d, 2, dtype=dtype), temporal_steps=T, align_halo=False)
    assert r.temporal_steps == T
    shape = tuple(s + 2 * h for s, h in zip((75, 301), r.halo_widths))
    u = np.random.default_rng(14).standard_normal(shape).astype(dtype)
    (got,) = _run(r, [u])
    want = O.temporal_launch(u, np.full(shape, np.nan, dtype=dtype), D.heat2d, 2, r.halo_widths, T)
    inner = _interior(shape, r.halo_widths)
    assert np.array_equal(got[inner], want[inner])
    _check_halo_untouched(got, r.halo_widths)


@pytest.mark.parametrize("name,ndim,dtype,tile,vec,threads", [
    ("lap7", 3, "float32", (2, 8, 128), 8, 128), ("lap7", 3, "float64", (1, 4, 128), 4, 64),
    ("heat2d", 2, "float64", (8, 128), 4, 128), ("heat2d", 2, "float32", (16, 128), 8, 128)])
def test_wider_units_are_bit_exact(name, ndim, dtype, tile, vec, threads):
    """Units of two 16-byte vectors (``kernel_hints={"vec": ...}``) over
    ragged column tiles: same bits as the oracle, halo untouched."""
    import cutile

    fn = D.CASES[name][0]
    r = cutile.compile(_stencil(fn, ndim, dtype=dtype), temporal_blocking=False,
                       tile_sizes=tile, kernel_hints={"vec": vec, "threads": threads})
    assert r.kernel_hints["vec"] == vec
    size = {3: (13, 37, 150), 2: (75, 301)}[ndim]
    shape = tuple(s + 2 * h for s, h in zip(size, r.halo_widths))
    u = np.random.default_rng(5).standard_normal(shape).astype(dtype)
    (got,) = _run(r, [u])
    want = O.apply_stencil(u, fn, ndim, r.halo_widths)
    inner = _interior(shape, r.halo_widths)
    assert np.array_equal(got[inner], want[inner])
    _check_halo_untouched(got, r.halo_widths)


@pytest.mark.parametrize("defines", [("-DCSD_CHAIN_SKEW=0",), ("-DCSD_UNROLL_RAGGED=0",),
                                     ("-DCSD_UNROLL_UNITS=0",)])
@pytest.mark.parametrize("name,ndim,T", [("lap7", 3, 2), ("heat2d", 2, 4)])
def test_engine_schedule_switches_keep_chains_exact(monkeypatch, defines, name, ndim, T):
    """The engine's alternative schedules (per-stage barriers instead of the
    skewed chain, loop instead of unrolled units) compute the same bits."""
    import cutile
    from cutile.runtime import native

    monkeypatch.setattr(native, "NVRTC_OPTIONS", native.NVRTC_OPTIONS + tuple(defines))
    fn = D.CASES[name][0]
    r = cutile.compile(_stencil(fn, ndim), temporal_steps=T, align_halo=False)
    sizes = {2: (61, 90), 3: (21, 17, 46)}
    shape = tuple(s + 2 * h for s, h in zip(sizes[ndim], r.halo_widths))
    u = np.random.default_rng(7).standard_normal(shape)
    (got,) = _run(r, [u])
    want = O.temporal_launch(u, np.full(shape, np.nan), fn, ndim, r.halo_widths, T)
    inner = _interior(shape, r.halo_widths)
    assert np.array_equal(got[inner], want[inner])
    _check_halo_untouched(got, r.halo_widths)
