"""Bricked layout on the GPU: to_bricks / from_bricks against the reference's
reshape/transpose (restated in the oracle), launch_<name>_bricked against the
oracle's bricked launch (interior = stencil, halo = 0), and the bricked
kernel on resident bricks against the flat kernel."""

import numpy as np
import pytest

import stencil_defs as D
from oracle import stencil_oracle as O

pytestmark = pytest.mark.gpu

SHAPES = {1: [(37,), (64,)], 2: [(21, 30), (34, 66)], 3: [(11, 13, 18), (18, 18, 34)]}
FNS = {1: D.heat1d, 2: D.heat2d, 3: D.lap7}


@pytest.mark.parametrize("ndim", [1, 2, 3])
@pytest.mark.parametrize("b", [4, 8])
@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_to_from_bricks_match_the_reference_layout(ndim, b, dtype):
    import torch

    from cutile.runtime import native

    for shape in SHAPES[ndim]:
        a = np.random.default_rng(sum(shape)).random(shape).astype(dtype)
        t = torch.from_numpy(a).cuda()
        bt = native.to_bricks(t, b)
        want = O.to_bricks(a, b)
        assert tuple(bt.shape) == want.shape
        assert np.array_equal(bt.cpu().numpy(), want)
        back = native.from_bricks(bt, shape, b)
        assert np.array_equal(back.cpu().numpy(), a)


@pytest.mark.parametrize("ndim", [1, 2, 3])
@pytest.mark.parametrize("dtype", ["float64", "float32"])
@pytest.mark.parametrize("T", [1, 2])
def test_launch_bricked_matches_oracle(ndim, dtype, T):
    import torch

    from cutile import compile as stencil_compile
    from cutile import stencil

    r = stencil_compile(stencil(ndim=ndim, dtype=dtype)(FNS[ndim]), layout="bricked",
                        brick_size=8, temporal_steps=T)
    mod = r.load_module()
    launch = getattr(mod, f"launch_{r.name}_bricked")
    for shape in SHAPES[ndim]:
        u = np.random.default_rng(len(shape)).random(shape).astype(dtype)
        a = torch.from_numpy(u).cuda()
        out = torch.full_like(a, float("nan"))
        launch(a, out)
        want = O.bricked_launch(u, FNS[ndim], ndim, r.halo_widths, T)
        assert np.array_equal(out.cpu().numpy(), want), shape


@pytest.mark.parametrize("ndim", [2, 3])
def test_resident_bricks_equal_flat_kernel(ndim):
    import torch

    from cutile import compile as stencil_compile
    from cutile import stencil

    r = stencil_compile(stencil(ndim=ndim)(FNS[ndim]), layout="bricked", brick_size=8,
                        temporal_blocking=False)
    mod = r.load_module()
    shape = SHAPES[ndim][1]
    u = np.random.default_rng(3).random(shape)
    a = torch.from_numpy(u).cuda()
    flat_out = torch.zeros_like(a)
    getattr(mod, f"launch_{r.name}")(a, flat_out)
    ab = mod.to_bricks(a)
    ob = torch.full_like(ab, 7.0)
    getattr(mod, f"launch_{r.name}_on_bricks")(ab, ob, shape)
    got = mod.from_bricks(ob, shape).cpu().numpy()
    inner = tuple(slice(1, s - 1) for s in shape)
    assert np.array_equal(got[inner], flat_out.cpu().numpy()[inner])
    # cells outside the interior are not written
    halo_mask = np.ones(shape, bool)
    halo_mask[inner] = False
    assert (got[halo_mask] == 7.0).all()


@pytest.mark.parametrize("dtype", ["float64", "float32"])
@pytest.mark.parametrize("b", [4, 8, 16])
@pytest.mark.parametrize("shape", [(18, 18, 34), (21, 19, 45), (9, 40, 70)])
def test_bricked_tma_staging_equals_cp_async_and_flat(dtype, b, shape):
    """Bricks staged by 5-D tensor copies (whole-brick rows, tiles on brick
    boundaries) give the bits of the per-group cp.async staging and of the
    flat kernel, on shapes that are not whole bricks."""
    import torch

    from cutile import compile as stencil_compile
    from cutile import stencil
    from cutile.runtime import native

    r = stencil_compile(stencil(ndim=3, dtype=dtype)(D.lap7), layout="bricked", brick_size=b,
                        temporal_blocking=False)
    mod = r.load_module()
    prog = mod.program()
    assert prog.kernel("bricked").desc["brick_tma"] == 1
    u = np.random.default_rng(sum(shape) + b).random(shape).astype(dtype)
    a = torch.from_numpy(u).cuda()
    flat_out = torch.zeros_like(a)
    getattr(mod, f"launch_{r.name}")(a, flat_out)
    ab = mod.to_bricks(a)
    outs = []
    for loader in (native.CSD_LOADER_TMA, native.CSD_LOADER_LDG):
        ob = torch.full_like(ab, 7.0)
        prog.launch_on_bricks((ab,), (ob,), shape, loader=loader)
        outs.append(mod.from_bricks(ob, shape).cpu().numpy())
    torch.cuda.synchronize()
    inner = tuple(slice(1, s - 1) for s in shape)
    assert np.array_equal(outs[0], outs[1])
    assert np.array_equal(outs[0][inner], flat_out.cpu().numpy()[inner])
    want = O.apply_stencil(u, D.lap7, 3, (1, 1, 1))
    assert np.array_equal(outs[0][inner], want[inner])
    halo_mask = np.ones(shape, bool)
    halo_mask[inner] = False
    assert (outs[0][halo_mask] == 7.0).all()
    assert native.error_word(reset=True) == 0


def test_bricked_box27_tma_staging():
    """A 27-point box (corner reads across brick rows) on TMA-staged bricks."""
    import tempfile

    import torch

    import ref_corpus as RC
    from cutile import compile as stencil_compile
    from cutile.runtime import native

    entries, _ = RC.load()
    with tempfile.TemporaryDirectory() as tmp:
        fn = RC.build(tmp, "wide_stencils/box27", entries["wide_stencils/box27"])
    r = stencil_compile(fn, layout="bricked", brick_size=8, temporal_blocking=False)
    mod = r.load_module()
    shape = (20, 27, 53)
    u = np.random.default_rng(5).random(shape)
    ab = mod.to_bricks(torch.from_numpy(u).cuda())
    ob = torch.zeros_like(ab)
    getattr(mod, f"launch_{r.name}_on_bricks")(ab, ob, shape)
    got = mod.from_bricks(ob, shape).cpu().numpy()
    want = O.apply_stencil(u, fn, 3, (1, 1, 1))
    inner = tuple(slice(1, s - 1) for s in shape)
    assert np.array_equal(got[inner], want[inner])
    assert native.error_word(reset=True) == 0


@pytest.mark.parametrize("dtype", ["float64", "float32"])
@pytest.mark.parametrize("loader", [-1, 1])
def test_brick_sized_halo_starts_the_interior_on_a_brick(dtype, loader):
    """A field stored with a zero halo of one brick per side (the bench's
    bricked layout), launched with ``halo=``: the interior, 13 x 37 x 150
    cells from offset 8, equals the oracle's stencil on the same array;
    nothing outside the interior is written."""
    import torch

    from cutile import compile as stencil_compile
    from cutile import stencil

    r = stencil_compile(stencil(ndim=3, dtype=dtype)(D.lap7), layout="bricked", brick_size=8,
                        temporal_blocking=False)
    assert r.halo_widths == (1, 1, 1)
    halo = (8, 8, 8)
    inner_n = (13, 37, 150)
    shape = tuple(n + 2 * h for n, h in zip(inner_n, halo))
    u = np.zeros(shape, dtype=dtype)
    inner = tuple(slice(h, s - h) for h, s in zip(halo, shape))
    u[inner] = np.random.default_rng(21).standard_normal(inner_n).astype(dtype)
    mod = r.load_module()
    ab = mod.to_bricks(torch.from_numpy(u).cuda())
    ob = torch.full_like(ab, 7.0)
    r.load_module().program().launch_on_bricks((ab,), (ob,), shape, loader=loader, halo=halo)
    got = mod.from_bricks(ob, shape).cpu().numpy()
    want = O.apply_stencil(u, D.lap7, 3, halo)
    assert np.array_equal(got[inner], want[inner])
    mask = np.ones(shape, bool)
    mask[inner] = False
    assert np.all(got[mask] == 7.0)
