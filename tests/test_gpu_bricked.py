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
