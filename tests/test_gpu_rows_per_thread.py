"""Plans with several Y rows per thread (3-D): a thread evaluates RPY rows of
VEC points and reads each staged strip once for every row that needs it.
Results must equal the oracle bit for bit, including Y extents that are not
a multiple of the rows per unit, fused boundaries and the bricked layout."""

import numpy as np
import pytest

import stencil_defs as D
import wide_defs as W
from oracle import stencil_oracle as O

pytestmark = pytest.mark.gpu

PLANS = [(2, (1, 8, 64)), (4, (1, 16, 64)), (2, (2, 4, 128))]


def _interior(shape, halo):
    return tuple(slice(h, s - h) for h, s in zip(halo, shape))


def _launch(r, arrays, step=False):
    import torch

    mod = r.load_module()
    fn = getattr(mod, f"{'step' if step else 'launch'}_{r.name}")
    tin = [torch.from_numpy(a).cuda() for a in arrays]
    tout = torch.full_like(tin[0], float("nan"))
    fn(*tin, tout)
    torch.cuda.synchronize()
    return tout.cpu().numpy()


@pytest.mark.parametrize("rpy,tile", PLANS)
@pytest.mark.parametrize("dtype", ["float64", "float32"])
@pytest.mark.parametrize("size", [(21, 30, 70), (9, 17, 130)])
def test_lap7_rows_per_thread(rpy, tile, dtype, size):
    import cutile
    from cutile import stencil

    r = cutile.compile(stencil(ndim=3, dtype=dtype)(D.lap7), temporal_blocking=False,
                       tile_sizes=tile, kernel_hints={"rows_per_thread": rpy, "threads": 128})
    vec = 4 if dtype == "float32" else 2
    assert f", {rpy}, {vec}> Cfg_lap7_tma" in r.cuda_source   # RPY, VEC
    shape = tuple(s + 2 * h for s, h in zip(size, r.halo_widths))
    u = np.random.default_rng(sum(size) + rpy).standard_normal(shape).astype(dtype)
    got = _launch(r, [u])
    want = O.apply_stencil(u, D.lap7, 3, r.halo_widths)
    inner = _interior(shape, r.halo_widths)
    assert np.array_equal(got[inner], want[inner])
    mask = np.ones(shape, bool)
    mask[inner] = False
    assert np.all(np.isnan(got[mask]))


@pytest.mark.parametrize("rpy,tile", PLANS[:2])
def test_box27_rows_per_thread(tmp_path, rpy, tile):
    import cutile

    fn = W.load_box("box27_rpy", 1, directory=str(tmp_path))
    r = cutile.compile(fn, temporal_blocking=False, tile_sizes=tile,
                       kernel_hints={"rows_per_thread": rpy, "threads": 128})
    shape = tuple(s + 2 * h for s, h in zip((13, 35, 66), r.halo_widths))
    u = np.random.default_rng(27 + rpy).standard_normal(shape)
    got = _launch(r, [u])
    want = O.apply_stencil(u, fn._fn, 3, r.halo_widths)
    inner = _interior(shape, r.halo_widths)
    assert np.array_equal(got[inner], want[inner])


@pytest.mark.parametrize("kind", ["dirichlet", "periodic", "reflecting"])
def test_fused_boundary_rows_per_thread(kind):
    import cutile
    from cutile import stencil

    bnd = {"type": kind, "value": -0.25} if kind == "dirichlet" else kind
    r = cutile.compile(stencil(ndim=3, boundary=bnd)(D.lap7), temporal_blocking=False,
                       tile_sizes=(1, 8, 64), kernel_hints={"rows_per_thread": 2, "threads": 128})
    shape = tuple(s + 2 * h for s, h in zip((26, 19, 300), r.halo_widths))
    u = np.random.default_rng(31).random(shape)
    got = _launch(r, [u], step=True)
    want = O.stencil_with_boundary([u], D.lap7, 3, r.halo_widths, kind, -0.25)
    inner = _interior(shape, r.halo_widths)
    assert np.array_equal(got[inner], want[inner])


def test_bricked_rows_per_thread():
    import torch

    import cutile
    from cutile import stencil

    r = cutile.compile(stencil(ndim=3)(D.lap7), temporal_blocking=False, layout="bricked",
                       brick_size=8, tile_sizes=(1, 8, 64),
                       kernel_hints={"rows_per_thread": 2, "threads": 128})
    shape = tuple(s + 2 * h for s, h in zip((12, 21, 40), r.halo_widths))
    u = np.random.default_rng(41).standard_normal(shape)
    mod = r.load_module()
    tin = torch.from_numpy(u).cuda()
    tout = torch.zeros_like(tin)
    mod.launch_lap7_bricked(tin, tout)
    torch.cuda.synchronize()
    want = O.apply_stencil(u, D.lap7, 3, r.halo_widths)
    inner = _interior(shape, r.halo_widths)
    assert np.array_equal(tout.cpu().numpy()[inner], want[inner])
