"""Work split of the persistent kernels (csd_plan_items / csd_item_place) on
the host: every interior row of every column is written by exactly one item,
items are never empty, the uniform split is unchanged for kernels without a
fused boundary, and the fused-boundary split gives X-edge columns and each
column's first and last item fewer rows."""

import itertools

import pytest

CSD_BC_NONE, CSD_BC_PERIODIC = 0, 3


def _plan(bc, rows, tx, ty, nz, slots, zchunk=0, desc_zchunk=0):
    from cutile.runtime import native

    d = {"rows": rows, "zchunk": desc_zchunk, "bc_mode": bc}
    return native.plan_items(d, tx, ty, nz, slots, zchunk)


def _coverage(items, tx, ty, nz):
    cover = {}
    for (x, y, z0, n) in items:
        assert 0 <= x < tx and 0 <= y < ty
        assert n > 0 and z0 >= 0 and z0 + n <= nz
        cover.setdefault((x, y), []).append((z0, n))
    assert set(cover) == {(x, y) for x in range(tx) for y in range(ty)}
    for spans in cover.values():
        spans.sort()
        z = 0
        for z0, n in spans:
            assert z0 == z
            z += n
        assert z == nz
    return cover


CASES = list(itertools.product(
    (CSD_BC_NONE, CSD_BC_PERIODIC), (1, 2, 8), (1, 2, 3, 5, 32), (1, 3), (1, 7, 40, 300, 4096),
    (148, 296, 444)))


def test_every_row_written_once():
    for bc, rows, tx, ty, nz, slots in CASES:
        split, items = _plan(bc, rows, tx, ty, nz, slots)
        assert len(items) == split["items"], (bc, rows, tx, ty, nz, slots)
        _coverage(items, tx, ty, nz)


@pytest.mark.parametrize("zchunk,desc_zchunk", [(24, 0), (0, -4), (0, 16)])
def test_explicit_or_multiwave_split_stays_uniform(zchunk, desc_zchunk):
    split, items = _plan(CSD_BC_PERIODIC, 8, 32, 1, 4096, 296, zchunk, desc_zchunk)
    assert split["ecols"] == 0 and split["zshift"] == 0
    _coverage(items, 32, 1, 4096)
    lens = {n for (_, _, z0, n) in items if z0 + n < 4096}
    assert len(lens) == 1


def test_no_boundary_split_is_the_uniform_one():
    split, items = _plan(CSD_BC_NONE, 8, 32, 1, 4096, 296)
    assert split == {"items": 288, "zchunk": 456, "ecols": 0, "items_main": 0, "zchunk_e": 456,
                     "zshift": 0, "zshift_e": 0, "tiles_z": 9}
    assert items[0] == (0, 0, 0, 456) and items[33] == (1, 0, 456, 456)


def test_boundary_split_shortens_edge_items_within_one_wave():
    # Gray-Scott 4096^2 FP32+Kahan: 32 columns of 128, two CTAs per SM
    split, items = _plan(CSD_BC_PERIODIC, 8, 32, 1, 4096, 296)
    assert split["ecols"] == 2 and split["items"] <= 296
    cover = _coverage(items, 32, 1, 4096)
    mid = max(n for spans in cover.values() for _, n in spans)
    edge = max(n for x in (0, 31) for _, n in cover[(x, 0)])
    assert edge <= 0.8 * mid
    inner = sorted(cover[(5, 0)])
    assert inner[0][1] < inner[1][1] and inner[-1][1] < inner[1][1]


def test_single_wave_kept_when_it_fills_the_slots():
    """512 columns on 1184 resident slots (the flat 7-point sweep at 512^3):
    two items per column, one wave, 86 % of the slots busy."""
    split, items = _plan(CSD_BC_NONE, 1, 4, 128, 512, 1184)
    assert split["items"] == 1024 <= 1184


@pytest.mark.parametrize("tx,ty,slots", [(5, 129, 1184), (4, 128, 444), (3, 80, 444)])
def test_poorly_filled_single_wave_becomes_about_seven_waves(tx, ty, slots):
    """Columns that would leave more than a fifth of the slots idle (the
    bricked sweep's 645 columns on 1184 slots; 512 columns on 444 slots,
    which spill into a thin second wave) are cut into shorter items, about
    seven waves, every row still written once."""
    split, items = _plan(CSD_BC_NONE, 1, tx, ty, 512, slots)
    waves = split["items"] / slots
    assert 5.5 <= waves <= 8.5, waves
    _coverage(items, tx, ty, 512)


def test_chains_default_to_eight_waves():
    from cutile.passes.tiling import EnginePlan, fit_plan

    p = fit_plan(EnginePlan(3, rows=1, tile_y=8, tile_x=64, vec=2, threads=128, stages=1,
                            zchunk=0, temporal=2), (1, 1, 1), 8, 1)
    assert p.waves == 8
    p1 = fit_plan(EnginePlan(3, rows=1, tile_y=4, tile_x=128, vec=2, threads=128, stages=1,
                             zchunk=0), (1, 1, 1), 8, 1)
    assert p1.waves == 1
