"""GPU parity on the reference's own stencils and inputs, bit for bit.

Every ``@stencil`` defined in the reference's test suite (its GPU application
set with seed-42 inputs, precedence and element-wise math known answers,
term-order and exact-constant cases, fused members, the 27- and 125-point
boxes) and the random expressions of its generator for the seeds its property
tests use, compiled by ``cutile.compile`` and run through libcsd; the output
interior must equal what the reference's NumPy executor computed
(``tests/golden/ref_corpus.npz``), and the halo must stay untouched.
"""

import numpy as np
import pytest

import ref_corpus as RC

pytestmark = pytest.mark.gpu

_CORPUS, _OUT = RC.load()


@pytest.mark.parametrize("key", sorted(_CORPUS))
def test_reference_corpus_bit_exact(tmp_path, key):
    import torch

    import cutile
    from cutile.runtime import native

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    e = _CORPUS[key]
    fn = RC.build(tmp_path, key, e)
    r = cutile.compile(fn, temporal_blocking=False)
    assert list(r.halo_widths) == e["halo"], "halo differs from the reference compile()'s"
    assert list(r.inputs) == e["used"]
    by_name = dict(zip(e["args"], RC.inputs(e)))
    ins = [torch.from_numpy(by_name[n]).cuda() for n in r.inputs]
    out = torch.full_like(ins[0], float("nan"))
    getattr(r.load_module(), f"launch_{r.name}")(*ins, out)
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    inner = RC.interior(got.shape, e["halo"])
    assert np.array_equal(got[inner], _OUT[key]), e["origin"]
    mask = np.ones(got.shape, bool)
    mask[inner] = False
    assert np.all(np.isnan(got[mask])), "kernel wrote outside the interior"
    assert native.error_word(reset=True) == 0


FUSED_GROUPS = {
    "pair": ("test_fused/_pair/a", "test_fused/_pair/b"),
    "unused_parameter": ("test_fused/TestFusedGPU/test_member_with_an_unused_parameter_validates/p",
                         "test_fused/TestFusedGPU/test_member_with_an_unused_parameter_validates/q"),
    "three_field_products": ("test_fused/TestFusedGPU/test_three_field_products_match_the_reference/flux",
                             "test_fused/TestFusedGPU/test_three_field_products_match_the_reference/div"),
    "box27_with_lap": ("wide_stencils/box27",
                       "test_fused/TestCompileFused/test_tile_tier_and_probe_use_the_merged_kernel/lap"),
}


@pytest.mark.parametrize("group", sorted(FUSED_GROUPS))
def test_reference_fused_groups_bit_exact(tmp_path, group):
    """The reference's compile_fused member sets (tests/test_fused.py): one
    fused kernel, inputs merged by parameter name, every output equal to its
    member applied alone by the oracle."""
    import torch

    import cutile
    from cutile.runtime import native
    from oracle import stencil_oracle as O

    keys = FUSED_GROUPS[group]
    fns = [RC.build(tmp_path, k, _CORPUS[k]) for k in keys]
    r = cutile.compile_fused(fns)
    ndim = _CORPUS[keys[0]]["ndim"]
    sizes = {1: (200,), 2: (24, 40), 3: (10, 12, 20)}[ndim]
    shape = tuple(n + 2 * h for n, h in zip(sizes, r.halo_widths))
    rng = np.random.default_rng(len(group))
    arrays = {name: rng.random(shape) + 0.5 for name in r.inputs}
    ins = [torch.from_numpy(arrays[n]).cuda() for n in r.inputs]
    outs = [torch.full_like(ins[0], float("nan")) for _ in fns]
    getattr(r.load_module(), f"launch_{r.name}")(*ins, *outs)
    torch.cuda.synchronize()
    inner = RC.interior(shape, r.halo_widths)
    for fn, out in zip(fns, outs):
        want = O.evaluate(arrays, fn, ndim, r.halo_widths, shape, np.float64)
        got = out.cpu().numpy()[inner]
        assert np.array_equal(got, np.broadcast_to(want, got.shape)), (group, fn._fn.__name__)
    assert native.error_word(reset=True) == 0
