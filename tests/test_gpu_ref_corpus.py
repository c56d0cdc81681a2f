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
