"""The autotuner on the GPU: it times fitted candidate plans, caches the
winner per footprint/dtype/size class, and compile(autotune=True, domain=...)
builds the tuned plan, which stays bit-exact against the oracle."""

import numpy as np
import pytest

import stencil_defs as D
from oracle import stencil_oracle as O

pytestmark = pytest.mark.gpu


def test_autotune_picks_a_timed_plan_and_caches_it(tmp_path, monkeypatch):
    from cutile import stencil
    from cutile.runtime import autotune as A

    monkeypatch.setattr(A, "cache_path", lambda: str(tmp_path / "autotune.json"))
    fn = stencil(ndim=3)(D.lap7)
    res = A.autotune(fn, (48, 40, 64), max_candidates=6, iters=3)
    assert res.time_ms > 0 and res.throughput_gpoints > 0
    assert res.candidates == 6 and res.plan is not None
    again = A.autotune(fn, (48, 40, 64), max_candidates=6, iters=3)
    assert again.plan == res.plan and again.time_ms == res.time_ms   # from the cache
    # another size class is tuned separately
    key_small = A.cache_key(A._footprint(fn, 8), "float64", (48, 40, 64), A._gpu_name())
    key_big = A.cache_key(A._footprint(fn, 8), "float64", (256, 256, 256), A._gpu_name())
    assert key_small != key_big


@pytest.mark.parametrize("ndim", [2, 3])
def test_compile_with_autotune_stays_bit_exact(tmp_path, monkeypatch, ndim):
    import torch

    from cutile import compile as stencil_compile
    from cutile import stencil
    from cutile.runtime import autotune as A

    monkeypatch.setattr(A, "cache_path", lambda: str(tmp_path / "autotune.json"))
    fn, dom = (D.heat2d, (70, 90)) if ndim == 2 else (D.lap7, (20, 24, 40))
    r = stencil_compile(stencil(ndim=ndim)(fn), domain=dom, autotune=True)
    h = r.halo_widths
    u = np.zeros(tuple(n + 2 * x for n, x in zip(dom, h)))
    u[tuple(slice(x, -x) for x in h)] = np.random.default_rng(4).random(dom)
    a = torch.from_numpy(u).cuda()
    b = torch.zeros_like(a)
    getattr(r.load_module(), f"launch_{r.name}")(a, b)
    want = O.temporal_launch(u, np.zeros_like(u), fn, ndim, h, r.temporal_steps)
    assert np.array_equal(b.cpu().numpy(), want)
