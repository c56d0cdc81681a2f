"""FP64 device reductions (mass, energy, residual, max) against exact sums."""

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _inner(a, halo):
    return a[tuple(slice(h, s - h) for h, s in zip(halo, a.shape))]


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("shape,halo", [((70,), (3,)), ((33, 47), (1, 2)), ((9, 17, 40), (1, 1, 16))])
def test_reductions_match_exact_sums(dtype, shape, halo):
    import torch

    from cutile.runtime import reductions as R

    rng = np.random.default_rng(sum(shape))
    a = rng.standard_normal(shape).astype(dtype)
    b = rng.standard_normal(shape).astype(dtype)
    ta, tb = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
    ia, ib = _inner(a, halo).astype(np.float64), _inner(b, halo).astype(np.float64)
    scale = float(np.abs(ia).sum()) + 1.0
    assert abs(R.mass(ta, halo).item() - math.fsum(ia.ravel())) <= 1e-13 * scale
    sq = math.fsum((ia * ia).ravel())
    assert abs(R.energy(ta, halo).item() - sq) <= 1e-13 * sq
    d2 = math.fsum(((ia - ib) ** 2).ravel())
    assert abs(R.residual(ta, tb, halo).item() - math.sqrt(d2)) <= 1e-13 * math.sqrt(d2)
    assert R.max_abs(ta, halo).item() == float(np.abs(ia).max())
    assert R.max_abs_diff(ta, tb, halo).item() == float(np.abs(ia - ib).max())


def test_reductions_are_deterministic():
    import torch

    from cutile.runtime import reductions as R

    t = torch.randn(130, 257, 64, dtype=torch.float64, device="cuda")
    first = R.mass(t, (1, 1, 1)).item()
    for _ in range(5):
        assert R.mass(t, (1, 1, 1)).item() == first
    # only the interior is read: changing the halo does not change the sum
    t[0].fill_(1e9)
    assert R.mass(t, (1, 1, 1)).item() == first
