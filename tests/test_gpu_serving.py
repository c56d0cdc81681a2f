"""Serving on the GPU: every solve's result in the continuous-batching mix is
bit-identical to the same solve run alone through the drop-in launch, and to
the NumPy oracle for sampled requests; admission keeps to the budget."""

import numpy as np
import pytest

import stencil_defs as D
from oracle import stencil_oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def kinds():
    return D.serving_kinds()


def _requests(seed=11, n=20):
    from cutile.runtime.serving import SolveRequest

    rng = np.random.default_rng(seed)
    names = list(D.SERVE_KINDS)
    reqs = []
    t = 0.0
    for i in range(n):
        kind = names[i % len(names)]
        if kind == "lap7":
            m = int(rng.integers(12, 40))
            shape = (m + 2, m + 2, m + 2)
        else:
            m = int(rng.integers(20, 150))
            shape = (m + 2, int(rng.integers(20, 150)) + 2)
        t += float(rng.exponential(0.0005))
        reqs.append(SolveRequest(kind, ("float32", "float64")[int(rng.integers(0, 2))], shape,
                                 int(rng.integers(3, 40)), arrival=t, seed=1000 + i))
    return reqs


def test_mix_equals_alone_bit_exact_under_a_tight_budget(kinds):
    import torch

    from cutile.runtime.serving import StencilServer

    reqs = _requests()
    probe = StencilServer(kinds)
    budget = 3 * max(probe.memory_of(r) for r in reqs)
    server = StencilServer(kinds, budget_bytes=budget)
    res = server.run(reqs, realtime=False)
    torch.cuda.synchronize()
    assert server.stats.peak_bytes <= budget
    assert server.stats.max_active >= 2
    for r, out in zip(reqs, res):
        alone, _ = server.run_alone(r)
        for a, b in zip(out.state, alone):
            assert torch.equal(a, b), (r.rid, r.kind, r.dtype, r.shape)


def test_mix_matches_the_oracle(kinds):
    import torch

    from cutile.runtime.serving import SolveRequest, StencilServer

    rng = np.random.default_rng(5)
    cases = [("heat2d", (42, 37)), ("upwind2d", (30, 55)), ("wave2d", (33, 33)),
             ("lap7", (14, 18, 20))]
    reqs = []
    for i, (kind, shape) in enumerate(cases):
        fn, ndim, nstate = D.SERVE_KINDS[kind]
        u = np.zeros(shape)
        u[tuple(slice(1, s - 1) for s in shape)] = rng.random(tuple(s - 2 for s in shape))
        init = (u,) * nstate
        reqs.append(SolveRequest(kind, "float64", shape, 7 + i, arrival=0.0, init=init))
    server = StencilServer(kinds)
    res = server.run(reqs, realtime=False)
    torch.cuda.synchronize()
    for r, out in zip(reqs, res):
        fn, ndim, nstate = D.SERVE_KINDS[r.kind]
        halo = (1,) * ndim
        state = [a.copy() for a in r.init]
        for _ in range(r.steps):
            new = np.zeros_like(state[0])
            inner = tuple(slice(1, s - 1) for s in r.shape)
            names = ["u", "up"][:nstate]
            new[inner] = O.evaluate(dict(zip(names, state)), fn, ndim, halo, state[0].shape,
                                    state[0].dtype)
            state = [new] + state[:-1]
        got = out.state[0].cpu().numpy()
        assert np.array_equal(got, state[0]), r.kind
