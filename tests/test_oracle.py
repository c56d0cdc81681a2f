"""The CPU oracle agrees with the reference's own executor (golden fixtures
made by tests/golden/make_golden.py from reference/stencil_ref.py)."""

import numpy as np
import pytest

import random_exprs
import stencil_defs as D
from oracle import stencil_oracle as O


@pytest.mark.parametrize("name", sorted(D.CASES))
def test_single_application_matches_reference(golden, name):
    fn, ndim, nin = D.CASES[name]
    halo = tuple(golden[f"case/{name}/halo"])
    ins = [golden[f"case/{name}/in{k}"] for k in range(nin)]
    got = O.apply_stencil(ins[0], fn, ndim, halo) if nin == 1 else O.apply_multi(ins, fn, ndim, halo)
    assert np.array_equal(got, golden[f"case/{name}/out"])


def test_time_march_heat2d_matches_reference(golden):
    got = O.time_march(golden["march/heat2d/in"], D.heat2d, 2, (1, 1), 25)[-1]
    assert np.array_equal(got, golden["march/heat2d/out"])


def test_time_march_periodic_matches_reference(golden):
    spec = O.uniform_spec("periodic", 1)
    got = O.time_march(golden["march/heat1d_periodic/in"], D.heat1d, 1, (1,), 10, spec)[-1]
    assert np.array_equal(got, golden["march/heat1d_periodic/out"])


@pytest.mark.parametrize("ndim", [1, 2, 3])
@pytest.mark.parametrize("h", [1, 2])
@pytest.mark.parametrize("kind", ["dirichlet", "neumann", "periodic", "reflecting"])
def test_boundary_fill_matches_reference(golden, ndim, h, kind):
    key = f"bc/{ndim}d/h{h}/{kind}"
    a = golden[key + "/in"].copy()
    O.apply_boundary(a, O.uniform_spec(kind, ndim, 0.75), (h,) * ndim)
    assert np.array_equal(a, golden[key + "/out"])


@pytest.mark.parametrize("seed", range(40))
def test_random_expressions_match_reference(golden, golden_exprs, tmp_path, seed):
    e = golden_exprs[str(seed)]
    fn = random_exprs.build(tmp_path, f"r{seed}", e["fields"], e["idx"], e["body"], decorated=False)
    shape = tuple(e["shape"])
    ins = {f: golden[f"rand/{seed}/{f}"] for f in e["used"]}
    got = O.evaluate(ins, fn, len(e["idx"]), tuple(e["halo"]), shape, np.float64)
    got = np.broadcast_to(np.asarray(got, np.float64), golden[f"rand/{seed}/out"].shape)
    assert np.array_equal(got, golden[f"rand/{seed}/out"]), e["body"]


def test_generator_is_reproducible():
    assert random_exprs.case(5) == random_exprs.case(5)


def test_laplacian_known_answer():
    """-6 at a delta (the reference's examples/laplacian_3d.py check)."""
    u = np.zeros((7, 7, 7))
    u[3, 3, 3] = 1.0

    def lap(u, i, j, k):
        return (u[i - 1, j, k] + u[i + 1, j, k] + u[i, j - 1, k] + u[i, j + 1, k]
                + u[i, j, k - 1] + u[i, j, k + 1] - 6.0 * u[i, j, k])

    out = O.apply_stencil(u, lap, 3, (1, 1, 1))
    assert out[3, 3, 3] == -6.0 and out[2, 3, 3] == 1.0


def test_temporal_launch_zero_intermediate_halos():
    rng = np.random.default_rng(1)
    u = rng.random((12, 12))
    out = O.temporal_launch(u, np.full_like(u, 7.0), D.heat2d, 2, (1, 1), 3)
    # halo of the output untouched, interior = 3 steps with zero intermediate halos
    assert np.all(out[0, :] == 7.0)
    step1 = O.apply_stencil(u, D.heat2d, 2, (1, 1))
    z = np.zeros_like(u)
    z[1:-1, 1:-1] = step1[1:-1, 1:-1]
    step2 = O.apply_stencil(z, D.heat2d, 2, (1, 1))
    z2 = np.zeros_like(u)
    z2[1:-1, 1:-1] = step2[1:-1, 1:-1]
    step3 = O.apply_stencil(z2, D.heat2d, 2, (1, 1))
    assert np.array_equal(out[1:-1, 1:-1], step3[1:-1, 1:-1])


def test_bricks_round_trip():
    rng = np.random.default_rng(2)
    a = rng.random((10, 13, 7))
    b = O.to_bricks(a, 4)
    assert b.shape == (3, 4, 2, 4, 4, 4)
    assert np.array_equal(O.from_bricks(b, a.shape, 4), a)


# --------------------------------------------------------------------------- #
# The reference-test corpus: every @stencil of the reference's tests plus its
# random-expression generator's cases, as evaluated by the reference's own
# executor (tests/ref_corpus.py, tests/golden/make_golden.py)
# --------------------------------------------------------------------------- #

import ref_corpus as RC  # noqa: E402

_CORPUS, _CORPUS_OUT = RC.load()


@pytest.mark.parametrize("key", sorted(_CORPUS))
def test_oracle_matches_reference_corpus(tmp_path, key):
    e = _CORPUS[key]
    fn = RC.build(tmp_path, key, e)
    ins = RC.inputs(e)
    dt = np.float32 if e["dtype"] == "float32" else np.float64
    got = O.evaluate(dict(zip(e["args"], ins)), fn, e["ndim"], tuple(e["halo"]), tuple(e["shape"]), dt)
    want = _CORPUS_OUT[key]
    got = np.broadcast_to(np.asarray(got, dt), want.shape)
    assert got.dtype == want.dtype and np.array_equal(got, want), e["origin"]


def test_corpus_covers_the_reference_suites():
    """The fixture holds the application set, the wide boxes, the precedence
    and element-wise math cases and the generator's 47 distinct cases."""
    origins = {e["origin"].split(":")[0] for e in _CORPUS.values()}
    for f in ("tests/test_cutile_gpu_apps.py", "tests/wide_stencils.py", "tests/test_expr_precedence.py",
              "tests/test_frontend_math.py", "tests/test_term_order.py", "tests/test_exact_constants.py",
              "tests/random_stencils.py"):
        assert f in origins
    assert sum(k.startswith("random_stencils/") for k in _CORPUS) == 47
    assert {"wide_stencils/box125", "wide_stencils/box27"} <= set(_CORPUS)
