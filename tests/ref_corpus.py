"""The reference-test stencil corpus: fixture loading and input generation.

``tests/golden/make_golden.py`` extracts every ``@stencil`` function that the
reference's own test suite defines (its GPU application set, precedence and
element-wise math known-answer tests, term-order and exact-constant cases,
fused members, the 27/125-point boxes of its wide tier) plus the random
expressions its generator ``tests/random_stencils.py`` draws for the seeds its
tests use, evaluates each with the reference's NumPy executor
(``cutile/reference/stencil_ref.py``), and writes

* ``golden/ref_corpus.json``: per entry the standalone module source (the
  decorated function with the constants it captures), ``ndim``, dtype, the
  halo the reference's ``compile()`` gives it, the array shape and how its
  inputs are drawn;
* ``golden/ref_corpus.npz``: the interior of each output.

Inputs are not stored: :func:`inputs` regenerates them from the recorded
recipe (NumPy's legacy ``RandomState`` stream, which NumPy keeps frozen, or
``default_rng(seed).random``), so the fixtures stay small.  Both the
generator and the tests call this module, so they draw the same arrays.
"""

from __future__ import annotations

import importlib.util
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")


def load():
    """Return ``(entries, outputs)``: the JSON entries by key and the npz arrays."""
    with open(os.path.join(GOLDEN, "ref_corpus.json")) as f:
        entries = json.load(f)
    with np.load(os.path.join(GOLDEN, "ref_corpus.npz")) as z:
        outs = {k: z[k] for k in z.files}
    return entries, outs


def inputs(entry) -> list[np.ndarray]:
    """Regenerate an entry's input arrays (one per stencil argument, in order).

    Recipes (each mirrors how the reference's test draws its inputs):

    * ``legacy_randn`` — ``np.random.seed(seed)`` then one ``randn(*shape)`` per
      input (the application set, seed 42);
    * ``legacy_unit`` — as above with ``0.2 + 0.6 * rand`` (its Gray-Scott cases);
    * ``legacy_rand05`` — ``RandomState(seed).rand(*shape) + 0.5`` per used field,
      zeros for fields the body never reads (the random-expression property test);
    * ``rng_pos`` — ``default_rng(seed).random(shape) + 0.5`` per input.
    """
    shape = tuple(entry["shape"])
    n = len(entry["args"])
    kind, seed = entry["inputs"], entry["seed"]
    dt = np.float32 if entry["dtype"] == "float32" else np.float64
    if kind == "legacy_randn":
        np.random.seed(seed)
        arrs = [np.random.randn(*shape).astype(np.float64) for _ in range(n)]
    elif kind == "legacy_unit":
        np.random.seed(seed)
        arrs = [0.2 + 0.6 * np.random.rand(*shape).astype(np.float64) for _ in range(n)]
    elif kind == "legacy_rand05":
        rs = np.random.RandomState(seed)
        used = set(entry["used"])
        drawn = {a: rs.rand(*shape) + 0.5 for a in entry["args"] if a in used}
        arrs = [drawn.get(a, np.zeros(shape)) for a in entry["args"]]
    elif kind == "rng_pos":
        rng = np.random.default_rng(seed)
        arrs = [rng.random(shape) + 0.5 for _ in range(n)]
    else:
        raise ValueError(f"unknown input recipe {kind!r}")
    return [np.ascontiguousarray(a.astype(dt)) for a in arrs]


def interior(shape, halo):
    return tuple(slice(h, s - h) for h, s in zip(halo, shape))


def build(tmpdir, key: str, entry):
    """Write the entry's module source to *tmpdir* and import its stencil.

    The frontend reads a function's source with ``inspect``, so the stencil
    has to live in a real file; the module imports ``stencil``/``where`` from
    whichever ``cutile`` package is first on ``sys.path``.
    """
    name = "refc_" + "".join(c if c.isalnum() else "_" for c in key)
    path = os.path.join(str(tmpdir), name + ".py")
    with open(path, "w") as f:
        f.write(entry["source"])
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return getattr(mod, entry["func"])
