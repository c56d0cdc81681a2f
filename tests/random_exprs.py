"""Seeded random stencil bodies for property tests.

Each expression mixes linear terms, products of two reads, divisions by a
positive denominator, ``max``/``min``/``abs``, ``where`` on a comparison,
negations and nested sub-sums, with constants that are exact in float32
(0.25), inexact (0.1, 1/3 written as a literal) and integers, over 1-4
fields, 1-3 dimensions and radius 1-4.  ``build`` writes the function to a
file and imports it (the frontend reads source with ``inspect``).
"""

from __future__ import annotations

import importlib.util
import os
import random
import re

FIELDS = ["a", "b", "c", "d"]
INDEX = ["i", "j", "k"]
KINDS = ["lin", "lin", "prod", "div", "max", "min", "abs", "where", "nest", "neg", "sub"]
EXACT = [0.25, 0.5, 2.0, -0.125, 1.0, 4.0, 0.75]
INEXACT = [0.1, 0.3333333333333333, -0.08333333333333333, 0.038095238095238099, 0.7, 1.1]
INTS = [2, 3, -1, 7]

# (ndim, nfields, radius) shapes cycled over by seed
SHAPES = [(1, 1, 1), (1, 2, 3), (2, 1, 2), (2, 2, 1), (2, 3, 3), (3, 1, 1), (3, 2, 2),
          (3, 3, 1), (3, 1, 4), (2, 4, 2)]


def _idx(v, o):
    return v if o == 0 else (f"{v} + {o}" if o > 0 else f"{v} - {-o}")


def generate(seed: int, ndim: int, nfields: int, radius: int, nterms: int):
    rng = random.Random(seed * 7919 + 13)
    fields, idx = FIELDS[:nfields], INDEX[:ndim]

    def coef():
        r = rng.random()
        if r < 0.35:
            return repr(rng.choice(EXACT))
        if r < 0.7:
            return repr(rng.choice(INEXACT))
        if r < 0.85:
            return str(rng.choice(INTS))
        return repr(round(rng.uniform(-2, 2), 5))

    def acc():
        f = rng.choice(fields)
        return f"{f}[{', '.join(_idx(v, rng.randint(-radius, radius)) for v in idx)}]"

    def term(depth=0):
        kind = rng.choice(KINDS)
        if kind == "lin":
            return f"{coef()} * {acc()}"
        if kind == "prod":
            return f"{coef()} * {acc()} * {acc()}"
        if kind == "div":
            return f"{acc()} / ({acc()} + 2.5)"
        if kind == "max":
            return f"{coef()} * max({acc()}, {acc()})"
        if kind == "min":
            return f"min({acc()}, {coef()})"
        if kind == "abs":
            return f"{coef()} * abs({acc()} - {acc()})"
        if kind == "where":
            return f"where({acc()} > {acc()}, {acc()}, {coef()} * {acc()})"
        if kind == "neg":
            return f"-{acc()}"
        if kind == "sub":
            return f"({acc()} - {coef()} * {acc()})"
        if depth < 2:
            return f"{coef()} * ({term(depth + 1)} - ({term(depth + 1)}))"
        return f"{coef()} * {acc()}"

    parts = [term() for _ in range(nterms)]
    body = parts[0] + "".join(f" {rng.choice(['+', '-'])} {p}" for p in parts[1:])
    return fields, idx, body


def used_fields(body, fields):
    return [f for f in fields if re.search(rf"\b{f}\[", body)]


def source(name, fields, idx, body, decorated=True, dtype="float64"):
    head = "from cutile import stencil, where\n\n" if decorated else "\n"
    dec = ""
    if decorated:
        dt = f', dtype="{dtype}"' if dtype != "float64" else ""
        dec = f"@stencil(ndim={len(idx)}{dt})\n"
    return (f"{head}{dec}def {name}({', '.join(fields)}, {', '.join(idx)}):\n"
            f"    return ({body})\n")


def build(directory, name, fields, idx, body, decorated=True, dtype="float64"):
    path = os.path.join(str(directory), f"{name}.py")
    with open(path, "w") as f:
        f.write(source(name, fields, idx, body, decorated, dtype))
    spec = importlib.util.spec_from_file_location(f"rand_stencil_{name}", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return getattr(mod, name)


def case(seed: int, nterms: int | None = None):
    ndim, nfields, radius = SHAPES[seed % len(SHAPES)]
    nterms = nterms or [3, 6, 12][seed % 3]
    fields, idx, body = generate(seed, ndim, nfields, radius, nterms)
    return ndim, nfields, radius, fields, idx, body
