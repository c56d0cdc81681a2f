"""Generate golden fixtures by running the REFERENCE's own CPU executor.

Run on a machine that has the reference checkout (the fixtures it writes are what
the tests read; the tests never need the reference itself):

    python tests/golden/make_golden.py /path/to/reference

It imports the reference's ``cutile/reference/stencil_ref.py`` and
``elementwise.py`` through a bare package shim (the rest of the reference
needs xDSL, which is not installed), evaluates the stencils of
``tests/stencil_defs.py`` and seeded random expressions (``tests/
random_exprs.py``) with ``apply_stencil`` / ``time_march`` /
``apply_boundary``, and writes inputs + outputs to ``golden.npz`` and the
random expression sources to ``golden_exprs.json`` beside this script.
"""

from __future__ import annotations

import json
import os
import sys
import tempfile
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
TESTS = os.path.dirname(HERE)
sys.path.insert(0, TESTS)


def load_reference(ref_root: str):
    for name, sub in (("cutile", ""), ("cutile.reference", "reference")):
        pkg = types.ModuleType(name)
        pkg.__path__ = [os.path.join(ref_root, "cutile", sub) if sub else os.path.join(ref_root, "cutile")]
        sys.modules[name] = pkg
    from cutile.reference import stencil_ref  # noqa: E402

    return stencil_ref


def main(ref_root: str) -> None:
    ref = load_reference(ref_root)
    import random_exprs
    import stencil_defs as D

    out: dict[str, np.ndarray] = {}
    rng = np.random.default_rng(20261203)

    def arr(shape, kind="rand"):
        if kind == "pos":
            return rng.random(shape) + 0.5
        return rng.standard_normal(shape)

    # 1) one application of every named case
    sizes = {1: (70,), 2: (26, 38), 3: (14, 12, 20)}
    for name, (fn, ndim, nin) in D.CASES.items():
        h = 2 if name in ("lap4_1d", "wave4") else 1
        shape = tuple(s + 2 * h for s in sizes[ndim])
        halo = (h,) * ndim
        ins = [arr(shape, "pos" if name in ("gs_u", "gs_v") else "rand") for _ in range(nin)]
        if nin == 1:
            res = ref.apply_stencil(ins[0], fn, ndim, halo)
        else:
            from cutile.reference.elementwise import array_aware

            proxies = [ref._ArrayProxy(a, halo) for a in ins]
            r = array_aware(fn)(*proxies, *([0] * ndim))
            res = ins[0].copy()
            res[tuple(slice(hh, s - hh) for hh, s in zip(halo, shape))] = r
        for k, a in enumerate(ins):
            out[f"case/{name}/in{k}"] = a
        out[f"case/{name}/halo"] = np.array(halo)
        out[f"case/{name}/out"] = res

    # 2) time marching: heat 2-D with zero Dirichlet halo, 25 steps; 1-D
    #    periodic heat with the boundary re-applied every step
    u0 = np.zeros((34, 34))
    u0[1:-1, 1:-1] = np.random.default_rng(0).random((32, 32))
    hist = ref.time_march(u0, D.heat2d, 2, (1, 1), 25)
    out["march/heat2d/in"] = u0
    out["march/heat2d/out"] = hist[-1]
    u1 = arr((66,))
    spec = {0: ("periodic", "periodic")}
    hist = ref.time_march(u1, D.heat1d, 1, (1,), 10, boundary_spec=spec)
    out["march/heat1d_periodic/in"] = u1
    out["march/heat1d_periodic/out"] = hist[-1]

    # 3) boundary fills: every kind, 1-3 D, halo 1 and 2
    for ndim, shape in ((1, (17,)), (2, (11, 9)), (3, (8, 7, 9))):
        for h in (1, 2):
            full = tuple(s + 2 * h for s in shape)
            for kind in ("dirichlet", "neumann", "periodic", "reflecting"):
                a = arr(full)
                b = a.copy()
                side = (kind, 0.75) if kind == "dirichlet" else kind
                ref.apply_boundary(b, {d: (side, side) for d in range(ndim)}, (h,) * ndim)
                key = f"bc/{ndim}d/h{h}/{kind}"
                out[key + "/in"] = a
                out[key + "/out"] = b

    # 4) random expressions through the reference executor
    exprs = {}
    with tempfile.TemporaryDirectory() as tmp:
        for seed in range(40):
            ndim, nfields, radius, fields, idx, body = random_exprs.case(seed)
            fn = random_exprs.build(tmp, f"r{seed}", fields, idx, body, decorated=False)
            halo = (radius,) * ndim
            shape = tuple(7 + 2 * radius + (seed % 3) for _ in range(ndim))
            used = random_exprs.used_fields(body, fields)
            ins = {f: rng.random(shape) + 0.5 for f in used}
            from cutile.reference.elementwise import array_aware

            args = [ref._ArrayProxy(ins.get(f, np.zeros(shape)), halo) for f in fields]
            res = np.asarray(array_aware(fn)(*args, *([0] * ndim)), dtype=np.float64)
            exprs[str(seed)] = {"fields": fields, "idx": idx, "body": body, "used": used,
                                "halo": list(halo), "shape": list(shape)}
            for f in used:
                out[f"rand/{seed}/{f}"] = ins[f]
            out[f"rand/{seed}/out"] = np.broadcast_to(res, tuple(s - 2 * radius for s in shape)).copy()

    np.savez_compressed(os.path.join(HERE, "golden.npz"), **out)
    with open(os.path.join(HERE, "golden_exprs.json"), "w") as f:
        json.dump(exprs, f, indent=1, sort_keys=True)
    print(f"wrote {len(out)} arrays, {len(exprs)} expressions")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
