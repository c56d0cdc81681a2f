"""Generate golden fixtures by running the REFERENCE's own CPU executor.

Run on a machine that has the reference checkout (the fixtures it writes are what
the tests read; the tests never need the reference itself):

    python tests/golden/make_golden.py /path/to/reference

The reference checkout's path is a required argument.

It imports the reference's ``cutile/reference/stencil_ref.py`` and
``elementwise.py`` through a bare package shim (the rest of the reference
needs xDSL, which is not installed), evaluates the stencils of
``tests/stencil_defs.py`` and seeded random expressions (``tests/
random_exprs.py``) with ``apply_stencil`` / ``time_march`` /
``apply_boundary``, and writes inputs + outputs to ``golden.npz`` and the
random expression sources to ``golden_exprs.json`` beside this script.

It also writes the reference-test corpus (``ref_corpus.json`` +
``ref_corpus.npz``, read through ``tests/ref_corpus.py``): every ``@stencil``
function defined anywhere in the reference's ``tests/`` directory, found by
walking each file's syntax tree, written out as a standalone module with the
numeric constants it captures from enclosing scopes, and the random
expressions of the reference's own generator (``tests/random_stencils.py``)
for the seeds and shapes of its property tests
(``tests/test_random_expressions.py:21,62-75,99-106``).  Each is evaluated
by the reference's ``_ArrayProxy`` + ``array_aware`` executor on inputs drawn
the way the reference's test draws them, with the halo the reference's
``compile()`` gives the stencil (footprint per dimension, innermost rounded up
to 128 bytes: launcher.py:257-273, 488-491).
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


# ---------------------------------------------------------------------------
# reference-test corpus
# ---------------------------------------------------------------------------

import ast  # noqa: E402

DEFAULT_DOMAIN = {1: (200,), 2: (24, 40), 3: (10, 12, 20)}


def _is_stencil_decorator(d) -> bool:
    if isinstance(d, ast.Name):
        return d.id == "stencil"
    return isinstance(d, ast.Call) and isinstance(d.func, ast.Name) and d.func.id == "stencil"


def _raises_match(node):
    """The ``match=`` text of a ``with pytest.raises(...)`` statement, else None."""
    if not isinstance(node, ast.With):
        return None
    for item in node.items:
        c = item.context_expr
        if isinstance(c, ast.Call) and getattr(c.func, "attr", "") == "raises":
            for k in c.keywords:
                if k.arg == "match":
                    return ast.literal_eval(k.value)
            return ""
    return None


def _walk_defs(tree):
    """Yield ``(funcdef, enclosing scopes, expected error)`` for every
    stencil-decorated def; the expected error is the ``match=`` text when the
    def sits inside ``with pytest.raises(...)`` (a case the frontend must
    reject), else None."""

    def rec(node, scopes, raises):
        for child in ast.iter_child_nodes(node):
            r = _raises_match(child)
            inner = raises if r is None else r
            if isinstance(child, ast.FunctionDef) and any(map(_is_stencil_decorator, child.decorator_list)):
                yield child, scopes, raises
            if isinstance(child, (ast.FunctionDef, ast.ClassDef)):
                yield from rec(child, scopes + [child], inner)
            elif not isinstance(child, ast.FunctionDef):
                yield from rec(child, scopes, inner)

    yield from rec(tree, [tree], None)


def _captured_constants(fdef, scopes):
    """Numeric constants the stencil body reads from its enclosing scopes.

    Every simple ``NAME = <expr>`` assignment of an enclosing module or
    function that precedes the def is evaluated in order (arithmetic on
    literals and earlier names only); the ones the body names are kept.
    """
    names_used = {n.id for n in ast.walk(fdef) if isinstance(n, ast.Name) and isinstance(n.ctx, ast.Load)}
    env: dict[str, float] = {}
    for scope in scopes:
        body = scope.body if hasattr(scope, "body") else []
        for st in body:
            if st.lineno >= fdef.lineno and scope is scopes[-1]:
                break
            if not (isinstance(st, ast.Assign) and len(st.targets) == 1):
                continue
            tgt = st.targets[0]
            names = ([tgt.id] if isinstance(tgt, ast.Name) else
                     [e.id for e in tgt.elts] if isinstance(tgt, ast.Tuple)
                     and all(isinstance(e, ast.Name) for e in tgt.elts) else None)
            if names is None:
                continue
            try:
                val = eval(compile(ast.Expression(st.value), "<c>", "eval"), {"__builtins__": {}}, dict(env))
            except Exception:
                continue
            vals = [val] if isinstance(tgt, ast.Name) else list(val) if isinstance(val, tuple) else []
            for n, v in zip(names, vals):
                if isinstance(v, (int, float)) and not isinstance(v, bool):
                    env[n] = v
    return {k: v for k, v in env.items() if k in names_used}


def _module_source(src_text, fdef, consts) -> str:
    seg = ast.get_source_segment(src_text, fdef, padded=True) or ""
    # decorators are not part of the def's segment: take the lines from the
    # first decorator, dedented
    lines = src_text.splitlines()
    first = min(d.lineno for d in fdef.decorator_list)
    block = lines[first - 1:fdef.end_lineno]
    indent = min(len(l) - len(l.lstrip()) for l in block if l.strip())
    body = "\n".join(l[indent:] for l in block)
    del seg
    head = "from cutile import stencil, where\n\n"
    cl = "".join(f"{k} = {v!r}\n" for k, v in consts.items())
    return head + cl + ("\n" if cl else "") + body + "\n"


def _domain_from_call(fdef, scopes):
    """``self._validate*(fn, (n0, n1, ...))`` in the enclosing function."""
    encl = scopes[-1]
    for node in ast.walk(encl):
        if (isinstance(node, ast.Call) and len(node.args) >= 2 and isinstance(node.args[0], ast.Name)
                and node.args[0].id == fdef.name and isinstance(node.args[1], ast.Tuple)):
            try:
                return tuple(ast.literal_eval(node.args[1])), getattr(node.func, "attr", "")
            except ValueError:
                return None, ""
    return None, ""


class _Recorder:
    def __init__(self, ref, arr, halo, log):
        self._p = ref._ArrayProxy(arr, halo)
        self._log = log

    def __getitem__(self, key):
        k = key if isinstance(key, tuple) else (key,)
        self._log.append(tuple(int(o) for o in k))
        return self._p[key]


def _params(fdef):
    params = [a.arg for a in fdef.args.args]
    subscripted, index_names = [], set()
    for n in ast.walk(fdef):
        if isinstance(n, ast.Subscript) and isinstance(n.value, ast.Name) and n.value.id in params:
            if n.value.id not in subscripted:
                subscripted.append(n.value.id)
            for m in ast.walk(n.slice):
                if isinstance(m, ast.Name) and m.id in params:
                    index_names.add(m.id)
    arrays = [p for p in params if p not in index_names]
    order = [p for p in params if p in subscripted]
    return arrays, order, [p for p in params if p in index_names]


def _decorator_kwargs(fdef):
    for d in fdef.decorator_list:
        if isinstance(d, ast.Call):
            return {k.arg: ast.literal_eval(k.value) for k in d.keywords if k.arg in ("ndim", "order", "dtype")}
    return {}


def _pad_inner(halo, dtype_bytes):
    align = max(1, 128 // dtype_bytes)
    return tuple(halo[:-1]) + (-(-halo[-1] // align) * align,)


def _evaluate(ref, fn, arrays, halo, ndim, dtype):
    from cutile.reference.elementwise import array_aware

    proxies = [ref._ArrayProxy(a, halo) for a in arrays]
    res = array_aware(fn)(*proxies, *([0] * ndim))
    interior = tuple(s - 2 * h for s, h in zip(arrays[0].shape, halo))
    return np.broadcast_to(np.asarray(res, dtype=dtype), interior).copy()


def _corpus_entry(ref, rc, key, origin, source, func, ndim, dtype, args, used, domain, recipe, seed):
    """Load the module, find its footprint, draw inputs, evaluate."""
    import importlib.util

    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "m.py")
        with open(path, "w") as f:
            f.write(source)
        spec = importlib.util.spec_from_file_location("refcorpus_mod", path)
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        fn = getattr(mod, func)
        fn = getattr(fn, "_fn", fn)
        # footprint: run once on zeros with a wide halo and record offsets
        log: list = []
        probe = [_Recorder(ref, np.zeros((20,) * ndim), (8,) * ndim, log) for _ in args]
        from cutile.reference.elementwise import array_aware

        array_aware(fn)(*probe, *([0] * ndim))
        foot = tuple(max(abs(o[d]) for o in log) for d in range(ndim))
        nbytes = 4 if dtype == "float32" else 8
        halo = _pad_inner(foot, nbytes)
        shape = tuple(n + 2 * h for n, h in zip(domain, halo))
        entry = {"origin": origin, "source": source, "func": func, "ndim": ndim, "dtype": dtype,
                 "args": args, "used": used, "footprint": list(foot), "halo": list(halo),
                 "shape": list(shape), "inputs": recipe, "seed": seed}
        ins = rc.inputs(entry)
        out = _evaluate(ref, fn, ins, halo, ndim, np.float32 if dtype == "float32" else np.float64)
        return entry, out


def build_corpus(ref, ref_root: str):
    import ref_corpus as rc

    sys.modules["cutile"].stencil = _fake_stencil
    from cutile.reference import elementwise

    sys.modules["cutile"].where = elementwise.where
    entries, outs, skipped, rejects = {}, {}, {}, {}
    tdir = os.path.join(ref_root, "tests")
    for fname in sorted(os.listdir(tdir)):
        if not fname.endswith(".py"):
            continue
        text = open(os.path.join(tdir, fname)).read()
        tree = ast.parse(text)
        for fdef, scopes, expect_error in _walk_defs(tree):
            chain = [getattr(s, "name", "") for s in scopes[1:]]
            key = "/".join([fname[:-3]] + chain + [fdef.name])
            if key in entries or key in rejects:
                key += f"@{fdef.lineno}"
            origin = f"tests/{fname}:{fdef.lineno}"
            args, used, idx = _params(fdef)
            kw = _decorator_kwargs(fdef)
            consts = _captured_constants(fdef, scopes)
            source = _module_source(text, fdef, consts)
            if expect_error is not None:
                rejects[key] = {"origin": origin, "source": source, "func": fdef.name, "match": expect_error}
                continue
            try:
                ndim = kw.get("ndim") or len(idx)
                dtype = kw.get("dtype", "float64")
                dom, via = _domain_from_call(fdef, scopes)
                if fname == "test_cutile_gpu_apps.py" and dom is not None:
                    recipe = "legacy_unit" if "gray_scott" in chain[-1] else "legacy_randn"
                    seed = 42
                else:
                    dom = dom or DEFAULT_DOMAIN[ndim]
                    recipe, seed = "rng_pos", 1000 + fdef.lineno
                e, o = _corpus_entry(ref, rc, key, origin, source, fdef.name, ndim, dtype,
                                     args, used, dom, recipe, seed)
            except Exception as exc:  # the reference itself cannot evaluate it
                skipped[key] = f"{origin}: {type(exc).__name__}: {exc}"
                continue
            entries[key], outs[key] = e, o

    # the reference generator's random expressions, as its property tests draw them
    sys.path.insert(0, tdir)
    import random_stencils as RS

    shapes = ast.literal_eval(
        next(l for l in open(os.path.join(tdir, "test_random_expressions.py")) if l.startswith("_SHAPES"))
        .split("=", 1)[1].strip())
    cases = [(s, [3, 6, 12][s % 3]) for s in range(40)] + [(s, 12) for s in (2, 3, 10, 30, 41, 57, 73, 99)]
    with tempfile.TemporaryDirectory() as tmp:
        for seed, nterms in cases:
            ndim, nfields, radius = shapes[seed % len(shapes)]
            fields, idx, body = RS.generate(seed, ndim, nfields, radius, nterms)
            _, src = RS.make_stencil(tmp, f"r{seed}_{nterms}", fields, idx, body)
            key = f"random_stencils/seed{seed}_terms{nterms}"
            dom = tuple(12 for _ in range(ndim))
            e, o = _corpus_entry(ref, rc, key, "tests/random_stencils.py:25 (seed %d, %d terms)" % (seed, nterms),
                                 src, f"r{seed}_{nterms}", ndim, "float64", fields,
                                 RS.used_fields(body, fields), dom, "legacy_rand05", seed)
            entries[key], outs[key] = e, o
    return entries, outs, skipped, rejects


def _fake_stencil(fn=None, **kw):
    """Stand-in for the reference's decorator (which needs xDSL): returns the
    plain function, which is all the NumPy executor runs."""
    if fn is not None:
        return fn
    return lambda f: f


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

    entries, outs, skipped, rejects = build_corpus(ref, ref_root)
    np.savez_compressed(os.path.join(HERE, "ref_corpus.npz"), **outs)
    with open(os.path.join(HERE, "ref_corpus.json"), "w") as f:
        json.dump(entries, f, indent=1, sort_keys=True)
    with open(os.path.join(HERE, "ref_rejects.json"), "w") as f:
        json.dump(rejects, f, indent=1, sort_keys=True)
    print(f"corpus: {len(entries)} stencils, {len(skipped)} the reference executor cannot run:")
    for k, why in sorted(skipped.items()):
        print("  ", k, "--", why)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <path to the reference checkout>")
    main(sys.argv[1])
