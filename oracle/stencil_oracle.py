"""CPU oracle for the stencil path -- TEST INFRASTRUCTURE, NOT THE PRODUCT.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import this module, and only to check or time the reference's CPU
algorithm.  The product path (``cutile`` / libcsd) never calls it.

A NumPy restatement of the reference's executor and launcher semantics:

* ``apply_stencil``  -- reference/stencil_ref.py:52-87 (``_ArrayProxy``
  shifted interior views, builtins max/min swapped for array versions as in
  reference/elementwise.py:40-52; a copy of ``u`` with only the interior
  replaced);
* ``apply_boundary`` -- reference/stencil_ref.py:102-201 (per dimension,
  low side then high side, Dirichlet / Neumann / periodic / reflecting);
* ``time_march``     -- reference/stencil_ref.py:208-245;
* ``temporal_launch`` -- what one call of the reference's generated
  ``launch_<name>`` with ``temporal_steps = T`` computes
  (stencil_to_target.py:740-843, target_to_python.py:329-399): T kernel
  applications through scratch buffers whose halos are zero, only the
  output's interior written;
* ``fused_apply``    -- one ``launch_<a_b>`` of ``compile_fused``
  (stencil_to_target.py:968-1049): each member on the merged inputs, by name;
* ``bricked_launch`` -- ``launch_<name>_bricked`` (multigpu_emitter.py:426-473):
  the flat result with zero halo written over the whole output.

Pinned against the reference itself: ``tests/golden/make_golden.py`` runs the
reference's own ``stencil_ref`` functions in the build container and stores
their outputs; ``tests/test_oracle.py`` checks this module against them.
"""

from __future__ import annotations

import builtins
import math
import types

import numpy as np


# --------------------------------------------------------------------------- #
# Array-aware helpers (reference/elementwise.py:17-52)
# --------------------------------------------------------------------------- #


def _xp(*args):
    for a in args:
        if type(a).__module__.split(".")[0] == "numpy":
            return np
    return None


def maximum(a, b):
    return builtins.max(a, b) if _xp(a, b) is None else np.maximum(a, b)


def minimum(a, b):
    return builtins.min(a, b) if _xp(a, b) is None else np.minimum(a, b)


def where(cond, a, b):
    return (a if cond else b) if _xp(cond, a, b) is None else np.where(cond, a, b)


def sqrt(x):
    return math.sqrt(x) if _xp(x) is None else np.sqrt(x)


def array_aware(fn):
    g = dict(fn.__globals__)
    b = dict(vars(builtins))
    b["max"] = maximum
    b["min"] = minimum
    g["__builtins__"] = b
    g.setdefault("where", where)
    g.setdefault("sqrt", sqrt)
    return types.FunctionType(fn.__code__, g, fn.__name__, fn.__defaults__, fn.__closure__)


def raw_fn(fn):
    """The plain Python function behind a ``@stencil`` wrapper."""
    return getattr(fn, "_fn", fn)


# --------------------------------------------------------------------------- #
# Executor
# --------------------------------------------------------------------------- #


class ArrayProxy:
    """``proxy[k]`` -> ``u[h+k : n-h+k]`` per dim (stencil_ref.py:21-45)."""

    def __init__(self, data: np.ndarray, halo):
        self._data = data
        self._halo = tuple(halo)

    def __getitem__(self, key):
        if not isinstance(key, tuple):
            key = (key,)
        sl = []
        for dim, off in enumerate(key):
            h = self._halo[dim]
            n = self._data.shape[dim]
            sl.append(slice(h + off, n - h + off))
        return self._data[tuple(sl)]


def _interior(shape, halo):
    return tuple(slice(h, s - h) for h, s in zip(halo, shape))


def apply_stencil(u: np.ndarray, fn, ndim: int, halo_widths) -> np.ndarray:
    """One application; returns a copy of ``u`` with the interior updated."""
    res = array_aware(raw_fn(fn))(ArrayProxy(u, halo_widths), *([0] * ndim))
    out = u.copy()
    out[_interior(u.shape, halo_widths)] = res
    return out


def apply_multi(arrays, fn, ndim: int, halo_widths) -> np.ndarray:
    """Multi-input application (the reference tests' ``_apply_multi_input``):
    positional arrays for the stencil's array parameters; a copy of the first
    array with the interior replaced."""
    res = array_aware(raw_fn(fn))(*[ArrayProxy(a, halo_widths) for a in arrays], *([0] * ndim))
    out = arrays[0].copy()
    out[_interior(arrays[0].shape, halo_widths)] = res
    return out


def evaluate(arrays_by_param: dict, fn, ndim: int, halo_widths, shape, dtype):
    """Interior values of ``fn`` with its array parameters bound by name;
    parameters that are not given read zeros (launcher.py:134-169)."""
    import inspect

    f = raw_fn(fn)
    params = list(inspect.signature(f).parameters)[:-ndim]
    args = [ArrayProxy(arrays_by_param.get(p, np.zeros(shape, dtype)), halo_widths) for p in params]
    return array_aware(f)(*args, *([0] * ndim))


# --------------------------------------------------------------------------- #
# Boundary conditions (stencil_ref.py:102-201)
# --------------------------------------------------------------------------- #


def _parse_bc(spec):
    if isinstance(spec, str):
        return spec, 0.0
    if isinstance(spec, tuple):
        return spec[0], spec[1]
    raise TypeError(f"Unsupported boundary spec: {spec!r}")


def _apply_bc_side(u, ndim, dim, h, n, kind, value, side):
    if kind == "dirichlet":
        sl = [slice(None)] * ndim
        sl[dim] = slice(0, h) if side == "low" else slice(n - h, n)
        u[tuple(sl)] = value
        return
    for k in range(h):
        src = [slice(None)] * ndim
        dst = [slice(None)] * ndim
        if kind == "neumann":
            src[dim], dst[dim] = (h, h - 1 - k) if side == "low" else (n - h - 1, n - h + k)
        elif kind == "periodic":
            src[dim], dst[dim] = (n - 2 * h + k, k) if side == "low" else (h + k, n - h + k)
        elif kind == "reflecting":
            src[dim], dst[dim] = (2 * h - 1 - k, k) if side == "low" else (n - h - 1 - k, n - h + k)
        else:
            raise ValueError(f"unknown boundary kind {kind!r}")
        u[tuple(dst)] = u[tuple(src)]


def apply_boundary(u: np.ndarray, boundary_spec: dict, halo_widths) -> None:
    """In place; ``boundary_spec`` maps dim -> (low, high) kinds."""
    ndim = u.ndim
    for dim in range(ndim):
        if dim not in boundary_spec:
            continue
        low, high = boundary_spec[dim]
        h = halo_widths[dim]
        n = u.shape[dim]
        lk, lv = _parse_bc(low)
        hk, hv = _parse_bc(high)
        _apply_bc_side(u, ndim, dim, h, n, lk, lv, "low")
        _apply_bc_side(u, ndim, dim, h, n, hk, hv, "high")


def uniform_spec(kind: str, ndim: int, value: float = 0.0) -> dict:
    side = (kind, value) if kind == "dirichlet" else kind
    return {d: (side, side) for d in range(ndim)}


def time_march(u0, fn, ndim, halo_widths, steps, boundary_spec=None):
    """Snapshots ``[u0, u1, ..., u_steps]`` (stencil_ref.py:208-245)."""
    history = [u0.copy()]
    u = u0.copy()
    for _ in range(steps):
        u = apply_stencil(u, fn, ndim, halo_widths)
        if boundary_spec is not None:
            apply_boundary(u, boundary_spec, halo_widths)
        history.append(u.copy())
    return history


# --------------------------------------------------------------------------- #
# Launcher semantics
# --------------------------------------------------------------------------- #


def temporal_launch(u_in: np.ndarray, u_out: np.ndarray, fn, ndim: int, halo_widths,
                    steps: int) -> np.ndarray:
    """Result of one ``launch_<name>(u_in, u_out)`` with ``temporal_steps = steps``:
    a new array equal to ``u_out`` with its interior set to the ``steps``-th
    iterate, intermediate iterates having zero halos."""
    f = array_aware(raw_fn(fn))
    inner = _interior(u_in.shape, halo_widths)
    cur = u_in
    for s in range(steps):
        res = f(ArrayProxy(cur, halo_widths), *([0] * ndim))
        nxt = u_out.copy() if s == steps - 1 else np.zeros_like(u_in)
        nxt[inner] = res
        cur = nxt
    return cur


def kahan_temporal_launch(u_in, c_in, incr_fn, ndim: int, halo_widths, steps: int,
                          u_out=None, c_out=None):
    """One launch of a Kahan-compensated stencil with ``temporal_steps = steps``:
    ``steps`` compensated updates (``kahan_update``) chained the way
    ``temporal_launch`` chains a single field -- intermediate iterates of u and
    of its compensation have zero halos -- with only the outputs' interiors
    written.  Returns ``(u, c)``."""
    inner = _interior(u_in.shape, halo_widths)
    cu, cc = u_in, c_in
    for s in range(steps):
        inc = evaluate_ops({"u": cu}, incr_fn, ndim, halo_widths, u_in.shape, u_in.dtype)[0]
        nu, nc = kahan_update(cu[inner], cc[inner], inc)
        last = s == steps - 1
        a = (u_out.copy() if u_out is not None else np.zeros_like(u_in)) if last else np.zeros_like(u_in)
        b = (c_out.copy() if c_out is not None else np.zeros_like(c_in)) if last else np.zeros_like(c_in)
        a[inner], b[inner] = nu, nc
        cu, cc = a, b
    return cu, cc


def fused_apply(inputs_by_name: dict, fns, ndim: int, halo_widths, outs=None):
    """Outputs of one fused launch: each member evaluated on the named inputs,
    written into a copy of the corresponding output (zeros if not given)."""
    first = next(iter(inputs_by_name.values()))
    results = []
    for k, fn in enumerate(fns):
        base = np.zeros_like(first) if outs is None else outs[k].copy()
        base[_interior(first.shape, halo_widths)] = evaluate(
            inputs_by_name, fn, ndim, halo_widths, first.shape, first.dtype)
        results.append(base)
    return results


def stencil_with_boundary(inputs, fn, ndim: int, halo_widths, kind: str, value: float = 0.0):
    """``out = stencil(apply_boundary(in))`` for every input (what a fused
    boundary step computes); the inputs themselves are not modified."""
    spec = uniform_spec(kind, ndim, value)
    filled = []
    for a in inputs:
        b = a.copy()
        apply_boundary(b, spec, halo_widths)
        filled.append(b)
    return apply_multi(filled, fn, ndim, halo_widths)


def bricked_launch(u_in: np.ndarray, fn, ndim: int, halo_widths, steps: int = 1) -> np.ndarray:
    """``launch_<name>_bricked``: the flat result over a zero-halo output."""
    return temporal_launch(u_in, np.zeros_like(u_in), fn, ndim, halo_widths, steps)


def to_bricks(flat: np.ndarray, b: int) -> np.ndarray:
    """Flat -> brick-major copy (multigpu_emitter.py:370-404): pad each dim
    to a multiple of ``b`` with zeros, reshape to ``(n0/b, b, n1/b, b, ...)``,
    move brick indices first."""
    shape = flat.shape
    padded_shape = tuple(-(-s // b) * b for s in shape)
    padded = np.zeros(padded_shape, flat.dtype)
    padded[tuple(slice(0, s) for s in shape)] = flat
    nd = flat.ndim
    split = []
    for s in padded_shape:
        split += [s // b, b]
    r = padded.reshape(split)
    return np.ascontiguousarray(r.transpose(list(range(0, 2 * nd, 2)) + list(range(1, 2 * nd, 2))))


def from_bricks(bricked: np.ndarray, shape, b: int) -> np.ndarray:
    nd = len(shape)
    perm = []
    for i in range(nd):
        perm += [i, nd + i]
    padded_shape = tuple(-(-s // b) * b for s in shape)
    flat = bricked.transpose(perm).reshape(padded_shape)
    return np.ascontiguousarray(flat[tuple(slice(0, s) for s in shape)])


def pad_inner_halo(halo_widths, dtype_bytes: int, align_bytes: int = 128):
    """launcher.py:257-273."""
    align = max(1, align_bytes // dtype_bytes)
    inner = -(-halo_widths[-1] // align) * align
    return tuple(halo_widths[:-1]) + (inner,)


def temporal_depth(tile, halo, max_steps: int = 8, smem: int = 49152, dtype_bytes: int = 8) -> int:
    """temporal.py:66-76: largest T with prod(tile + 2*T*halo)*bytes*2 <= smem."""
    for t in range(max_steps, 1, -1):
        expanded = [tile[d] + 2 * t * halo[d] for d in range(len(tile))]
        if math.prod(expanded) * dtype_bytes * 2 <= smem:
            return t
    return 1


__all__ = [name for name in dir() if not name.startswith("_")]


def kahan_update(u_in, c_in, incr):
    """Kahan-compensated ``u += incr`` in the arrays' dtype (float32):
    ``y = incr - c; t = u + y; c' = (t - u) - y``; returns ``(t, c')``."""
    dt = u_in.dtype
    y = np.asarray(incr, dtype=dt) - c_in
    t = u_in + y
    c2 = (t - u_in) - y
    return t, c2


def fused_kahan_step(inputs_by_name: dict, comps: dict, incr_fns: dict, ndim: int, halo,
                     boundary: str | None = None):
    """One step of a Kahan-compensated fused update.

    ``incr_fns`` maps an updated field name to its increment function;
    ``comps`` maps the field name to its compensation array.  With a
    boundary kind, the inputs are boundary-filled (copies) first, as the
    fused-boundary kernels stage them.  Returns ``{name: (u_new, c_new)}``
    with only the interiors meaningful.
    """
    ins = {}
    for k, a in inputs_by_name.items():
        b = a.copy()
        if boundary is not None:
            apply_boundary(b, uniform_spec(boundary, ndim), halo)
        ins[k] = b
    first = next(iter(ins.values()))
    inner = _interior(first.shape, halo)
    out = {}
    for name, fn in incr_fns.items():
        incr = evaluate(ins, fn, ndim, halo, first.shape, first.dtype)
        t, c2 = kahan_update(ins[name][inner], comps[name][inner], incr)
        u_new = np.zeros_like(first)
        c_new = np.zeros_like(first)
        u_new[inner] = t
        c_new[inner] = c2
        out[name] = (u_new, c_new)
    return out


# --------------------------------------------------------------------------- #
# Runge-Kutta stages with FP64 combination, CFL steps (batched solvers)
# --------------------------------------------------------------------------- #


def evaluate_ops(arrays_by_param: dict, fn, ndim: int, halo, shape, dtype, scalars=None):
    """Like ``evaluate`` but scalar parameters are bound from ``scalars`` and a
    tuple-returning body gives a tuple."""
    import inspect

    f = raw_fn(fn)
    params = list(inspect.signature(f).parameters)[:-ndim]
    scalars = scalars or {}
    args = []
    for p in params:
        if p in scalars:
            args.append(float(scalars[p]))
        else:
            args.append(ArrayProxy(arrays_by_param.get(p, np.zeros(shape, dtype)), halo))
    res = array_aware(f)(*args, *([0] * ndim))
    return res if isinstance(res, tuple) else (res,)


def reflect_fill(u: np.ndarray, halo, odd_dims=()) -> None:
    """Reflecting walls with the sign of mirrored values flipped in ``odd_dims``
    (a wall's normal momentum); corners take the product of the signs."""
    apply_boundary(u, uniform_spec("reflecting", u.ndim), halo)
    for d in odd_dims:
        sl = [slice(None)] * u.ndim
        sl[d] = slice(0, halo[d])
        u[tuple(sl)] *= -1
        sl[d] = slice(u.shape[d] - halo[d], u.shape[d])
        u[tuple(sl)] *= -1


def rk_stage(op, names, stage, base, acc, coeffs, dt: float, ndim: int, halo, scalars=None,
             boundary=None, odd=None):
    """One fused RK stage as the stage kernels compute it.

    ``stage``/``base``/``acc``: tuples of state arrays (base/acc may be None);
    ``coeffs = (a, b, c, w)``.  The stage state is boundary-filled (copies)
    first when ``boundary`` is ``"reflecting"`` (``odd[m]``: dims whose mirror
    flips field m's sign).  Returns (next, acc_next) tuples, interiors only
    meaningful; the combination is FP64 in the kernels' order with one
    rounding to the field dtype.
    """
    a, b, c, w = coeffs
    filled = []
    for m, s in enumerate(stage):
        t = s.copy()
        if boundary == "reflecting":
            reflect_fill(t, halo, (odd or {}).get(m, ()))
        elif boundary is not None:
            apply_boundary(t, uniform_spec(boundary, ndim), halo)
        filled.append(t)
    dt_ = stage[0].dtype
    L = evaluate_ops(dict(zip(names, filled)), op, ndim, halo, stage[0].shape, dt_, scalars)
    inner = _interior(stage[0].shape, halo)
    nxt, accn = [], []
    cdt = c * dt
    for m, lm in enumerate(L):
        lm64 = np.asarray(lm, dtype=np.float64)
        x = None
        if a != 0.0:
            bb = base[m][inner].astype(np.float64)
            x = bb if a == 1.0 else a * bb
        if b != 0.0:
            sv = stage[m][inner].astype(np.float64)
            y = sv if b == 1.0 else b * sv
            x = y if x is None else x + y
        term = cdt * lm64
        x = term if x is None else x + term
        out = np.zeros_like(stage[m])
        out[inner] = x.astype(dt_)
        nxt.append(out)
        if w is not None:
            ao = np.zeros_like(stage[m])
            ao[inner] = (acc[m][inner].astype(np.float64) + (w * dt) * lm64).astype(dt_)
            accn.append(ao)
    return tuple(nxt), tuple(accn)


RK_TABLES = {
    "euler": [(1.0, 0.0, 1.0, None, "u", "u", None, "s1")],
    "rk2": [(1.0, 0.0, 0.5, None, "u", "u", None, "s1"),
            (1.0, 0.0, 1.0, None, "u", "s1", None, "u")],
    "rk4": [(1.0, 0.0, 0.5, 1.0 / 6.0, "u", "u", "u", "s1"),
            (1.0, 0.0, 0.5, 1.0 / 3.0, "u", "s1", "acc", "s2"),
            (1.0, 0.0, 1.0, 1.0 / 3.0, "u", "s2", "acc", "s3"),
            (1.0, 0.0, 1.0 / 6.0, None, "acc", "s3", None, "u")],
    "ssprk3": [(1.0, 0.0, 1.0, None, "u", "u", None, "s1"),
               (0.75, 0.25, 0.25, None, "u", "s1", None, "s2"),
               (1.0 / 3.0, 2.0 / 3.0, 2.0 / 3.0, None, "u", "s2", None, "u")],
}


def rk_step(op, names, state, method: str, dt: float, ndim: int, halo, scalars=None,
            boundary=None, odd=None):
    """One RK step (the fused-stage formulation); returns the new state tuple."""
    bufs = {"u": tuple(state)}
    for a, b, c, w, base, stage, acc_in, out in RK_TABLES[method]:
        nxt, accn = rk_stage(op, names, bufs[stage], bufs[base] if a != 0.0 else None,
                             bufs[acc_in] if w is not None else None, (a, b, c, w), dt, ndim,
                             halo, scalars, boundary, odd)
        inner = _interior(state[0].shape, halo)
        if out == "u":
            new = []
            for old, n in zip(bufs["u"], nxt):
                t = old.copy()
                t[inner] = n[inner]
                new.append(t)
            bufs["u"] = tuple(new)
        else:
            bufs[out] = nxt
        if w is not None:
            bufs["acc"] = accn
    if RK_TABLES[method][-1][7] != "u":
        last = bufs[RK_TABLES[method][-1][7]]
        new = []
        for old, n in zip(state, last):
            t = old.copy()
            inner = _interior(old.shape, halo)
            t[inner] = n[inner]
            new.append(t)
        bufs["u"] = tuple(new)
    return bufs["u"]


def cfl_dt(speed_fn, state, names, ndim, halo, cfl: float, scale: float) -> float:
    """dt = cfl * scale / max(signal speed over the interior)."""
    (sp,) = evaluate_ops(dict(zip(names, state)), speed_fn, ndim, halo, state[0].shape,
                         state[0].dtype)
    smax = float(np.max(np.asarray(sp, dtype=np.float64)))
    return (cfl * scale) / smax
