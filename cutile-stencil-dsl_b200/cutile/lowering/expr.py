"""Stencil body -> exact evaluation program.

The reference turns the D1 body into one Python expression string
(``_reconstruct_expr``, cutile/lowering/stencil_to_target.py:335-451): it
folds constant sub-expressions in float64 (only when both operands are
constants, which is exactly when Python itself evaluates them first), keeps
the DSL's left-to-right term order, and re-associates a top-level sum in
spatial order for very wide stencils.

Here the same walk produces an SSA program that the CUDA emitter turns into
one statement per op, so no parenthesisation can change the evaluation
order, plus a readable infix ``expression`` for inspection.  Each value
carries its NumPy type, because the oracle is NumPy running the user's
function and its promotion rules decide the precision of every operation:

* ``w`` -- a Python float (weak scalar): constants and folded
  sub-expressions.  Combined with an array it is rounded to the array's
  dtype (NEP 50), so a float32 stencil multiplies by ``float32(0.1)``;
* ``f32`` / ``f64`` -- arrays;  ``array op array`` promotes to the wider;
* ``b`` -- a boolean array from a comparison, done in the promoted dtype of
  its operands; ``wb`` a Python bool (both operands weak);
* ``where(cond, a, b)`` follows ``np.where``: two weak branches give
  float64, one weak branch takes the other's dtype; a Python-bool condition
  with weak branches stays a Python float (the oracle's ``where`` picks one).

Statement format (one string each, parsed back by the CUDA emitter):
``v<k> = <op> <operands> : <type>`` with ops ``const <repr>``,
``load a<j>``, ``addf/subf/mulf/divf/maxf/minf x, y``, ``negf/absf/sqrt x``,
``cmp.<pred> x, y``, ``select c, x, y`` and ``cast x``, and the operand
list naming values (``v<k>``) or accesses (``a<j>``).
"""

from __future__ import annotations

import math

import numpy as np

from cutile.dialects import arith as A
from cutile.dialects.cutile_stencil.dialect import AccessOp, YieldOp
from cutile.ir.core import FloatAttr

_CMPF_SYMBOLS = {1: "==", 2: ">", 3: ">=", 4: "<", 5: "<=", 6: "!=", 13: "!="}
_CMPF_NAMES = {1: "oeq", 2: "ogt", 3: "oge", 4: "olt", 5: "ole", 6: "one", 13: "une"}

_BIN = {A.AddfOp: ("addf", "+"), A.SubfOp: ("subf", "-"), A.MulfOp: ("mulf", "*"),
        A.DivfOp: ("divf", "/")}


def _f32_exact(value: float) -> bool:
    """True when *value* survives a float32 round trip (stencil_to_target.py:255-257)."""
    return math.isfinite(value) and float(np.float32(value)) == value


def _fold(kind: str, a: float, b: float):
    try:
        if kind == "addf":
            return a + b
        if kind == "subf":
            return a - b
        if kind == "mulf":
            return a * b
        if kind == "divf":
            return a / b
    except ZeroDivisionError:
        return None
    return None


def _promote(*types: str) -> str:
    arrays = [t for t in types if t in ("f32", "f64")]
    if not arrays:
        return "w"
    return "f64" if "f64" in arrays else "f32"


def _top_level_ops(expr: str) -> set[str]:
    found: set[str] = set()
    depth = 0
    for k, ch in enumerate(expr):
        if ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        elif depth == 0 and ch in "+-*/" and expr[k - 1:k] == " " and expr[k + 1:k + 2] == " ":
            found.add(ch)
    return found


def _paren(expr: str, ops: tuple[str, ...]) -> str:
    return f"({expr})" if _top_level_ops(expr) & set(ops) else expr


class Program:
    """Result of lowering one stencil body."""

    def __init__(self):
        self.lines: list[str] = []
        self.result: str = ""
        self.result_type: str = "w"
        self.expression: str = ""
        self.access_uses: dict[int, int] = {}
        self.extra_returns: list[tuple[str, int]] = []
        self.n_outputs = 1


def build_program(block, access_index: dict, field_dtype: str, spatial_order: bool = False,
                  access_offsets: dict | None = None, scalar_args=()) -> Program:
    """Lower the D1 *block* into a :class:`Program`.

    ``access_index`` maps each access op result to its index in the kernel's
    (possibly merged) access list; ``field_dtype`` is ``"f32"`` or ``"f64"``;
    ``scalar_args`` are the block arguments of the stencil's scalar
    parameters (operands ``s<k>``: Python floats given at launch).
    """
    prog = Program()
    const: dict = {}     # value -> python float (folded constants)
    vtype: dict = {}     # value -> numpy kind
    name: dict = {}      # value -> SSA operand name
    infix: dict = {}     # value -> readable expression
    counter = [0]
    for k, arg in enumerate(scalar_args):
        name[arg] = f"s{k}"
        vtype[arg] = "w"
        infix[arg] = f"s{k}"

    def new(line_rhs: str, t: str) -> str:
        n = f"v{counter[0]}"
        counter[0] += 1
        prog.lines.append(f"{n} = {line_rhs} : {t}")
        return n

    def operand(v) -> str:
        if v in const:
            if v not in name:
                name[v] = new(f"const {const[v]!r}", "w")
            return name[v]
        return name[v]

    def text(v) -> str:
        if v in const:
            return repr(float(const[v]))
        return infix[v]

    result_value = None
    for op in block.ops:
        if isinstance(op, AccessOp):
            j = access_index[op.res]
            name[op.res] = f"a{j}"
            vtype[op.res] = field_dtype
            infix[op.res] = f"a{j}"
            prog.access_uses[j] = prog.access_uses.get(j, 0)
        elif isinstance(op, A.ConstantOp):
            val = op.properties["value"]
            const[op.result] = float(val.data) if isinstance(val, FloatAttr) else float(val.data)
            vtype[op.result] = "w"
        elif isinstance(op, tuple(_BIN)):
            kind, sym = _BIN[type(op)]
            lhs, rhs = op.lhs, op.rhs
            if lhs in const and rhs in const:
                folded = _fold(kind, const[lhs], const[rhs])
                if folded is not None and math.isfinite(folded):
                    const[op.result] = folded
                    vtype[op.result] = "w"
                    continue
            t = _promote(vtype[lhs], vtype[rhs])
            name[op.result] = new(f"{kind} {operand(lhs)}, {operand(rhs)}", t)
            vtype[op.result] = t
            left, right = text(lhs), text(rhs)
            if kind == "subf":
                right = _paren(right, ("+", "-"))
            elif kind == "mulf":
                left = _paren(left, ("+", "-"))
                right = _paren(right, ("+", "-", "/"))
            elif kind == "divf":
                left = _paren(left, ("+", "-"))
                right = _paren(right, ("+", "-", "*", "/"))
            elif kind == "addf":
                right = _paren(right, ("+", "-"))
            infix[op.result] = f"{left} {sym} {right}"
        elif isinstance(op, A.NegfOp):
            x = op.operand
            if x in const:
                const[op.result] = -const[x]
                vtype[op.result] = "w"
                continue
            name[op.result] = new(f"negf {operand(x)}", vtype[x])
            vtype[op.result] = vtype[x]
            infix[op.result] = f"-({text(x)})"
        elif isinstance(op, (A.MaximumfOp, A.MinimumfOp)):
            is_max = isinstance(op, A.MaximumfOp)
            if op.lhs in const and op.rhs in const:
                const[op.result] = (max if is_max else min)(const[op.lhs], const[op.rhs])
                vtype[op.result] = "w"
                continue
            t = _promote(vtype[op.lhs], vtype[op.rhs])
            kind = "maxf" if is_max else "minf"
            name[op.result] = new(f"{kind} {operand(op.lhs)}, {operand(op.rhs)}", t)
            vtype[op.result] = t
            infix[op.result] = f"{'maximum' if is_max else 'minimum'}({text(op.lhs)}, {text(op.rhs)})"
        elif isinstance(op, A.AbsFOp):
            x = op.operand
            if x in const:
                const[op.result] = abs(const[x])
                vtype[op.result] = "w"
                continue
            name[op.result] = new(f"absf {operand(x)}", vtype[x])
            vtype[op.result] = vtype[x]
            infix[op.result] = f"abs({text(x)})"
        elif isinstance(op, A.SqrtOp):
            x = op.operand
            if x in const and const[x] >= 0:
                const[op.result] = math.sqrt(const[x])
                vtype[op.result] = "w"
                continue
            name[op.result] = new(f"sqrt {operand(x)}", vtype[x])
            vtype[op.result] = vtype[x]
            infix[op.result] = f"sqrt({text(x)})"
        elif isinstance(op, A.CmpfOp):
            pred = op.predicate.data
            if pred not in _CMPF_NAMES:
                raise ValueError(f"Unsupported cmpf predicate {pred}")
            t = _promote(vtype[op.lhs], vtype[op.rhs])
            rt = "wb" if t == "w" else "b"
            # the comparison runs in the promoted dtype: record it on the op
            cmp_t = "f64" if t == "w" else t
            name[op.result] = new(
                f"cmp.{_CMPF_NAMES[pred]} {operand(op.lhs)}, {operand(op.rhs)} @{cmp_t}", rt)
            vtype[op.result] = rt
            infix[op.result] = f"({text(op.lhs)} {_CMPF_SYMBOLS[pred]} {text(op.rhs)})"
        elif isinstance(op, A.SelectOp):
            c, a, b = op.operands
            ta, tb = vtype[a], vtype[b]
            if vtype[c] == "wb" and ta == "w" and tb == "w":
                t = "w"
            elif ta == "w" and tb == "w":
                t = "f64"
            else:
                t = _promote(ta, tb)
            name[op.result] = new(f"select {operand(c)}, {operand(a)}, {operand(b)}", t)
            vtype[op.result] = t
            infix[op.result] = f"where({text(c)}, {text(a)}, {text(b)})"
        elif isinstance(op, YieldOp):
            result_value = op.value
            yields = list(op.values)
        else:
            raise ValueError(f"unsupported op in stencil body: {op.name}")

    if result_value is None:
        raise ValueError("stencil body has no yield")
    if len(yields) > 1:
        # tuple-returning body: one output per element, in order
        for i, v in enumerate(yields):
            prog.extra_returns.append((operand(v), i))
        prog.result = prog.extra_returns[0][0]
        prog.result_type = vtype[yields[0]]
        prog.expression = "(" + ", ".join(text(v) for v in yields) + ")"
        prog.n_outputs = len(yields)
        return prog
    if spatial_order and access_offsets:
        # Opt-in re-association of a top-level sum in spatial access order
        # (the reference's default above 64 loads, stencil_to_target.py:443-448).
        terms = _flatten_sum(result_value, const)
        if len(terms) > 1:
            terms.sort(key=lambda t: _term_offset(t[1], access_offsets))
            return _rebuild_sum(prog, terms, operand, text, vtype, new, const)
    prog.result = operand(result_value)
    prog.result_type = vtype[result_value]
    prog.expression = text(result_value)
    for line in prog.lines:
        for tok in line.replace(",", " ").split():
            if tok.startswith("a") and tok[1:].isdigit():
                j = int(tok[1:])
                prog.access_uses[j] = prog.access_uses.get(j, 0) + 1
    return prog


def _flatten_sum(value, const, sign=1):
    owner = getattr(value, "owner", None)
    if value not in const and isinstance(owner, A.AddfOp):
        return _flatten_sum(owner.lhs, const, sign) + _flatten_sum(owner.rhs, const, sign)
    if value not in const and isinstance(owner, A.SubfOp):
        return _flatten_sum(owner.lhs, const, sign) + _flatten_sum(owner.rhs, const, -sign)
    return [(sign, value)]


def _term_offset(value, access_offsets):
    found = []
    stack = [value]
    seen = set()
    while stack:
        v = stack.pop()
        if id(v) in seen:
            continue
        seen.add(id(v))
        if v in access_offsets:
            found.append(access_offsets[v])
            continue
        owner = getattr(v, "owner", None)
        if owner is not None and hasattr(owner, "operands"):
            stack.extend(owner.operands)
    return (1, min(found)) if found else (0, ())


def _rebuild_sum(prog, terms, operand, text, vtype, new, const):
    acc = None
    acc_t = "w"
    parts = []
    for i, (sign, v) in enumerate(terms):
        vn = operand(v)
        t = vtype.get(v, "w")
        if acc is None:
            if sign < 0:
                acc = new(f"negf {vn}", t)
                parts.append(f"-({text(v)})")
            else:
                acc = vn
                parts.append(text(v))
            acc_t = t
            continue
        acc_t = _promote(acc_t, t)
        acc = new(f"{'subf' if sign < 0 else 'addf'} {acc}, {vn}", acc_t)
        parts.append(f"{'-' if sign < 0 else '+'} {_paren(text(v), ('+', '-'))}")
    prog.result = acc
    prog.result_type = acc_t
    prog.expression = " ".join(parts)
    return prog


__all__ = ["Program", "build_program", "_f32_exact"]


def kahan_rewrite(prog: Program, center_access: dict, comp_access: int, out_index: int,
                  comp_out_index: int) -> int:
    """Turn a ``u + incr`` program into a Kahan-compensated FP32 update.

    ``center_access`` maps access indices that read a field at offset zero to
    that field; ``comp_access`` is the access index of the compensation field.
    The program's final ``addf`` (either operand order) must add a center read
    to the increment.  Returns the array index of the updated field.  The new
    tail is (all float32, round-to-nearest, no contraction)::

        y  = incr - c          t  = u + y
        c' = (t - u) - y       outputs: t -> out_index, c' -> comp_out_index
    """
    last = prog.lines[-1]
    lhs, rhs = last.split(" = ", 1)
    body, typ = rhs.rsplit(" : ", 1)
    if lhs != prog.result or not body.startswith("addf "):
        raise ValueError("Kahan-compensated updates need a body of the form `u + increment`")
    a, b = [t.strip() for t in body[5:].split(",")]
    def center(tok):
        return tok.startswith("a") and tok[1:].isdigit() and int(tok[1:]) in center_access
    if center(a):
        u, incr = a, b
    elif center(b):
        u, incr = b, a
    else:
        raise ValueError("Kahan-compensated updates need a body of the form `u[i, j] + increment`")
    field = center_access[int(u[1:])]
    lines = prog.lines[:-1]
    c = f"a{comp_access}"
    lines.append(f"k0 = cast {incr} : f32")
    lines.append(f"k1 = subf k0, {c} : f32")
    lines.append(f"k2 = addf {u}, k1 : f32")
    lines.append(f"k3 = subf k2, {u} : f32")
    lines.append(f"k4 = subf k3, k1 : f32")
    prog.lines = lines
    prog.result = "k2"
    prog.result_type = "f32"
    prog.extra_returns = [("k2", out_index), ("k4", comp_out_index)]
    prog.expression = f"kahan({prog.expression})"
    return field
