"""Python AST to Dialect 1 (``cutile_stencil``) IR.

Follows the reference parser (cutile/frontend/parser.py:62-664):

* array parameters are the parameters used as subscript targets, index
  variables the ones used inside subscripts (parser.py:482-523), with the
  same fallbacks;
* ``ndim``/``order`` are inferred from the accesses when not given
  (``order = 2 * max|offset|``, parser.py:157-177);
* constants come from the closure, an explicit ``constants`` dict and the
  numeric module globals the return expression names (parser.py:369-383,
  556-573);
* one ``access`` op per distinct ``(array, offset)`` in first-use order,
  then the expression as ``arith``/``math`` ops in Python evaluation order,
  then ``yield`` (parser.py:578-621);
* a ``str`` or ``dict`` boundary becomes a ``BoundaryAttr`` (parser.py:623-631).

Two extensions, both additive: straight-line local assignments
(``flux = ...; return ...``) bind their names to the assigned value (the
reference only harvests their accesses and then rejects the bare name), and
``sqrt(x)`` lowers to ``math.sqrt``.  A uniform ``BoundarySpec`` is accepted
as a boundary too (the reference silently drops it).
"""

from __future__ import annotations

import ast
import inspect
import math
import textwrap

from cutile.dialects import arith as A
from cutile.dialects.cutile_stencil.dialect import AccessOp, BoundaryAttr, FuncOp, YieldOp
from cutile.ir.core import (
    Block,
    DictionaryAttr,
    FileLineColLoc,
    FloatAttr,
    ModuleOp,
    Region,
    SSAValue,
    f32,
    f64,
)

_FLOAT_TYPE_MAP = {"float64": f64, "float32": f32}


class _ParseError(Exception):
    """Raised when the stencil function cannot be parsed."""


ParseError = _ParseError


# --------------------------------------------------------------------------- #
# Subscript offsets
# --------------------------------------------------------------------------- #


def _resolve_offset(node: ast.expr, index_vars: list[str]) -> list[int]:
    """``u[i-1, j+2]`` slice -> ``[-1, 2]`` (parser.py:62-77)."""
    elts = node.elts if isinstance(node, ast.Tuple) else [node]
    return [_resolve_single_offset(e, index_vars) for e in elts]


def _resolve_single_offset(node: ast.expr, index_vars: list[str]) -> int:
    """``i`` -> 0, ``i + k`` -> k, ``i - k`` -> -k, ``k + i`` -> k (parser.py:80-121)."""
    if isinstance(node, ast.Name):
        if node.id in index_vars:
            return 0
        raise _ParseError(f"Unknown index variable '{node.id}', expected one of {index_vars}")
    if isinstance(node, ast.BinOp):
        if isinstance(node.left, ast.Name) and node.left.id in index_vars:
            const = _eval_constant_expr(node.right)
            if isinstance(node.op, ast.Add):
                return const
            if isinstance(node.op, ast.Sub):
                return -const
            raise _ParseError(f"Unsupported offset operation: {type(node.op).__name__}")
        if isinstance(node.right, ast.Name) and node.right.id in index_vars:
            const = _eval_constant_expr(node.left)
            if isinstance(node.op, ast.Add):
                return const
            raise _ParseError(f"Unsupported offset operation: {type(node.op).__name__}")
    raise _ParseError(f"Cannot resolve subscript expression to an offset: {ast.dump(node)}")


def _eval_constant_expr(node: ast.expr) -> int:
    if isinstance(node, ast.Constant) and isinstance(node.value, (int, float)) \
            and not isinstance(node.value, bool):
        return int(node.value)
    if isinstance(node, ast.UnaryOp) and isinstance(node.op, ast.USub):
        return -_eval_constant_expr(node.operand)
    raise _ParseError(f"Expected compile-time integer constant, got: {ast.dump(node)}")


def _collect_accesses(node, array_params, index_vars):
    """All ``(array, offsets, node)`` in *node*, in source order (parser.py:135-154)."""
    out = []
    if isinstance(node, ast.Subscript) and isinstance(node.value, ast.Name) \
            and node.value.id in array_params:
        out.append((node.value.id, _resolve_offset(node.slice, index_vars), node))
        return out
    for child in ast.iter_child_nodes(node):
        if isinstance(child, ast.expr):
            out.extend(_collect_accesses(child, array_params, index_vars))
    return out


def _infer_ndim_order(accesses) -> tuple[int, int]:
    if not accesses:
        raise _ParseError("No array accesses found; cannot infer ndim/order")
    ndim = len(accesses[0][1])
    max_offset = 0
    for item in accesses:
        offsets = item[1]
        if len(offsets) != ndim:
            raise _ParseError(f"Inconsistent dimensionality: expected {ndim}, got {len(offsets)}")
        for o in offsets:
            max_offset = max(max_offset, abs(o))
    return ndim, 2 * max_offset


# --------------------------------------------------------------------------- #
# Expression builder
# --------------------------------------------------------------------------- #


class _ExprBuilder:
    """AST expression -> arith/math ops appended to *block* (parser.py:185-361)."""

    _BINARY_CALLS = {"max": A.MaximumfOp, "maximum": A.MaximumfOp,
                     "min": A.MinimumfOp, "minimum": A.MinimumfOp}
    _COMPARE_OPS = {ast.Gt: "ogt", ast.GtE: "oge", ast.Lt: "olt", ast.LtE: "ole",
                    ast.Eq: "oeq", ast.NotEq: "une"}
    _BINOPS = {ast.Add: A.AddfOp, ast.Sub: A.SubfOp, ast.Mult: A.MulfOp, ast.Div: A.DivfOp}

    def __init__(self, block, float_type, access_map, constant_map, index_vars,
                 source_file=None, source_line_offset=0):
        self.block = block
        self.float_type = float_type
        self.access_map = access_map
        self.constant_map = constant_map
        self.index_vars = index_vars
        self.locals: dict[str, SSAValue] = {}
        self._const_cache: dict[tuple, SSAValue] = {}
        self._source_file = source_file
        self._source_line_offset = source_line_offset

    def _loc(self, op, node):
        if self._source_file is not None:
            op.location = FileLineColLoc(self._source_file,
                                         getattr(node, "lineno", 0) + self._source_line_offset,
                                         getattr(node, "col_offset", 0))

    def _add(self, op, node):
        self._loc(op, node)
        self.block.add_op(op)
        return op.results[0]

    def _emit_const(self, value: float, node=None) -> SSAValue:
        key = (value, math.copysign(1.0, value)) if value == value else ("nan",)
        if key in self._const_cache:
            return self._const_cache[key]
        v = self._add(A.ConstantOp(FloatAttr(value, self.float_type)), node)
        self._const_cache[key] = v
        return v

    def build(self, node: ast.expr) -> SSAValue:
        if isinstance(node, ast.BinOp):
            op_cls = self._BINOPS.get(type(node.op))
            left = self.build(node.left)
            right = self.build(node.right)
            if op_cls is None:
                raise _ParseError(f"Unsupported binary operator: {type(node.op).__name__}")
            return self._add(op_cls(left, right), node)
        if isinstance(node, ast.UnaryOp):
            if isinstance(node.op, ast.USub):
                return self._add(A.NegfOp(self.build(node.operand)), node)
            if isinstance(node.op, ast.UAdd):
                return self.build(node.operand)
            raise _ParseError(f"Unsupported unary operator: {type(node.op).__name__}")
        if isinstance(node, ast.Constant):
            if isinstance(node.value, (int, float)) and not isinstance(node.value, bool):
                return self._emit_const(float(node.value), node)
            raise _ParseError(f"Unsupported constant type: {type(node.value)}")
        if isinstance(node, ast.Subscript):
            if not isinstance(node.value, ast.Name):
                raise _ParseError("Subscript target must be a simple name")
            key = (node.value.id, tuple(_resolve_offset(node.slice, self.index_vars)))
            if key not in self.access_map:
                raise _ParseError(f"Access {key[0]}{list(key[1])} not found in access map")
            return self.access_map[key]
        if isinstance(node, ast.Name):
            if node.id in self.locals:
                return self.locals[node.id]
            if node.id in self.constant_map:
                return self._emit_const(self.constant_map[node.id], node)
            raise _ParseError(
                f"Unknown variable '{node.id}'. Not an array parameter or known constant. "
                f"If it is a closure variable, pass it via the 'constants' argument.")
        if isinstance(node, ast.Call):
            return self._build_call(node)
        if isinstance(node, ast.Compare):
            if len(node.ops) != 1 or len(node.comparators) != 1:
                raise _ParseError("Unsupported chained comparison")
            pred = self._COMPARE_OPS.get(type(node.ops[0]))
            if pred is None:
                raise _ParseError(f"Unsupported comparison: {type(node.ops[0]).__name__}")
            lhs = self.build(node.left)
            rhs = self.build(node.comparators[0])
            return self._add(A.CmpfOp(lhs, rhs, pred), node)
        raise _ParseError(f"Unsupported expression node: {type(node).__name__} ({ast.dump(node)})")

    def _build_call(self, node: ast.Call) -> SSAValue:
        func = node.func
        fname = func.id if isinstance(func, ast.Name) else (
            func.attr if isinstance(func, ast.Attribute) else None)
        if node.keywords or fname is None:
            raise _ParseError(f"Unsupported call: {ast.dump(node)}")
        n = len(node.args)
        if fname in self._BINARY_CALLS and n == 2:
            a = self.build(node.args[0])
            b = self.build(node.args[1])
            op = self._BINARY_CALLS[fname](a, b)
        elif fname in ("abs", "fabs") and n == 1:
            op = A.AbsFOp(self.build(node.args[0]))
        elif fname == "sqrt" and n == 1:
            op = A.SqrtOp(self.build(node.args[0]))
        elif fname == "where" and n == 3:
            cond = self.build(node.args[0])
            a = self.build(node.args[1])
            b = self.build(node.args[2])
            op = A.SelectOp(cond, a, b)
        else:
            raise _ParseError(
                f"Unsupported call '{fname}' with {n} argument(s); supported: max(a, b), "
                f"min(a, b), abs(x), sqrt(x), where(cond, a, b)")
        return self._add(op, node)


# --------------------------------------------------------------------------- #
# Main parser
# --------------------------------------------------------------------------- #


def _extract_constants(fn) -> dict[str, float]:
    """Numeric closure variables (parser.py:369-383)."""
    constants: dict[str, float] = {}
    if fn.__code__.co_freevars and fn.__closure__:
        for name, cell in zip(fn.__code__.co_freevars, fn.__closure__):
            try:
                val = cell.cell_contents
            except ValueError:
                continue
            if isinstance(val, (int, float)) and not isinstance(val, bool):
                constants[name] = float(val)
    return constants


def _boundary_attr(boundary):
    if boundary is None:
        return None
    if isinstance(boundary, str):
        return BoundaryAttr(boundary)
    if isinstance(boundary, dict):
        bc_type = boundary.get("type", boundary.get("bc_type", "dirichlet"))
        return BoundaryAttr(bc_type, boundary.get("value", None))
    to_dict = getattr(boundary, "to_dict", None)
    if to_dict is not None:
        d = to_dict()
        return BoundaryAttr(d["type"], d.get("value"))
    return None


def parse_stencil(fn, ndim: int | None, order: int | None, dtype: str = "float64",
                  boundary=None, constants: dict[str, float] | None = None) -> ModuleOp:
    """Parse a stencil function into a ``ModuleOp`` holding one D1 ``FuncOp``."""
    source = textwrap.dedent(inspect.getsource(fn))
    tree = ast.parse(source)
    source_file = None
    source_line_offset = 0
    try:
        source_file = inspect.getfile(fn)
        _, start = inspect.getsourcelines(fn)
        source_line_offset = start - 1
    except (OSError, TypeError):
        pass

    func_def = next((n for n in ast.walk(tree)
                     if isinstance(n, (ast.FunctionDef, ast.AsyncFunctionDef))), None)
    if func_def is None:
        raise _ParseError("No function definition found in source")
    func_name = func_def.name
    params = [a.arg for a in func_def.args.args]
    if len(params) < 2:
        raise _ParseError(
            f"Stencil function '{func_name}' must have at least 2 parameters "
            f"(array + index variables), got {len(params)}: {params}")

    return_node = next((n for n in ast.walk(func_def)
                        if isinstance(n, ast.Return) and n.value is not None), None)
    if return_node is None:
        raise _ParseError(f"Stencil function '{func_name}' must have a return statement")
    return_expr = return_node.value
    assigns = [s for s in func_def.body if isinstance(s, ast.Assign)]

    # Array parameters vs index variables, from subscript usage.
    subscript_arrays: set[str] = set()
    subscript_indices: set[str] = set()
    for root in [return_expr] + [s.value for s in assigns]:
        for node in ast.walk(root):
            if isinstance(node, ast.Subscript) and isinstance(node.value, ast.Name) \
                    and node.value.id in params:
                subscript_arrays.add(node.value.id)
                for sub in ast.walk(node.slice):
                    if isinstance(sub, ast.Name) and sub.id in params:
                        subscript_indices.add(sub.id)
    array_params = [p for p in params if p in subscript_arrays]
    index_vars = [p for p in params if p in subscript_indices]
    if not array_params:
        array_params = [params[0]]
        index_vars = params[1:]
    if not index_vars:
        index_vars = [p for p in params if p not in set(array_params)]
    # Scalar parameters (an extension): parameters that are neither arrays
    # nor index variables but are read as bare names; their values are given
    # at launch (per grid) and behave like Python float constants.
    bare_names = {n.id for root in [return_expr] + [s.value for s in assigns]
                  for n in ast.walk(root) if isinstance(n, ast.Name)}
    scalar_params = [p for p in params if p not in set(array_params) and p not in set(index_vars)
                     and p in bare_names]

    # Accesses: the return expression's first, then the assignments'
    # (parser.py:528-535).
    all_accesses = _collect_accesses(return_expr, array_params, index_vars)
    for s in assigns:
        all_accesses.extend(_collect_accesses(s.value, array_params, index_vars))

    if ndim is None or order is None:
        inf_ndim, inf_order = _infer_ndim_order(all_accesses)
        ndim = inf_ndim if ndim is None else ndim
        order = inf_order if order is None else order

    float_type = _FLOAT_TYPE_MAP.get(dtype)
    if float_type is None:
        raise _ParseError(f"Unsupported dtype '{dtype}'. Use 'float32' or 'float64'.")

    all_constants = _extract_constants(fn)
    if constants:
        all_constants.update(constants)
    referenced = {n.id for root in [return_expr] + [s.value for s in assigns]
                  for n in ast.walk(root) if isinstance(n, ast.Name)}
    local_names = {t.id for s in assigns for t in s.targets if isinstance(t, ast.Name)}
    for name in sorted(referenced):
        if name not in all_constants and name not in set(array_params) and name not in local_names:
            if hasattr(fn, "__globals__") and name in fn.__globals__:
                val = fn.__globals__[name]
                if isinstance(val, (int, float)) and not isinstance(val, bool):
                    all_constants[name] = float(val)

    block = Block()
    field_args = {}
    for idx, ap in enumerate(array_params):
        field_args[ap] = block.insert_arg(float_type, idx)
    scalar_args = {}
    for k, sp in enumerate(scalar_params):
        scalar_args[sp] = block.insert_arg(f64, len(array_params) + k)
    unique: dict[tuple, SSAValue] = {}
    for name, offsets, node in all_accesses:
        key = (name, tuple(offsets))
        if key in unique:
            continue
        acc = AccessOp(field_args[name], list(offsets), float_type, index_names=index_vars)
        if source_file is not None and node is not None:
            acc.location = FileLineColLoc(source_file,
                                          getattr(node, "lineno", 0) + source_line_offset,
                                          getattr(node, "col_offset", 0))
        block.add_op(acc)
        unique[key] = acc.res

    builder = _ExprBuilder(block, float_type, unique, all_constants, index_vars,
                           source_file, source_line_offset)
    builder.locals.update(scalar_args)
    for s in assigns:
        if len(s.targets) != 1 or not isinstance(s.targets[0], ast.Name):
            raise _ParseError("Only simple 'name = expression' assignments are supported")
        builder.locals[s.targets[0].id] = builder.build(s.value)
    if isinstance(return_expr, ast.Tuple):
        # several outputs from one body (an extension): shared sub-expressions
        # are evaluated once for all of them
        results = [builder.build(e) for e in return_expr.elts]
    else:
        results = [builder.build(return_expr)]
    block.add_op(YieldOp(*results))

    constants_attr = None
    if all_constants:
        constants_attr = DictionaryAttr({k: FloatAttr(v, float_type)
                                         for k, v in all_constants.items()})
    func_op = FuncOp(func_name=func_name, ndim=ndim, order=order, body=Region(block),
                     dtype=dtype, boundary=_boundary_attr(boundary), constants=constants_attr,
                     arg_names=array_params)
    if scalar_params:
        from cutile.ir.core import ArrayAttr, StringAttr

        func_op.properties["scalar_names"] = ArrayAttr([StringAttr(n) for n in scalar_params])
    if source_file is not None:
        func_op.location = FileLineColLoc(source_file,
                                          getattr(func_def, "lineno", 0) + source_line_offset,
                                          getattr(func_def, "col_offset", 0))
    return ModuleOp([func_op])
