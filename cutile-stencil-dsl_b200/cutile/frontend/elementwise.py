"""Element-wise helpers usable in stencil bodies and on the host.

Inside a ``@stencil`` body the parser lowers ``max``/``min``/``abs``/``where``
(and ``sqrt``) to IR ops.  When the same Python function runs on NumPy or
torch arrays (``CompileResult.validate``), the builtins ``max``/``min`` reject
arrays, so these dispatch to the array library of their operands, as the
reference's ``cutile.reference.elementwise`` does (elementwise.py:17-52).
"""

from __future__ import annotations

import builtins
import importlib
import math
import types


def _xp(*args):
    for a in args:
        mod = type(a).__module__.split(".")[0]
        if mod in ("numpy", "torch"):
            return importlib.import_module(mod)
    return None


def maximum(a, b):
    xp = _xp(a, b)
    return builtins.max(a, b) if xp is None else xp.maximum(*_coerce(xp, a, b))


def minimum(a, b):
    xp = _xp(a, b)
    return builtins.min(a, b) if xp is None else xp.minimum(*_coerce(xp, a, b))


def where(cond, a, b):
    xp = _xp(cond, a, b)
    return (a if cond else b) if xp is None else xp.where(*_coerce(xp, cond, a, b))


def sqrt(x):
    xp = _xp(x)
    return math.sqrt(x) if xp is None else xp.sqrt(x)


def _coerce(xp, *args):
    if xp.__name__ != "torch":
        return args
    ref = next(a for a in args if isinstance(a, xp.Tensor))
    return tuple(a if isinstance(a, xp.Tensor) else xp.tensor(a, dtype=ref.dtype, device=ref.device)
                 for a in args)


def array_aware(fn):
    """``fn`` with ``max``/``min`` swapped for the array-aware versions and
    ``where``/``sqrt`` available, so a stencil body runs on array slices."""
    g = dict(fn.__globals__)
    b = dict(vars(builtins))
    b["max"] = maximum
    b["min"] = minimum
    g["__builtins__"] = b
    g.setdefault("where", where)
    g.setdefault("sqrt", sqrt)
    return types.FunctionType(fn.__code__, g, fn.__name__, fn.__defaults__, fn.__closure__)
