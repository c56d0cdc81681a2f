"""The ``@stencil`` decorator (reference: cutile/frontend/decorator.py:16-61)."""

from __future__ import annotations

import functools

from cutile.frontend.parser import parse_stencil


def stencil(fn=None, *, ndim=None, order=None, dtype="float64", boundary=None):
    """Turn a Python stencil function into Dialect 1 IR.

    Usage::

        @stencil(ndim=2, order=2)
        def heat(u, i, j):
            return 0.25 * (u[i-1, j] + u[i+1, j] + u[i, j-1] + u[i, j+1])

    The wrapper keeps the original callable and gains ``_ir`` (a
    ``ModuleOp``), ``_fn``, ``_ndim``, ``_order``, ``_dtype`` and
    ``_boundary``.  Both ``@stencil`` and ``@stencil(...)`` work.
    """

    def _wrap(func):
        ir = parse_stencil(func, ndim=ndim, order=order, dtype=dtype, boundary=boundary)

        @functools.wraps(func)
        def wrapper(*args, **kwargs):
            return func(*args, **kwargs)

        wrapper._ir = ir
        wrapper._fn = func
        wrapper._ndim = ndim
        wrapper._order = order
        wrapper._dtype = dtype
        wrapper._boundary = boundary
        return wrapper

    if fn is not None:
        return _wrap(fn)
    return _wrap
