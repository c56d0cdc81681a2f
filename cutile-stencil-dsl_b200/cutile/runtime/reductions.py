"""FP64 global reductions on the device: mass, energy, residual, max.

Fields may be float32 or float64; accumulation is FP64 in a fixed order
(``csd_reduce``: one partial per block, then one block over the partials),
so a result depends on the number of blocks only, never on scheduling --
repeated runs and co-scheduled work give identical bits.  Results stay on
the device as 0-d float64 tensors (read them with ``.item()`` when needed).
"""

from __future__ import annotations

import ctypes
import threading

from cutile.runtime import native

SUM, SUMSQ, MAXABS, DIFF_SUMSQ, DIFF_MAXABS = 0, 1, 2, 3, 4
DEFAULT_BLOCKS = 296  # 2 per SM on B200; fixed so results do not depend on the device

_scratch: dict = {}
_lock = threading.Lock()


def _partials(device, nblocks: int):
    import torch

    key = (device, nblocks)
    with _lock:
        buf = _scratch.get(key)
        if buf is None:
            buf = torch.empty(nblocks, dtype=torch.float64, device=device)
            _scratch[key] = buf
    return buf


def reduce(op: int, a, halo, b=None, out=None, stream=None, nblocks: int = DEFAULT_BLOCKS,
           partials=None):
    """Generic entry: ``op`` over the interior of ``a`` (and ``b``)."""
    import torch

    lib = native.library()
    fa = native.field_of(a)
    fb = native.field_of(b) if b is not None else None
    h = (ctypes.c_int * 3)(*([int(x) for x in halo] + [0] * (3 - len(halo))))
    if out is None:
        out = torch.empty((), dtype=torch.float64, device=a.device)
    if partials is None:
        partials = _partials(a.device, nblocks)
    native.check(lib.csd_reduce(ctypes.byref(fa), ctypes.byref(fb) if fb is not None else None,
                                h, op, ctypes.c_void_p(partials.data_ptr()), nblocks,
                                ctypes.c_void_p(out.data_ptr()),
                                ctypes.c_void_p(native.stream_handle(stream))))
    return out


def mass(u, halo, **kw):
    """Sum of the interior (FP64)."""
    return reduce(SUM, u, halo, **kw)


def energy(u, halo, **kw):
    """Sum of squares of the interior (FP64)."""
    return reduce(SUMSQ, u, halo, **kw)


def residual(a, b, halo, **kw):
    """L2 norm of ``a - b`` over the interior (FP64, sqrt taken on the device)."""
    import torch

    return torch.sqrt(reduce(DIFF_SUMSQ, a, halo, b=b, **kw))


def max_abs(u, halo, **kw):
    return reduce(MAXABS, u, halo, **kw)


def max_abs_diff(a, b, halo, **kw):
    return reduce(DIFF_MAXABS, a, halo, b=b, **kw)


__all__ = ["reduce", "mass", "energy", "residual", "max_abs", "max_abs_diff", "SUM", "SUMSQ",
           "MAXABS", "DIFF_SUMSQ", "DIFF_MAXABS", "DEFAULT_BLOCKS"]
