"""The allocation-free reduction entry point, called through the C ABI.

``csd_reduce_noalloc`` serves callers that cannot allocate device memory
(their device memory is owned by another allocator, or their step loop must
not pay for cudaMalloc's synchronisation): it keeps its scratch in a fixed
static device array instead of a caller-provided buffer.  Its results must
equal those of ``csd_reduce`` with caller scratch, on consecutive calls that
reuse the shared array, bit for bit (both run the same deterministic
two-pass kernels with the same block count), up to the array's full
1024-block size.  This file is collected last on purpose.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _lib():
    from cutile.runtime import native

    lib = native.library()
    lib.csd_reduce_noalloc.argtypes = [ctypes.POINTER(native.Field), ctypes.POINTER(native.Field),
                                       ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_int,
                                       ctypes.c_void_p, ctypes.c_void_p]
    return lib, native


def _noalloc(lib, native, op, a, b, halo, nblocks, out):
    fa = native.field_of(a)
    fb = native.field_of(b) if b is not None else None
    h = (ctypes.c_int * 3)(*(list(halo) + [0] * (3 - len(halo))))
    return lib.csd_reduce_noalloc(ctypes.byref(fa), ctypes.byref(fb) if fb is not None else None,
                                  h, op, nblocks, ctypes.c_void_p(out.data_ptr()),
                                  ctypes.c_void_p(native.stream_handle(None)))


@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_noalloc_reduction_matches_caller_scratch_twice(dtype):
    import torch

    from cutile.runtime import reductions as R

    lib, native = _lib()
    dt = getattr(torch, dtype)
    gen = torch.Generator(device="cuda").manual_seed(7)
    a = torch.randn((40, 33, 70), dtype=dt, device="cuda", generator=gen)
    b = torch.randn((40, 33, 70), dtype=dt, device="cuda", generator=gen)
    halo = (1, 2, 3)
    out = torch.empty((), dtype=torch.float64, device="cuda")
    for op in (R.SUM, R.SUMSQ, R.MAXABS, R.DIFF_SUMSQ, R.DIFF_MAXABS):
        bb = b if op in (R.DIFF_SUMSQ, R.DIFF_MAXABS) else None
        for nblocks in (296, 1024):
            want = R.reduce(op, a, halo, b=bb, nblocks=nblocks).item()
            for _ in range(2):  # two calls in a row share the static scratch
                out.fill_(np.nan)
                assert _noalloc(lib, native, op, a, bb, halo, nblocks, out) == 0, \
                    lib.csd_last_error().decode()
                got = out.item()
                # the same deterministic kernels with the same block count:
                # the sums agree bit for bit
                assert got == want, (op, nblocks, got, want)


def test_noalloc_rejects_more_blocks_than_the_static_scratch():
    import torch

    lib, native = _lib()
    a = torch.ones((8, 8), dtype=torch.float64, device="cuda")
    out = torch.empty((), dtype=torch.float64, device="cuda")
    rc = _noalloc(lib, native, 0, a, None, (1, 1), 1025, out)
    assert rc != 0
    assert "1024" in lib.csd_last_error().decode()
