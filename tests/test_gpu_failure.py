"""Device-side failure reporting without a GPU fault.

Every wait of the streaming engine is bounded (``timeout_ns``); a wait that
runs out stops its CTA after draining the copies it requested and sets the
device error word, which ``csd_error_word`` reports as CSD_ETIMEOUT.  The
failure is made on purpose by the launch option ``withhold_chunk``: one input
chunk of CTA 0 is never requested, so the wait for it cannot succeed (a flag
that nothing sets).  Nothing traps, faults or spins without a bound, and the
context stays usable: the next launch is checked bit for bit.
"""

import numpy as np
import pytest

import stencil_defs as D
from oracle import stencil_oracle as O

pytestmark = pytest.mark.gpu


def _lap7(dtype="float64"):
    import cutile
    from cutile import stencil

    return cutile.compile(stencil(ndim=3, order=2, dtype=dtype)(D.lap7), temporal_blocking=False)


def _field(r, n, seed):
    h = r.halo_widths
    shape = tuple(s + 2 * x for s, x in zip(n, h))
    u = np.zeros(shape)
    inner = tuple(slice(x, s - x) for x, s in zip(h, shape))
    u[inner] = np.random.default_rng(seed).standard_normal(n)
    return u, inner


@pytest.mark.parametrize("loader", [0, 1])
def test_withheld_chunk_times_out_then_next_launch_is_exact(loader):
    import torch

    from cutile.runtime import native

    r = _lap7()
    prog = r.load_module().program()
    u, inner = _field(r, (96, 40, 64), 11)
    a = torch.from_numpy(u).cuda()
    b = torch.zeros_like(a)
    assert native.error_word(reset=True) == 0
    prog.launch((a,), (b,), loader=loader, timeout_ns=2_000_000, withhold_chunk=1)
    rc, word = native.error_status(reset=True)
    assert rc == native.CSD_ETIMEOUT and word == native.CSD_ERR_TIMEOUT
    # the context is intact and the word was cleared
    assert native.error_status(reset=True) == (0, 0)
    c = torch.full_like(a, float("nan"))
    prog.launch((a,), (c,), loader=loader)
    torch.cuda.synchronize()
    want = O.apply_stencil(u, D.lap7, 3, r.halo_widths)
    assert np.array_equal(c.cpu().numpy()[inner], want[inner])
    assert native.error_word(reset=True) == 0


def test_withheld_chunk_in_a_fused_boundary_step():
    """The fused boundary patch runs after the failed wait; it stays in
    bounds and the kernel reports the timeout."""
    import torch

    import cutile
    from cutile import stencil
    from cutile.runtime import native

    r = cutile.compile_fused([stencil(ndim=2)(D.gs_u), stencil(ndim=2)(D.gs_v)],
                             precision="fp64", boundary="periodic")
    h = r.halo_widths
    u, v = D.gray_scott_init(300, seed=2, halo=h)
    t = [torch.from_numpy(x).cuda() for x in (u, v)]
    o = [torch.zeros_like(t[0]) for _ in range(2)]
    prog = r.load_module().program()
    prog.step(t, o, timeout_ns=2_000_000, withhold_chunk=2)
    rc, word = native.error_status(reset=True)
    assert rc == native.CSD_ETIMEOUT and word == native.CSD_ERR_TIMEOUT
    o = [torch.full_like(t[0], float("nan")) for _ in range(2)]
    prog.step(t, o)
    torch.cuda.synchronize()
    want_u = O.stencil_with_boundary([u, v], D.gs_u, 2, h, "periodic")
    want_v = O.stencil_with_boundary([u, v], D.gs_v, 2, h, "periodic")
    inner = tuple(slice(x, s - x) for x, s in zip(h, u.shape))
    assert np.array_equal(o[0].cpu().numpy()[inner], want_u[inner])
    assert np.array_equal(o[1].cpu().numpy()[inner], want_v[inner])
    assert native.error_word(reset=True) == 0


def test_short_wait_bound_on_a_large_launch_is_reported_or_clean():
    """A 1 us bound on every wait of a 256^3 sweep: each wait either sees its
    chunk or gives up; either way the launch ends, the status says which,
    and (the drain keeping no copy in flight past a CTA's exit) the next
    launch with the default bound is exact."""
    import torch

    from cutile.runtime import native

    r = _lap7()
    prog = r.load_module().program()
    u, inner = _field(r, (256, 256, 256), 12)
    a = torch.from_numpy(u).cuda()
    b = torch.zeros_like(a)
    prog.launch((a,), (b,), timeout_ns=1000)
    rc, word = native.error_status(reset=True)
    assert (rc, word) in ((0, 0), (native.CSD_ETIMEOUT, native.CSD_ERR_TIMEOUT))
    c = torch.full_like(a, float("nan"))
    prog.launch((a,), (c,))
    torch.cuda.synchronize()
    want = O.apply_stencil(u, D.lap7, 3, r.halo_widths)
    assert np.array_equal(c.cpu().numpy()[inner], want[inner])
    assert native.error_word(reset=True) == 0
