"""The wide and very wide tier on the engine: 27- and 125-point boxes (FP64
and FP32) and an eight-in / five-out compressible-flow fused update, bit-exact
against the NumPy oracle."""

import numpy as np
import pytest

import wide_defs as W
from oracle import stencil_oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("radius", [1, 2])
@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_box_bit_exact(radius, dtype, tmp_path):
    import torch

    from cutile import compile as stencil_compile

    fn = W.load_box(f"box{radius}_{dtype[-2:]}", radius, dtype=dtype, directory=str(tmp_path))
    raw = W.load_box(f"raw{radius}_{dtype[-2:]}", radius, decorated=False, directory=str(tmp_path))
    r = stencil_compile(fn, temporal_blocking=False)
    h = r.halo_widths
    dom = (20, 22, 40)
    u = np.zeros(tuple(n + 2 * x for n, x in zip(dom, h)), dtype=dtype)
    u[tuple(slice(x, -x) for x in h)] = np.random.default_rng(radius).standard_normal(dom)
    a = torch.from_numpy(u).cuda()
    b = torch.zeros_like(a)
    getattr(r.load_module(), f"launch_{r.name}")(a, b)
    want = O.apply_stencil(u, raw, 3, h)
    inner = tuple(slice(x, -x) for x in h)
    assert np.array_equal(b.cpu().numpy()[inner], want[inner])


def test_cns_fused_eight_in_five_out_bit_exact():
    import torch

    from cutile import compile_fused, stencil

    r = compile_fused([stencil(ndim=3)(f) for f in W.CNS_MEMBERS], temporal_steps=1)
    h = r.halo_widths
    fields = W.cns_init(18, halo=h)
    ins = [torch.from_numpy(fields[n]).cuda() for n in r.inputs]
    outs = [torch.zeros_like(ins[0]) for _ in W.CNS_MEMBERS]
    getattr(r.load_module(), f"launch_{r.name}")(*ins, *outs)
    want = O.fused_apply({n: fields[n] for n in r.inputs}, W.CNS_MEMBERS, 3, h)
    inner = tuple(slice(x, -x) for x in h)
    for k, (got, exp) in enumerate(zip(outs, want)):
        assert np.array_equal(got.cpu().numpy()[inner], exp[inner]), W.CNS_MEMBERS[k].__name__
