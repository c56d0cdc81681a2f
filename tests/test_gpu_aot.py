"""Ahead-of-time modules on the GPU: the nvcc-built cubin loaded through
``csd_module_load_image`` gives the same bits as the NVRTC module and as the
oracle (7-point sweep, fused periodic Kahan step, max reduction)."""

import numpy as np
import pytest

import stencil_defs as D
from oracle import stencil_oracle as O

pytestmark = pytest.mark.gpu


def test_aot_lap7_matches_jit_and_oracle(tmp_path):
    import torch

    import cutile
    from cutile import stencil

    r = cutile.compile(stencil(ndim=3)(D.lap7), temporal_blocking=False, align_halo=False)
    aot = cutile.load_aot(r.build_aot(str(tmp_path)).module)
    u = np.random.default_rng(11).standard_normal((40, 37, 70))
    tin = torch.from_numpy(u).cuda()
    outs = [torch.full_like(tin, float("nan")) for _ in range(2)]
    r.load_module().launch_lap7(tin, outs[0])
    aot.launch_lap7(tin, outs[1])
    torch.cuda.synchronize()
    assert aot.program()._module() is not r.load_module().program()._module()
    # halos stay NaN in both (only interiors are written)
    assert torch.equal(outs[0].nan_to_num(7.0), outs[1].nan_to_num(7.0))
    want = O.apply_stencil(u, D.lap7, 3, (1, 1, 1))
    got = outs[1].cpu().numpy()
    assert np.array_equal(got[1:-1, 1:-1, 1:-1], want[1:-1, 1:-1, 1:-1])


def test_aot_fused_kahan_step_matches_jit(tmp_path):
    import torch

    import cutile
    from cutile import stencil

    r = cutile.compile_fused([stencil(ndim=2)(D.gs_u), stencil(ndim=2)(D.gs_v)],
                             precision="fp32_kahan", boundary="periodic")
    aot = cutile.load_aot(r.build_aot(str(tmp_path)).module)
    h = r.halo_widths
    u, v = D.gray_scott_init(130, seed=12, halo=h, dtype="float32")
    rng = np.random.default_rng(13)
    cu = (rng.standard_normal(u.shape) * 1e-8).astype(np.float32)
    cv = (rng.standard_normal(u.shape) * 1e-8).astype(np.float32)
    t = [torch.from_numpy(a).cuda() for a in (u, v, cu, cv)]
    res = []
    for mod in (r.load_module(), aot):
        outs = [torch.zeros_like(t[0]) for _ in range(4)]
        mod.step_gs_u_gs_v(*t, *outs)
        res.append(outs)
    torch.cuda.synchronize()
    for a, b in zip(*res):
        assert torch.equal(a, b)
    want = O.fused_kahan_step({"u": u, "v": v}, {"u": cu, "v": cv},
                              {"u": D.gs_u_incr, "v": D.gs_v_incr}, 2, h, boundary="periodic")
    inner = tuple(slice(x, s - x) for x, s in zip(h, u.shape))
    assert np.array_equal(res[1][0].cpu().numpy()[inner], want["u"][0][inner])
    assert np.array_equal(res[1][3].cpu().numpy()[inner], want["v"][1][inner])


def test_aot_reduction_matches_jit(tmp_path):
    import torch

    import cutile
    from cutile import stencil

    r = cutile.compile(stencil(ndim=2, dtype="float32")(D.sw_speed), reduce="max",
                       align_halo=False)
    aot = cutile.load_aot(r.build_aot(str(tmp_path)).module)
    halo = r.halo_widths
    rng = np.random.default_rng(14)
    shape = tuple(90 + 2 * x for x in halo)
    h = (1.0 + 0.1 * rng.random(shape)).astype(np.float32)
    hu = (0.05 * rng.standard_normal(shape)).astype(np.float32)
    hv = (0.05 * rng.standard_normal(shape)).astype(np.float32)
    t = [torch.from_numpy(a).cuda() for a in (h, hu, hv)]
    jit = r.load_module().reduce_sw_speed(*t).item()
    got = aot.reduce_sw_speed(*t).item()
    assert got == jit and got > 0.0
