"""Ahead-of-time builds without a GPU: nvcc compiles every kind of generated
module (single, fused periodic, bricked, reduction) from the emitted ``.cu``,
the launcher module written beside the cubin exposes the same entry points as
the JIT module, and stale or foreign images are refused before any launch."""

import ctypes
import os
import shutil

import pytest

import stencil_defs as D

pytestmark = pytest.mark.skipif(shutil.which("nvcc") is None and not os.path.exists(
    "/usr/local/cuda/bin/nvcc"), reason="needs the CUDA toolkit's nvcc")


def _results():
    import cutile
    from cutile import stencil

    return {
        "lap7": cutile.compile(stencil(ndim=3)(D.lap7), temporal_blocking=False),
        "gs_kahan": cutile.compile_fused([stencil(ndim=2)(D.gs_u), stencil(ndim=2)(D.gs_v)],
                                         precision="fp32_kahan", boundary="periodic"),
        "lap7_bricked": cutile.compile(stencil(ndim=3)(D.lap7), temporal_blocking=False,
                                       layout="bricked", brick_size=8),
        "sw_speed": cutile.compile(stencil(ndim=2, dtype="float32")(D.sw_speed), reduce="max"),
    }


@pytest.fixture(scope="module")
def builds(tmp_path_factory):
    out = {}
    for key, r in _results().items():
        d = tmp_path_factory.mktemp(key)
        out[key] = (r, r.build_aot(str(d)))
    return out


def _entry_points(module):
    return sorted(n for n in dir(module) if n.split("_")[0] in
                  ("launch", "step", "apply", "reduce", "to", "from"))


@pytest.mark.parametrize("key", ["lap7", "gs_kahan", "lap7_bricked", "sw_speed"])
def test_aot_build_writes_cubin_and_launcher(builds, key):
    import cutile

    r, b = builds[key]
    for p in (b.cu, b.cubin, b.module):
        assert os.path.getsize(p) > 0
    with open(b.cubin, "rb") as f:
        assert f.read(4) == b"\x7fELF"
    with open(b.cu) as f:
        assert f.read() == r.cuda_source
    assert b.resources and all(v is not None and not v.spills for v in b.resources.values())
    aot = cutile.load_aot(b.module)
    assert aot.CUBIN == os.path.abspath(b.cubin)
    assert len(aot.CUBIN_SHA256) == 64
    assert _entry_points(aot) == _entry_points(r.load_module())
    assert aot.program().cubin == aot.CUBIN
    # the JIT module keeps its empty slots
    assert r.load_module().CUBIN is None and r.load_module().program().cubin is None


def test_aot_entries_match_jit_kernel_names(builds):
    r, b = builds["gs_kahan"]
    names = set(b.resources)
    for kern in r.load_module().program().spec["kernels"].values():
        assert {f"{kern}_tma", f"{kern}_ldg"} <= names


def test_stale_cubin_is_refused(builds, tmp_path):
    from cutile.runtime import native

    _, b = builds["lap7"]
    import cutile

    aot = cutile.load_aot(b.module)
    assert native.read_image(aot.CUBIN, aot.CUBIN_SHA256)[:4] == b"\x7fELF"
    copy = tmp_path / "lap7.cubin"
    data = bytearray(open(b.cubin, "rb").read())
    data[-1] ^= 0xFF
    copy.write_bytes(bytes(data))
    with pytest.raises(native.CsdError, match="does not match"):
        native.read_image(str(copy), aot.CUBIN_SHA256)
    with pytest.raises(native.CsdError, match="missing"):
        native.read_image(str(tmp_path / "absent.cubin"), None)


def test_load_image_refuses_non_cubin_bytes():
    from cutile.runtime import native

    lib = native.library()
    h = ctypes.c_void_p()
    junk = b"// not a cubin" + b"\0" * 80
    rc = lib.csd_module_load_image(junk, len(junk), ctypes.byref(h))
    assert rc != 0 and b"not a cubin" in lib.csd_last_error()
    assert lib.csd_module_load_image(None, 0, ctypes.byref(h)) != 0
