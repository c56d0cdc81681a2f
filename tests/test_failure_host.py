"""Failure paths that need no GPU: NVRTC errors, damaged cache entries, and
the C/ctypes layout of the launch options that carry the device-wait bound
and the failure-test hook."""

import ctypes
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

GOOD_SRC = 'extern "C" __global__ void k(float* p) { p[threadIdx.x] = 1.0f; }\n'


def test_nvrtc_error_reports_compile_status_and_log(tmp_path, monkeypatch):
    from cutile.runtime import native

    monkeypatch.setenv("CSD_CACHE_DIR", str(tmp_path))
    with pytest.raises(native.CsdError) as e:
        native.compile_source("this is not C++ at all;\n")
    assert e.value.code == 3  # CSD_ECOMPILE
    msg = str(e.value)
    assert "NVRTC compilation failed" in msg and "error" in msg.lower()
    # nothing was cached for the failed source
    assert not [p for p in os.listdir(tmp_path) if p.endswith(".cubin")]


def test_generated_module_with_a_broken_body_fails_to_compile(tmp_path, monkeypatch):
    """A module whose functor does not compile fails with the compile status,
    not later at launch."""
    import cutile
    import stencil_defs as D
    from cutile import stencil
    from cutile.runtime import native

    monkeypatch.setenv("CSD_CACHE_DIR", str(tmp_path))
    r = cutile.compile(stencil(ndim=2, order=2)(D.heat2d), temporal_blocking=False)
    bad = r.cuda_source.replace("__dadd_rn(", "__no_such_intrinsic(", 1)
    assert bad != r.cuda_source
    with pytest.raises(native.CsdError) as e:
        native.compile_source(bad)
    assert e.value.code == 3 and "__no_such_intrinsic" in str(e.value)


@pytest.mark.parametrize("damage", ["truncate", "flip", "no_record", "garbage"])
def test_damaged_cache_entry_is_rebuilt(tmp_path, monkeypatch, damage):
    from cutile.runtime import native

    monkeypatch.setenv("CSD_CACHE_DIR", str(tmp_path))
    path, _ = native.compile_source(GOOD_SRC)
    good = open(path, "rb").read()
    assert good[:4] == b"\x7fELF"
    sum_path = path[:-len(".cubin")] + ".sum"
    assert os.path.exists(sum_path)
    if damage == "truncate":
        open(path, "wb").write(good[:100])
    elif damage == "flip":
        data = bytearray(good)
        data[len(data) // 2] ^= 0x5A
        open(path, "wb").write(bytes(data))
    elif damage == "no_record":
        os.unlink(sum_path)
    else:
        open(path, "wb").write(b"// not a cubin\n" * 10)
    path2, _ = native.compile_source(GOOD_SRC)
    assert path2 == path
    assert open(path, "rb").read() == good
    assert os.path.exists(sum_path)


def test_cache_hit_returns_the_same_image(tmp_path, monkeypatch):
    from cutile.runtime import native

    monkeypatch.setenv("CSD_CACHE_DIR", str(tmp_path))
    p1, _ = native.compile_source(GOOD_SRC)
    t1 = os.path.getmtime(p1)
    p2, _ = native.compile_source(GOOD_SRC)
    assert p1 == p2 and os.path.getmtime(p2) == t1


def test_launch_opts_layout_matches_the_c_header(tmp_path):
    """ctypes' LaunchOpts has the size and field offsets of csd_launch_opts
    (compiled from include/csd.h with the host compiler)."""
    from cutile.runtime import native

    fields = [n for n, _ in native.LaunchOpts._fields_]
    prog = tmp_path / "layout.c"
    prog.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "csd.h"\nint main(void){\n'
        '  printf("%zu\\n", sizeof(csd_launch_opts));\n'
        + "".join(f'  printf("%zu\\n", offsetof(csd_launch_opts, {n}));\n' for n in fields)
        + "  return 0;\n}\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(prog), "-o", str(exe)],
                   check=True)
    vals = [int(x) for x in subprocess.run([str(exe)], check=True, capture_output=True,
                                           text=True).stdout.split()]
    assert vals[0] == ctypes.sizeof(native.LaunchOpts)
    for n, off in zip(fields, vals[1:]):
        assert getattr(native.LaunchOpts, n).offset == off, n


def test_make_opts_carries_timeout_and_hook():
    from cutile.runtime import native

    o = native.make_opts((1, 1, 16), timeout_ns=5_000_000, withhold_chunk=2)
    assert o.timeout_ns == 5_000_000 and o.withhold_chunk == 2
    assert native.make_opts((1, 1, 1)).withhold_chunk == 0
