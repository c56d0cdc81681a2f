"""ctypes binding of libcsd (the C ABI in include/csd.h).

This is the only way Python reaches the GPU: every launch goes through
``csd_launch`` / ``csd_apply_boundary`` on raw device pointers taken from
torch tensors.  There is no CPU fallback -- if the library or a CUDA device
is missing the calls raise.
"""

from __future__ import annotations

import ctypes
import os
import threading
from pathlib import Path

PKG_DIR = Path(__file__).resolve().parent.parent          # .../cutile
ROOT_DIR = PKG_DIR.parent                                  # .../cutile-stencil-dsl_b200
LIB_PATH = PKG_DIR / "_native" / "libcsd.so"
INCLUDE_DIR = ROOT_DIR / "csrc" / "include"
HEADER_NAMES = ("csd/params.h", "csd/ptx.cuh", "csd/engine.cuh")

CSD_LOADER_TMA = 0
CSD_LOADER_LDG = 1
BC_MODES = {"none": 0, "dirichlet": 1, "neumann": 2, "periodic": 3, "reflecting": 4}
DTYPE_CODES = {"float32": 1, "float64": 2}

NVRTC_OPTIONS = (
    "--gpu-architecture=sm_100a",
    "-std=c++17",
    "--fmad=false",
    "-default-device",
    "-DNDEBUG",
    "-lineinfo",
    "--ptxas-options=-v",
)


class CsdError(RuntimeError):
    """A libcsd call failed; the message is ``csd_last_error()`` and ``code``
    the status (``CSD_E*`` in include/csd.h)."""

    def __init__(self, msg: str, code: int = 0):
        super().__init__(msg)
        self.code = code


class Field(ctypes.Structure):
    _fields_ = [("ptr", ctypes.c_void_p), ("ndim", ctypes.c_int), ("dtype", ctypes.c_int),
                ("shape", ctypes.c_int64 * 3), ("strides", ctypes.c_int64 * 3)]


MAX_FIELDS = 8
MAX_SCALARS = 8


class LaunchOpts(ctypes.Structure):
    _fields_ = [("halo", ctypes.c_int * 3), ("zchunk", ctypes.c_int), ("grid", ctypes.c_int),
                ("loader", ctypes.c_int), ("bc_value", ctypes.c_double),
                ("timeout_ns", ctypes.c_uint64), ("scalars", ctypes.c_double * MAX_SCALARS),
                ("dyn", ctypes.c_void_p), ("red", ctypes.c_void_p),
                ("bc_odd", ctypes.c_int * MAX_FIELDS), ("grid_index", ctypes.c_void_p),
                ("withhold_chunk", ctypes.c_int)]


class KernelDesc(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint if n == "magic" else ctypes.c_int) for n in (
        "magic", "ndim", "nin", "nout", "dtype_bytes", "rz", "ry", "rx", "rows", "tile_y",
        "tile_x", "vec", "threads", "stages", "nslot", "halo_chunks", "pad_left", "box_w",
        "box_h", "smem_bytes", "zchunk", "temporal", "bc_mode", "min_blocks", "align",
        "nscalars", "ndyn", "reduce_max", "brick_shift", "brick_tma")]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class GridHead(ctypes.Structure):
    """The leading fields of ``csd_grid`` up to its work split (the TMA maps
    and pointers before them are opaque here)."""

    _fields_ = [("tmap", ctypes.c_ubyte * (128 * 8)), ("inp", ctypes.c_void_p * 8),
                ("out", ctypes.c_void_p * 8), ("dims", ctypes.c_longlong * 3),
                ("pitch_y", ctypes.c_longlong), ("pitch_z", ctypes.c_longlong),
                ("halo", ctypes.c_int * 3), ("interior", ctypes.c_int * 3),
                ("tiles", ctypes.c_int * 3), ("items", ctypes.c_int), ("zchunk", ctypes.c_int),
                ("xbase", ctypes.c_int), ("vec_store", ctypes.c_int), ("ndim", ctypes.c_int),
                ("ecols", ctypes.c_int), ("items_main", ctypes.c_int), ("zchunk_e", ctypes.c_int),
                ("zshift", ctypes.c_int), ("zshift_e", ctypes.c_int)]


_lib = None
_lib_lock = threading.Lock()


def library() -> ctypes.CDLL:
    """Load libcsd.so (built by ``__graft_entry__.build()`` / ``make -C csrc``)."""
    global _lib
    with _lib_lock:
        if _lib is not None:
            return _lib
        path = os.environ.get("CSD_LIBRARY", str(LIB_PATH))
        if not os.path.exists(path):
            raise CsdError(f"libcsd.so not found at {path}; build it with "
                           f"`make -C {ROOT_DIR / 'csrc'}`")
        lib = ctypes.CDLL(path)
        P = ctypes.c_void_p
        cp = ctypes.c_char_p
        lib.csd_version.restype = ctypes.c_int
        lib.csd_last_error.restype = cp
        lib.csd_module_load.argtypes = [cp, ctypes.c_int, ctypes.POINTER(cp), ctypes.POINTER(cp), cp,
                                        cp, ctypes.POINTER(P)]
        lib.csd_compile.argtypes = [cp, ctypes.c_int, ctypes.POINTER(cp), ctypes.POINTER(cp), cp, cp,
                                    ctypes.c_char_p, ctypes.c_size_t, ctypes.c_char_p,
                                    ctypes.c_size_t]
        lib.csd_module_load_image.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(P)]
        lib.csd_plan_items.argtypes = [ctypes.POINTER(KernelDesc), ctypes.c_longlong, ctypes.c_int,
                                       ctypes.c_void_p]
        pi = ctypes.POINTER(ctypes.c_int)
        lib.csd_grid_item_place.argtypes = [ctypes.c_void_p, ctypes.c_int, pi, pi, pi, pi]
        lib.csd_module_unload.argtypes = [P]
        lib.csd_kernel_get.argtypes = [P, cp, ctypes.POINTER(P)]
        lib.csd_kernel_describe.argtypes = [P, ctypes.POINTER(KernelDesc)]
        lib.csd_kernel_resources.argtypes = [P, ctypes.POINTER(ctypes.c_int),
                                             ctypes.POINTER(ctypes.c_int),
                                             ctypes.POINTER(ctypes.c_int)]
        lib.csd_launch.argtypes = [P, ctypes.POINTER(Field), ctypes.c_int, ctypes.POINTER(Field),
                                   ctypes.c_int, ctypes.POINTER(LaunchOpts), P]
        lib.csd_apply_boundary.argtypes = [ctypes.POINTER(Field), ctypes.POINTER(ctypes.c_int),
                                           ctypes.c_int, ctypes.c_double, P]
        lib.csd_error_word.argtypes = [ctypes.POINTER(ctypes.c_int), ctypes.c_int]
        lib.csd_bricked_elems.argtypes = [ctypes.POINTER(ctypes.c_longlong), ctypes.c_int,
                                          ctypes.c_int]
        lib.csd_bricked_elems.restype = ctypes.c_longlong
        lib.csd_to_bricks.argtypes = [ctypes.POINTER(Field), ctypes.c_int, P, P]
        lib.csd_from_bricks.argtypes = [P, ctypes.c_int, ctypes.POINTER(Field), P]
        lib.csd_grid_size.restype = ctypes.c_size_t
        lib.csd_cfl_update.argtypes = [ctypes.c_int, P, P, ctypes.c_double, ctypes.c_double, P, P]
        lib.csd_grid_build.argtypes = [P, ctypes.POINTER(Field), ctypes.c_int, ctypes.POINTER(Field),
                                       ctypes.c_int, ctypes.POINTER(LaunchOpts), P,
                                       ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
        lib.csd_launch_batch.argtypes = [P, P, P, ctypes.c_int, ctypes.c_int,
                                         ctypes.POINTER(LaunchOpts), P]
        lib.csd_reduce.argtypes = [ctypes.POINTER(Field), ctypes.POINTER(Field),
                                   ctypes.POINTER(ctypes.c_int), ctypes.c_int, P, ctypes.c_int, P,
                                   P]
        _lib = lib
        return lib


def check(rc: int) -> None:
    if rc != 0:
        msg = library().csd_last_error().decode(errors="replace")
        raise CsdError(f"libcsd error {rc}: {msg}", rc)


def _headers():
    texts = [(INCLUDE_DIR / n).read_text() for n in HEADER_NAMES]
    arr_t = ctypes.c_char_p * len(texts)
    return (len(texts), arr_t(*[t.encode() for t in texts]),
            arr_t(*[n.encode() for n in HEADER_NAMES]))


def default_cache_dir() -> str:
    env = os.environ.get("CSD_CACHE_DIR")
    if env:
        return env
    d = ROOT_DIR / "_build" / "jit"
    try:
        d.mkdir(parents=True, exist_ok=True)
        return str(d)
    except OSError:
        home = Path.home() / ".cache" / "cutile_b200"
        home.mkdir(parents=True, exist_ok=True)
        return str(home)


def _options(extra=()) -> bytes:
    return "\n".join(list(NVRTC_OPTIONS) + list(extra)).encode()


def compile_source(src: str, extra_options=()) -> tuple[str, str]:
    """NVRTC-compile a module (no GPU needed); returns (cubin path, log)."""
    lib = library()
    n, hdrs, names = _headers()
    path = ctypes.create_string_buffer(4096)
    log = ctypes.create_string_buffer(1 << 16)
    check(lib.csd_compile(src.encode(), n, hdrs, names, _options(extra_options),
                          default_cache_dir().encode(), path, 4096, log, 1 << 16))
    return path.value.decode(), log.value.decode(errors="replace")


# nvcc flags equivalent to NVRTC_OPTIONS for ahead-of-time builds of the same
# source (nvcc has no -default-device; the engine headers mark every device
# function themselves).
NVCC_OPTIONS = (
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-cubin",
    "-std=c++17",
    "-fmad=false",
    "-DNDEBUG",
    "-lineinfo",
    "-Xptxas", "-v",
)


def find_nvcc() -> str:
    """nvcc from ``CUDA_HOME``/``CUDA_PATH``, then ``PATH``, then /usr/local/cuda."""
    import shutil

    for env in ("CUDA_HOME", "CUDA_PATH"):
        root = os.environ.get(env)
        if root and os.path.exists(os.path.join(root, "bin", "nvcc")):
            return os.path.join(root, "bin", "nvcc")
    found = shutil.which("nvcc")
    if found:
        return found
    if os.path.exists("/usr/local/cuda/bin/nvcc"):
        return "/usr/local/cuda/bin/nvcc"
    raise CsdError("nvcc not found (set CUDA_HOME); ahead-of-time builds need the CUDA toolkit")


def aot_compile(cu_path: str, cubin_path: str, nvcc: str | None = None) -> str:
    """Compile a generated module's ``.cu`` to an sm_100a cubin with nvcc (no
    GPU needed); returns nvcc's log (the ptxas ``-v`` resource report)."""
    import subprocess

    cmd = [nvcc or find_nvcc(), *NVCC_OPTIONS, "-I", str(INCLUDE_DIR), cu_path, "-o", cubin_path]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    log = proc.stdout + proc.stderr
    if proc.returncode != 0:
        raise CsdError(f"nvcc failed ({proc.returncode}): {' '.join(cmd)}\n{log}")
    return log


def read_image(path: str, sha256: str | None = None) -> bytes:
    """Bytes of a prebuilt cubin, checked against ``sha256`` when given (a
    cubin rebuilt or replaced after its launcher module was written is
    refused rather than launched with a stale kernel contract)."""
    import hashlib

    if not os.path.exists(path):
        raise CsdError(f"prebuilt cubin {path} is missing")
    with open(path, "rb") as f:
        data = f.read()
    if sha256 is not None and hashlib.sha256(data).hexdigest() != sha256:
        raise CsdError(f"prebuilt cubin {path} does not match its launcher module "
                       f"(sha256 differs): rebuild it with CompileResult.build_aot")
    return data


class NativeModule:
    """A loaded module (per CUDA context): JIT-compiled from ``src`` with
    NVRTC, or, given ``image``, a prebuilt cubin of the same source."""

    def __init__(self, src: str, extra_options=(), image: bytes | None = None):
        lib = library()
        handle = ctypes.c_void_p()
        if image is not None:
            buf = ctypes.create_string_buffer(image, len(image))
            check(lib.csd_module_load_image(buf, len(image), ctypes.byref(handle)))
        else:
            n, hdrs, names = _headers()
            check(lib.csd_module_load(src.encode(), n, hdrs, names, _options(extra_options),
                                      default_cache_dir().encode(), ctypes.byref(handle)))
        self.handle = handle
        self._kernels: dict[str, NativeKernel] = {}

    def kernel(self, name: str) -> "NativeKernel":
        k = self._kernels.get(name)
        if k is None:
            handle = ctypes.c_void_p()
            check(library().csd_kernel_get(self.handle, name.encode(), ctypes.byref(handle)))
            k = NativeKernel(name, handle)
            self._kernels[name] = k
        return k


class NativeKernel:
    def __init__(self, name: str, handle: ctypes.c_void_p):
        self.name = name
        self.handle = handle
        d = KernelDesc()
        check(library().csd_kernel_describe(handle, ctypes.byref(d)))
        self.desc = d.as_dict()

    def resources(self) -> dict:
        regs, local, blocks = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(library().csd_kernel_resources(self.handle, ctypes.byref(regs), ctypes.byref(local),
                                             ctypes.byref(blocks)))
        return {"registers": regs.value, "local_bytes": local.value,
                "blocks_per_sm": blocks.value}


def field_of(t, pitched: bool = False) -> Field:
    """csd_field for a torch tensor (CUDA, float32/float64, C-contiguous; with
    ``pitched`` also a row-pitched view: unit innermost stride, padded rows)."""
    import torch

    if not isinstance(t, torch.Tensor):
        raise TypeError(f"expected a torch.Tensor, got {type(t).__name__}")
    if not t.is_cuda:
        raise ValueError("stencil fields must be CUDA tensors")
    if t.dtype == torch.float64:
        code = 2
    elif t.dtype == torch.float32:
        code = 1
    else:
        raise TypeError(f"unsupported dtype {t.dtype}")
    if t.dim() < 1 or t.dim() > 3:
        raise ValueError("fields must be 1-, 2- or 3-D")
    if not t.is_contiguous():
        if not pitched or t.stride(-1) != 1:
            raise ValueError("fields must be C-contiguous")
    f = Field()
    f.ptr = t.data_ptr()
    f.ndim = t.dim()
    f.dtype = code
    for i in range(t.dim()):
        f.shape[i] = t.shape[i]
        f.strides[i] = t.stride(i)
    return f


def stream_handle(stream) -> int | None:
    import torch

    if stream is None:
        return torch.cuda.current_stream().cuda_stream
    if isinstance(stream, int):
        return stream
    return getattr(stream, "cuda_stream", None) or getattr(stream, "ptr", None)


def make_opts(halo, *, zchunk: int = 0, grid: int = 0, loader: int = -1, bc_value: float = 0.0,
              timeout_ns: int = 0, scalars=(), dyn=None, red=None, bc_odd=(),
              withhold_chunk: int = 0) -> LaunchOpts:
    o = LaunchOpts()
    o.withhold_chunk = withhold_chunk
    for i, h in enumerate(halo):
        o.halo[i] = int(h)
    o.zchunk = zchunk
    o.grid = grid
    o.loader = loader
    o.bc_value = bc_value
    o.timeout_ns = timeout_ns
    if len(scalars) > MAX_SCALARS:
        raise ValueError(f"at most {MAX_SCALARS} scalar parameters")
    for i, v in enumerate(scalars):
        o.scalars[i] = float(v)
    o.dyn = None if dyn is None else (dyn if isinstance(dyn, int) else dyn.data_ptr())
    o.red = None if red is None else (red if isinstance(red, int) else red.data_ptr())
    for i, m in enumerate(bc_odd):
        o.bc_odd[i] = int(m)
    return o


def launch(kernel: NativeKernel, inputs, outputs, halo, stream=None, **kw) -> None:
    lib = library()
    fin = (Field * len(inputs))(*[field_of(t, True) for t in inputs])
    fout = (Field * max(1, len(outputs)))(*[field_of(t, True) for t in outputs])
    o = make_opts(halo, **kw)
    check(lib.csd_launch(kernel.handle, fin, len(inputs), fout, len(outputs), ctypes.byref(o),
                         ctypes.c_void_p(stream_handle(stream))))


def grid_size() -> int:
    return int(library().csd_grid_size())


def plan_items(desc: dict, tiles_x: int, tiles_y: int, nz: int, slots: int,
               zchunk: int = 0) -> tuple[dict, list]:
    """The work split ``csd_launch`` uses for a grid of ``tiles_x x tiles_y``
    columns and ``nz`` interior rows on ``slots`` resident CTAs (host only):
    the split fields and every item's ``(tx, ty, z0, nrows)``."""
    lib = library()
    kd = KernelDesc(**{k: v for k, v in desc.items() if k in dict(KernelDesc._fields_)})
    buf = ctypes.create_string_buffer(grid_size())
    head = GridHead.from_buffer(buf)
    head.tiles[0], head.tiles[1] = tiles_x, tiles_y
    head.interior[0] = nz
    check(lib.csd_plan_items(ctypes.byref(kd), slots, zchunk, ctypes.addressof(buf)))
    split = {k: getattr(head, k) for k in ("items", "zchunk", "ecols", "items_main", "zchunk_e",
                                           "zshift", "zshift_e")}
    split["tiles_z"] = head.tiles[2]
    out = []
    v = [ctypes.c_int() for _ in range(4)]
    for i in range(head.items):
        check(lib.csd_grid_item_place(ctypes.addressof(buf), i, *[ctypes.byref(x) for x in v]))
        out.append(tuple(x.value for x in v))
    return split, out


def grid_build(kernel: NativeKernel, inputs, outputs, halo, dest, **kw) -> tuple[int, int]:
    """Write the descriptor of one batched grid into host buffer ``dest``
    (a ctypes buffer of ``grid_size()`` bytes); returns (work items, loader)."""
    lib = library()
    fin = (Field * len(inputs))(*[field_of(t, True) for t in inputs])
    fout = (Field * max(1, len(outputs)))(*[field_of(t, True) for t in outputs])
    o = make_opts(halo, **kw)
    items = ctypes.c_int()
    loader = ctypes.c_int()
    check(lib.csd_grid_build(kernel.handle, fin, len(inputs), fout, len(outputs), ctypes.byref(o),
                             ctypes.cast(dest, ctypes.c_void_p), ctypes.byref(items),
                             ctypes.byref(loader)))
    return items.value, loader.value


def launch_batch(kernel: NativeKernel, grids_ptr: int, item_start_ptr: int, ngrids: int,
                 total_items: int, stream=None, grid: int = 0, timeout_ns: int = 0,
                 loader: int = 0, grid_index_ptr: int | None = None) -> None:
    lib = library()
    o = LaunchOpts()
    o.grid = grid
    o.loader = loader
    o.grid_index = grid_index_ptr
    o.timeout_ns = timeout_ns
    check(lib.csd_launch_batch(kernel.handle, ctypes.c_void_p(grids_ptr),
                               ctypes.c_void_p(item_start_ptr), ngrids, total_items,
                               ctypes.byref(o), ctypes.c_void_p(stream_handle(stream))))


def apply_boundary(t, halo, bc: str, value: float = 0.0, stream=None) -> None:
    lib = library()
    f = field_of(t)
    h = (ctypes.c_int * 3)(*([int(x) for x in halo] + [0] * (3 - len(halo))))
    check(lib.csd_apply_boundary(ctypes.byref(f), h, BC_MODES[bc], float(value),
                                 ctypes.c_void_p(stream_handle(stream))))


def cfl_update(smax, scale, cfl: float, dt, dt_max: float = 1e30, stream=None) -> None:
    """dt = min(cfl * scale / smax, dt_max) per grid, then smax = 0 (device arrays)."""
    check(library().csd_cfl_update(int(smax.numel()), ctypes.c_void_p(smax.data_ptr()),
                                   ctypes.c_void_p(scale.data_ptr()), float(cfl), float(dt_max),
                                   ctypes.c_void_p(dt.data_ptr()),
                                   ctypes.c_void_p(stream_handle(stream))))


def bricked_shape(shape, brick: int) -> tuple:
    """Shape of the bricked form of an array: brick-grid extents, then one
    brick (the reference's to_bricks layout)."""
    nb = tuple(-(-int(n) // brick) for n in shape)
    return nb + (brick,) * len(shape)


def _bricked_elems(shape, brick: int) -> int:
    return int(library().csd_bricked_elems((ctypes.c_longlong * len(shape))(*shape), len(shape),
                                           int(brick)))


def to_bricks(flat, brick: int, stream=None):
    """Device bricked copy of the C-contiguous device array ``flat``."""
    import torch

    out = torch.empty(bricked_shape(flat.shape, brick), dtype=flat.dtype, device=flat.device)
    f = field_of(flat)
    check(library().csd_to_bricks(ctypes.byref(f), int(brick), ctypes.c_void_p(out.data_ptr()),
                                  ctypes.c_void_p(stream_handle(stream))))
    return out


def from_bricks(bricked, shape, brick: int, out=None, stream=None):
    """Flat (C-contiguous) array of ``shape`` from its bricked form."""
    import torch

    shape = tuple(int(n) for n in shape)
    if bricked.numel() < _bricked_elems(shape, brick):
        raise ValueError("bricked array is smaller than the bricked form of the shape")
    if not bricked.is_contiguous():
        raise ValueError("bricked array must be contiguous")
    if out is None:
        out = torch.empty(shape, dtype=bricked.dtype, device=bricked.device)
    f = field_of(out)
    check(library().csd_from_bricks(ctypes.c_void_p(bricked.data_ptr()), int(brick),
                                    ctypes.byref(f), ctypes.c_void_p(stream_handle(stream))))
    return out


def bricked_field(t, shape, brick: int) -> Field:
    """csd_field of a bricked device array holding a ``shape`` array."""
    import torch

    shape = tuple(int(n) for n in shape)
    if not isinstance(t, torch.Tensor) or not t.is_cuda or not t.is_contiguous():
        raise ValueError("bricked fields must be contiguous CUDA tensors")
    need = _bricked_elems(shape, brick)
    if t.numel() < need:
        raise ValueError(f"bricked field holds {t.numel()} elements, the bricked form of "
                         f"{shape} needs {need}")
    f = Field()
    f.ptr = t.data_ptr()
    f.ndim = len(shape)
    f.dtype = 2 if t.dtype == torch.float64 else 1 if t.dtype == torch.float32 else 0
    if f.dtype == 0:
        raise TypeError(f"unsupported dtype {t.dtype}")
    stride = 1
    for i in reversed(range(len(shape))):
        f.shape[i] = shape[i]
        f.strides[i] = stride
        stride *= shape[i]
    return f


def launch_fields(kernel: NativeKernel, fin, fout, halo, stream=None, **kw) -> None:
    """csd_launch on prepared csd_field lists."""
    lib = library()
    a = (Field * len(fin))(*fin)
    b = (Field * max(1, len(fout)))(*fout)
    o = make_opts(halo, **kw)
    check(lib.csd_launch(kernel.handle, a, len(fin), b, len(fout), ctypes.byref(o),
                         ctypes.c_void_p(stream_handle(stream))))


CSD_ETIMEOUT = 5
CSD_ERR_TIMEOUT = 0x7001


def error_status(reset: bool = True) -> tuple[int, int]:
    """``(status, word)`` of ``csd_error_word``: status CSD_OK for a clear
    word, CSD_ETIMEOUT when a kernel's wait for input ran out; other
    statuses raise."""
    v = ctypes.c_int()
    rc = library().csd_error_word(ctypes.byref(v), 1 if reset else 0)
    if rc not in (0, CSD_ETIMEOUT):
        check(rc)
    return rc, v.value


def error_word(reset: bool = True) -> int:
    """The device error word (0 = no kernel reported a failure)."""
    return error_status(reset)[1]


__all__ = ["library", "check", "compile_source", "NativeModule", "NativeKernel", "launch",
           "apply_boundary", "error_word", "error_status", "CSD_ETIMEOUT", "CSD_ERR_TIMEOUT", "CsdError", "field_of", "default_cache_dir",
           "make_opts", "grid_size", "grid_build", "launch_batch", "bricked_shape",
           "to_bricks", "from_bricks", "bricked_field", "launch_fields",
           "GridHead", "plan_items", "NVCC_OPTIONS", "find_nvcc", "aot_compile", "read_image", "CSD_LOADER_TMA", "CSD_LOADER_LDG", "BC_MODES"]
