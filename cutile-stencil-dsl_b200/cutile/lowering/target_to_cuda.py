"""Dialect 3 -> CUDA C++ for the sm_100a stencil engine.

Replaces the reference's Dialect 3 -> cuTile Python emitter
(cutile/lowering/target_to_python.py:464-526).  For each ``cutile.kernel``:

* the body becomes a device functor ``Body_<name>::compute``: for every
  distinct ``(field, z offset, y offset)`` it loads one row *strip* from the
  staged tile (16-byte shared-memory vector loads), then evaluates the
  thread's ``VEC`` points with one statement per SSA op of the DSL body, in
  DSL order, using round-to-nearest intrinsics (``__dadd_rn`` ...) so no
  multiply-add contraction or re-association can change a bit; a value that
  one point needs at an X shift of another point's value (a face flux, a
  neighbour's velocity) is computed once (``_ShiftClasses``);
* two kernels instantiate the engine template around it: ``<name>_tma``
  (TMA tile copies) and ``<name>_ldg`` (cp.async copies, for arrays whose
  row pitch is not 16-byte aligned);
* ``<name>_desc`` exports the compile-time configuration to the host runtime.

Constants are emitted as exact hexadecimal float literals (the reference
needed a device array of float64 constants because cuTile rounds Python
scalars to float32, target_to_python.py:170-180, 429-451).
"""

from __future__ import annotations

import math
import struct

from cutile.dialects.cutile_target import KernelOp
from cutile.ir.core import ModuleOp

BC_CODES = {"none": "CSD_BC_NONE", "dirichlet": "CSD_BC_DIRICHLET", "neumann": "CSD_BC_NEUMANN",
            "periodic": "CSD_BC_PERIODIC", "reflecting": "CSD_BC_REFLECTING"}

_CTYPE = {"f32": "float", "f64": "double", "w": "double", "b": "bool", "wb": "bool"}


def hex_literal(value: float, ctype: str = "double") -> str:
    """Exact C literal for *value* in *ctype* (``float`` literals are the
    float32 rounding of the double, as NumPy rounds a Python float)."""
    if ctype == "float":
        v32 = struct.unpack("<f", struct.pack("<f", value))[0]
        if math.isfinite(v32):
            return f"{float(v32).hex()}f"
        bits = struct.unpack("<I", struct.pack("<f", v32))[0]
        return f"__int_as_float(0x{bits:08x})"
    if math.isfinite(value):
        return float(value).hex()
    bits = struct.unpack("<Q", struct.pack("<d", value))[0]
    return f"__longlong_as_double(0x{bits:016x}LL)"


def _internal_offsets(ndim: int, offsets) -> tuple[int, int, int]:
    if ndim == 3:
        return tuple(offsets)
    if ndim == 2:
        return (offsets[0], 0, offsets[1])
    return (0, 0, offsets[0])


def _parse_line(line: str):
    """``v3 = addf v1, a0 : f64`` -> ("v3", "addf", ["v1", "a0"], "f64", extra)."""
    if line.startswith("return "):
        parts = line.split()
        idx = int(parts[2][1:]) if len(parts) > 2 else None
        return ("", "return", [parts[1]], "", idx)
    lhs, rhs = line.split(" = ", 1)
    body, typ = rhs.rsplit(" : ", 1)
    parts = body.split(" ", 1)
    op = parts[0]
    rest = parts[1] if len(parts) > 1 else ""
    extra = None
    if op == "const":
        return (lhs, op, [], typ, float(rest))
    if "@" in rest:
        rest, extra = rest.split(" @")
    args = [a.strip() for a in rest.split(",")] if rest else []
    return (lhs, op, args, typ, extra)


class _BodyEmitter:
    def __init__(self, prefix: str):
        self.prefix = prefix
        self.types: dict[str, str] = {}
        self.consts: dict[str, float] = {}
        self.lines: list[str] = []

    def name(self, v: str) -> str:
        # accesses a<j>, scalars s<k> and device scalars d<k> are shared names
        return v if v[0] in "asd" else f"{self.prefix}{v}"

    def conv(self, v: str, to: str) -> str:
        """Operand *v* as C type of numpy kind *to* (f32/f64)."""
        t = self.types[v]
        if t == "w" and v in self.consts:
            return hex_literal(self.consts[v], "float" if to == "f32" else "double")
        n = self.name(v)
        if t in ("w", "f64") and to == "f32":
            return f"(float){n}"
        if t == "f32" and to == "f64":
            return f"(double){n}"
        return n

    def emit(self, lines: list[str], access_types: dict[str, str]) -> str:
        self.types.update(access_types)
        self.returns = []
        for raw in lines:
            lhs, op, args, typ, extra = _parse_line(raw)
            if op == "return":
                self.returns.append((args[0], extra))
                continue
            self.types[lhs] = typ
            if op == "const":
                self.consts[lhs] = extra
                continue
            ct = _CTYPE[typ]
            tgt = "f64" if typ in ("w", "f64") else typ
            sfx = "f" if tgt == "f32" else "d"
            if op == "divf":
                expr = f"csd::div_rn({self.conv(args[0], tgt)}, {self.conv(args[1], tgt)})"
            elif op in ("addf", "subf", "mulf"):
                fn = {"addf": "add", "subf": "sub", "mulf": "mul"}[op]
                expr = f"__{sfx}{fn}_rn({self.conv(args[0], tgt)}, {self.conv(args[1], tgt)})"
            elif op == "cast":
                expr = self.conv(args[0], tgt)
            elif op == "negf":
                expr = f"-({self.conv(args[0], tgt)})"
            elif op == "absf":
                expr = f"{'fabsf' if tgt == 'f32' else 'fabs'}({self.conv(args[0], tgt)})"
            elif op == "sqrt":
                expr = f"csd::sqrt_rn({self.conv(args[0], tgt)})"
            elif op in ("maxf", "minf"):
                fn = "csd_max" if op == "maxf" else "csd_min"
                expr = f"{fn}({self.conv(args[0], tgt)}, {self.conv(args[1], tgt)})"
            elif op.startswith("cmp."):
                pred = op.split(".", 1)[1]
                sym = {"oeq": "==", "ogt": ">", "oge": ">=", "olt": "<", "ole": "<=",
                       "one": "!=", "une": "!="}[pred]
                cmp_t = extra or "f64"
                a, b = self.conv(args[0], cmp_t), self.conv(args[1], cmp_t)
                if pred == "one":  # ordered not-equal: false on NaN
                    expr = f"(({a}) < ({b}) || ({a}) > ({b}))"
                else:
                    expr = f"(({a}) {sym} ({b}))"
            elif op == "select":
                c = self.name(args[0]) if self.types[args[0]] in ("b", "wb") else self.conv(args[0], "f64")
                expr = f"({c} ? {self.conv(args[1], tgt)} : {self.conv(args[2], tgt)})"
            else:
                raise ValueError(f"unknown SSA op {op!r}")
            self.lines.append(f"const {ct} {self.name(lhs)} = {expr};")
        return self.returns

    def result_as(self, v: str, store_t: str) -> str:
        t = self.types[v]
        if t in ("b", "wb"):
            return f"({store_t})({self.name(v)} ? 1 : 0)"
        if t == "w" and v in self.consts:
            return hex_literal(self.consts[v], store_t)
        return f"({store_t}){self.name(v)}"


def _pos_name(cid: int, pos) -> str:
    if pos is None:
        return f"c{cid}"
    return "c%d_%s" % (cid, "_".join(("m%d" % -p) if p < 0 else str(p) for p in pos))


class _ShiftClasses:
    """Values of the body up to a shift along Y and X.

    A value's class is its expression tree with every access's Y and X
    offsets made relative to the smallest Y and the smallest X offset in the
    tree (``(my, mx)``); the value at the thread's point ``(j, k)`` (row j of
    the unit, point k of the row) is then its class at absolute position
    ``(j + my, k + mx)``.  Two values of one class at one position are the
    same expression of the same staged cells, so a thread computes each
    (class, position) once: a flux at the face between points k and k+1
    serves as the east flux of k and the west flux of k+1, and a strip of
    row y + 1 read at offset dy serves row y at offset dy + 1.  Every value is
    still computed by the same round-to-nearest operations on the same
    operands, so results are bit-identical to evaluating each point alone.
    """

    def __init__(self):
        self.ids: dict = {}

    def intern(self, key) -> int:
        cid = self.ids.get(key)
        if cid is None:
            cid = self.ids[key] = len(self.ids)
        return cid


def emit_body(kernel: KernelOp) -> str:
    """Device functor for the kernel's stencil body(ies)."""
    name = kernel.kernel_name.data
    ndim = kernel.ndim.data
    dtype = kernel.dtype.data
    field_t = "f32" if dtype in ("float32", "fp32") else "f64"
    store_t = "float" if field_t == "f32" else "double"
    params = engine_params(kernel)
    vec = params["VEC"]   # X points per unit (engine Cfg::VEC; 16 bytes unless widened)
    rpy = params["RPY"]   # Y rows per thread (engine Cfg::RPY)
    accesses = [tuple(a.data for a in acc) for acc in kernel.accesses.data]
    acc_info = [_internal_offsets(ndim, offs) + (f,) for f, *offs in accesses]  # (dz, dy, dx, f)
    # strip groups: (field, dz, dy of the unit's row 0) -> X range, over all rows
    groups: dict[tuple, list] = {}
    for dz, dy, dx, f in acc_info:
        for j in range(rpy):
            groups.setdefault((f, dz, dy + j), []).append(dx)
    gkeys = list(groups)
    gindex = {key: gi for gi, key in enumerate(gkeys)}
    # small bodies let the engine unroll a stage's units (their coordinates
    # fold into per-thread constants); wide ones would keep several units'
    # strips live at once and spill
    body_lines = sum(len(prog.data) for prog in kernel.ssa_body.data)
    unroll = 4 if (len(gkeys) <= 8 and rpy == 1 and body_lines <= 48) else 0
    out = [f"struct Body_{name} {{",
           f"  static constexpr int UNROLL = {unroll};",
           "  template <class C>",
           "  __device__ __forceinline__ static void compute(const csd::TileView<C>& t, int r, int y,",
           "                                                 int x, csd::OutPack<typename C::T, "
           "C::NOUT, C::VEC * C::RPY>& o) {",
           f"    static_assert(C::VEC == {vec} && C::RPY == {rpy}, "
           f"\"body emitted for {vec} points x {rpy} rows per thread\");"]
    for gi, key in enumerate(gkeys):
        f, dz, dy = key
        lo, hi = min(groups[key]), max(groups[key])
        out.append(f"    const auto st{gi} = t.template strip<{f}, {dz}, {dy}, {lo}, {hi}>(r, y, x);")
    access_types = {}
    n_scal = kernel.scalar_count.data if kernel.scalar_count is not None else 0
    n_dyn = kernel.dyn_count.data if kernel.dyn_count is not None else 0
    for k in range(n_scal):
        out.append(f"    const double s{k} = t.scalar({k});")
        access_types[f"s{k}"] = "w"
    for k in range(n_dyn):
        out.append(f"    const double d{k} = t.dynamic({k});")
        access_types[f"d{k}"] = "w"

    # classes of every SSA value of every member (members share classes, so a
    # value two fused members both compute is computed once too)
    classes = _ShiftClasses()
    members = []
    for prog in kernel.ssa_body.data:
        info: dict = {}        # SSA name -> (class id, (my, mx) or None)
        lines, rets = [], []
        for raw in (x.data for x in prog):
            lhs, op, args, typ, extra = _parse_line(raw)
            if op == "return":
                rets.append((args[0], extra))
                continue
            if op == "const":
                info[lhs] = (classes.intern(("const", typ, repr(extra))), None)
                lines.append((lhs, op, [], typ, extra))
                continue
            parts = []
            for a in args:
                if a[0] == "a" and a[1:].isdigit():
                    dz, dy, dx, f = acc_info[int(a[1:])]
                    parts.append((classes.intern(("leaf", f, dz)), (dy, dx)))
                elif a[0] in "sd" and a[1:].isdigit():
                    parts.append((classes.intern(("scalar", a)), None))
                else:
                    parts.append(info[a])
            pos = [m for _, m in parts if m is not None]
            mn = (min(m[0] for m in pos), min(m[1] for m in pos)) if pos else None
            key = (op, typ, extra, tuple(
                (c, None if m is None else (m[0] - mn[0], m[1] - mn[1])) for c, m in parts))
            info[lhs] = (classes.intern(key), mn)
            lines.append((lhs, op, args, typ, extra))
        members.append((info, lines, rets))

    def rename(a: str, info: dict, j: int, k: int) -> str:
        if a[0] == "a" and a[1:].isdigit():
            dz, dy, dx, f = acc_info[int(a[1:])]
            key = (f, dz, dy + j)
            gi = gindex[key]
            idx = k + dx - min(groups[key])
            leaf = f"L{gi}_{idx}"
            if leaf not in access_types:
                access_types[leaf] = field_t
                out.append(f"    const {store_t} q_{leaf} = st{gi}.v[{idx}];")
            return leaf
        if a[0] in "sd" and a[1:].isdigit():
            return a
        cid, mn = info[a]
        return _pos_name(cid, None if mn is None else (j + mn[0], k + mn[1]))

    emitted: set = set()
    ssa: list[str] = []
    stores = []
    for j in range(rpy):
        for k in range(vec):
            for m, (info, lines, rets) in enumerate(members):
                for lhs, op, args, typ, extra in lines:
                    nm = rename(lhs, info, j, k)
                    if nm in emitted:
                        continue
                    emitted.add(nm)
                    if op == "const":
                        ssa.append(f"{nm} = const {extra!r} : {typ}")
                    else:
                        tail = f" @{extra}" if extra is not None else ""
                        ssa.append(f"{nm} = {op} {', '.join(rename(a, info, j, k) for a in args)}"
                                   f"{tail} : {typ}")
                for res, idx in rets:
                    stores.append((m if idx is None else idx, j * vec + k, rename(res, info, j, k)))
    em = _BodyEmitter("q_")
    em.emit(ssa, access_types)
    for line in em.lines:
        out.append("    " + line)
    for slot, e, res in stores:
        out.append(f"    o.v[{slot}][{e}] = {em.result_as(res, store_t)};")
    out.append("  }")
    out.append("};")
    return "\n".join(out)


def _internal_radius(ndim: int, radius) -> tuple[int, int, int]:
    r = list(radius)
    if ndim == 3:
        return (r[0], r[1], r[2])
    if ndim == 2:
        return (r[0], 0, r[1])
    return (0, 0, r[0])


def engine_params(kernel: KernelOp) -> dict:
    """Template parameters of the engine instance described by *kernel*."""
    ndim = kernel.ndim.data
    dtype = kernel.dtype.data
    tile = [a.data for a in kernel.tile_shape.data]
    hints = {}
    if kernel.kernel_hints is not None:
        items = [a.data for a in kernel.kernel_hints.data]
        hints = {k: eval(v, {}) for k, v in zip(items[0::2], items[1::2])}  # repr'd ints
    if ndim == 3:
        rows, ty, tx = tile
    elif ndim == 2:
        rows, tx = tile
        ty = 1
    else:
        (tx,) = tile
        rows, ty = 1, 1
    rz, ry, rx = _internal_radius(ndim, [a.data for a in kernel.radius.data])
    nout = sum(max(1, sum(1 for s in prog if s.data.startswith("return")))
               for prog in kernel.ssa_body.data)
    nin = len(kernel.input_names.data)
    return {
        "T": "float" if dtype in ("float32", "fp32") else "double",
        "dtype_bytes": 4 if dtype in ("float32", "fp32") else 8,
        "NIN": nin, "NOUT": nout, "RZ": rz, "RY": ry, "RX": rx, "ROWS": rows, "TY": ty, "TX": tx,
        "NT": int(hints.get("threads", 256)), "STAGES": int(hints.get("stages", 1)),
        "TEMPORAL": kernel.temporal_steps.data if kernel.temporal_steps is not None else 1,
        "BC": BC_CODES[kernel.boundary_mode.data if kernel.boundary_mode is not None else "none"],
        "MINB": int(hints.get("min_blocks", 1)), "ZCHUNK": (int(hints.get("zchunk", 0)) if int(hints.get("zchunk", 0)) > 0
                   else -int(hints.get("waves", 1)) if int(hints.get("waves", 1)) > 1 else 0),
        "ndim": ndim,
        "NSCAL": kernel.scalar_count.data if kernel.scalar_count is not None else 0,
        "NDYN": kernel.dyn_count.data if kernel.dyn_count is not None else 0,
        "REDUCE": kernel.reduce_max.data if kernel.reduce_max is not None else 0,
        "BRICK": _brick_code(kernel, ndim),
        "RPY": int(hints.get("rpy", 1)),
        "VEC": int(hints.get("vec", 4 if dtype in ("float32", "fp32") else 2)),
    }


def brick_tma_eligible(p: dict) -> bool:
    """Whether a bricked kernel's TMA entry can stage bricks with tensor copies
    (engine.cuh ``Cfg::BTMA``): 3-D bricks, one Z row per chunk, one step, no
    periodic wrap, a tile height dividing the brick or a multiple of it and
    a tile width that is a whole number of bricks, bricks at least 16 bytes wide, at most 256
    bricks per staged row."""
    code = p["BRICK"]
    if not code or (code >> 4) != 3:
        return False
    b = 1 << (code & 15)
    esz = p["dtype_bytes"]
    balign = max(b, 128 // esz)
    padl = -(-p["RX"] // b) * b
    boxw = -(-(padl + p["TX"] + p["RX"]) // balign) * balign
    return (p["ROWS"] == 1 and p["TEMPORAL"] == 1 and p["BC"] != BC_CODES["periodic"]
            and (b % p["TY"] == 0 or p["TY"] % b == 0) and p["TX"] % b == 0 and (b * esz) % 16 == 0
            and boxw // b <= 256)


def _brick_code(kernel: KernelOp, ndim: int) -> int:
    """(ndim << 4) | log2(brick size) for a bricked-layout kernel, else 0."""
    if kernel.layout is None or kernel.layout.data != "bricked":
        return 0
    b = kernel.brick_size.data if kernel.brick_size is not None else 0
    if b < 4 or b > 64 or (b & (b - 1)):
        raise ValueError(f"brick size must be a power of two in [4, 64], got {b}")
    return (ndim << 4) | (b.bit_length() - 1)


def emit_cuda(module: ModuleOp, preamble: bool = True) -> str:
    """CUDA translation unit for the kernel(s) in a D3 module (``preamble=False``
    gives just the kernels, to append to another unit)."""
    kernels = [op for op in module.body.block.ops if isinstance(op, KernelOp)]
    if not kernels:
        raise ValueError("No KernelOp found in target IR module")
    parts = ["// Generated B200 stencil kernel(s). Do not edit.",
             '#include "csd/engine.cuh"', "",
             "__device__ __forceinline__ double csd_max(double a, double b) "
             "{ return (a != a || a > b) ? a : b; }",
             "__device__ __forceinline__ double csd_min(double a, double b) "
             "{ return (a != a || a < b) ? a : b; }",
             "__device__ __forceinline__ float csd_max(float a, float b) "
             "{ return (a != a || a > b) ? a : b; }",
             "__device__ __forceinline__ float csd_min(float a, float b) "
             "{ return (a != a || a < b) ? a : b; }", ""]
    if not preamble:
        parts = []
    for kernel in kernels:
        name = kernel.kernel_name.data
        p = engine_params(kernel)
        parts.append(f"// expression: {kernel.expression.data}")
        parts.append(emit_body(kernel))
        parts.append("")
        brick_tma = brick_tma_eligible(p)
        for suffix, loader in (("tma", "CSD_LOADER_TMA"), ("ldg", "CSD_LOADER_LDG")):
            if p["BRICK"] and not brick_tma:
                loader = "CSD_LOADER_LDG"   # bricked fields the TMA boxes cannot stage
            cfg = (f"csd::Cfg<{p['T']}, {p['NIN']}, {p['NOUT']}, {p['RZ']}, {p['RY']}, {p['RX']}, "
                   f"{p['ROWS']}, {p['TY']}, {p['TX']}, {p['NT']}, {p['STAGES']}, {p['TEMPORAL']}, "
                   f"{loader}, {p['BC']}, {p['REDUCE']}, {p['BRICK']}, {p['RPY']}, {p['VEC']}>")
            parts.append(f"typedef {cfg} Cfg_{name}_{suffix};")
            parts.append(f'extern "C" __global__ void __launch_bounds__({p["NT"]}, {p["MINB"]})')
            parts.append(f"{name}_{suffix}(const __grid_constant__ csd_params p) {{")
            parts.append(f"  csd::stream_engine<Cfg_{name}_{suffix}, Body_{name}>(p);")
            parts.append("}")
        c = f"Cfg_{name}_tma"
        parts.append(f'extern "C" __device__ const csd_kernel_desc {name}_desc = {{')
        nout_desc = "0" if p["REDUCE"] else f"{c}::NOUT"
        parts.append(f"  CSD_DESC_MAGIC, {p['ndim']}, {c}::NIN, {nout_desc}, (int)sizeof({c}::T),")
        parts.append(f"  {c}::RZ * {c}::TEMPORAL, {c}::RY * {c}::TEMPORAL, {c}::RX * {c}::TEMPORAL,")
        parts.append(f"  {c}::ROWS, {c}::TY, {c}::TX, {c}::VEC, {c}::NT, {c}::STAGES, {c}::NSLOT,")
        # both entries launch with one shared-memory size: the larger one
        smem = (f"({c}::SMEM_BYTES > Cfg_{name}_ldg::SMEM_BYTES ? {c}::SMEM_BYTES : "
                f"Cfg_{name}_ldg::SMEM_BYTES)")
        parts.append(f"  {c}::HC * {c}::TEMPORAL, {c}::PADL, {c}::BOXW, {c}::BOXH, {smem},")
        parts.append(f"  {p['ZCHUNK']}, {c}::TEMPORAL, {c}::BC, {p['MINB']}, {c}::ALIGN,")
        parts.append(f"  {p['NSCAL']}, {p['NDYN']}, {p['REDUCE']}, {c}::BRICK_SHIFT, "
                     f"{1 if brick_tma else 0}}};")
        parts.append("")
    return "\n".join(parts) + "\n"


__all__ = ["emit_cuda", "emit_body", "engine_params", "hex_literal", "brick_tma_eligible"]
