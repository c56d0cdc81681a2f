"""Tiling: the reference's row-tile policy and the B200 engine's tile plan.

``TilingPass`` keeps the reference's interface and answers
(cutile/passes/tiling.py:68-207): tiers by distinct-access count (narrow
<= 16 < wide <= 64 < very wide), ``candidates()`` ladders with ``occupancy``
hints, ``tile_for()``, and the ``tile_sizes`` attribute on each apply.  Those
row tiles are what the reference's temporal-blocking formula sizes against
(temporal.py:66-76), so keeping them keeps ``compile()``'s default
``temporal_steps`` -- and therefore how many steps one ``launch_<name>``
call advances -- identical to the reference.

``EngineTilingPass`` is the B200 policy the kernels actually run with: a
streaming engine that walks dimension 0 and tiles the remaining dimensions
(see ``EnginePlan``), sized for 227 KB of shared memory per block, 148 SMs,
16-byte TMA rows and 128-bit vector stores.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field, replace
from typing import ClassVar

from cutile.dialects.stencil import AccessOp, ApplyOp
from cutile.ir.core import ArrayAttr, Context, IntAttr, ModuleOp, ModulePass, StringAttr


def unique_access_count(apply_op: ApplyOp) -> int:
    """Distinct ``(field, offset)`` reads of a ``stencil.apply`` (tiling.py:68-79)."""
    seen = set()
    for child in apply_op.region.walk():
        if isinstance(child, AccessOp):
            seen.add((id(child.temp), tuple(child.offset)))
    return len(seen)


@dataclass(frozen=True)
class TilingPass(ModulePass):
    """Row tiles from the stencil's access count (reference policy)."""

    name: ClassVar[str] = "stencil-tiling"

    shared_mem_bytes: int = 49152
    dtype_bytes: int = 8
    threads_per_block: int = 128
    wide_stencil_loads: int = 16
    very_wide_stencil_loads: int = 64
    narrow_elements_per_thread: int = 2
    wide_elements_per_thread: int = 1
    very_wide_occupancy: int = 4
    min_occupancy: int = 3
    wide_inner: int = 64
    max_inner: int = 1024

    def apply(self, ctx: Context, op: ModuleOp) -> None:
        for child in op.walk():
            if isinstance(child, ApplyOp):
                self._tile_apply(child)

    def _tile_apply(self, apply_op: ApplyOp) -> None:
        halo_attr = apply_op.attributes.get("halo_widths")
        if halo_attr is None:
            return
        ndim = len(halo_attr)
        tile, hints = self.candidates(ndim, unique_access_count(apply_op))[0]
        apply_op.attributes["tile_sizes"] = ArrayAttr([IntAttr(s) for s in tile])
        if "occupancy" in hints:
            apply_op.attributes["occupancy"] = IntAttr(hints["occupancy"])

    def tier(self, num_loads: int) -> str:
        if num_loads <= self.wide_stencil_loads:
            return "narrow"
        if num_loads > self.very_wide_stencil_loads:
            return "very_wide"
        return "wide"

    def elements_per_thread(self, num_loads: int) -> int:
        if self.tier(num_loads) == "wide":
            return self.wide_elements_per_thread
        return self.narrow_elements_per_thread

    def is_wide(self, num_loads: int) -> bool:
        return self.tier(num_loads) == "wide"

    def candidates(self, ndim: int, num_loads: int) -> list[tuple[tuple[int, ...], dict]]:
        """``(tile_sizes, kernel_hints)`` in order of preference (tiling.py:161-191)."""
        one_row = self._row_tile(ndim, self.wide_elements_per_thread, self.wide_inner)
        single_row = self._row_tile(ndim, self.wide_elements_per_thread, 2 * self.wide_inner)
        two_rows = self._row_tile(ndim, self.narrow_elements_per_thread, self.max_inner)
        tier = self.tier(num_loads)
        if tier == "narrow":
            return [(two_rows, {})]
        ladder = [(two_rows, {"occupancy": self.very_wide_occupancy})]
        ladder += [(one_row, {"occupancy": occ})
                   for occ in range(self.very_wide_occupancy, self.min_occupancy - 1, -1)]
        ladder.append((single_row, {"occupancy": self.min_occupancy}))
        unhinted = (one_row, {})
        ordered = [unhinted] + ladder if tier == "wide" else ladder + [unhinted]
        seen: list = []
        for cand in ordered:
            if cand not in seen:
                seen.append(cand)
        return seen

    def tile_for(self, ndim: int, num_loads: int) -> list[int]:
        return list(self.candidates(ndim, num_loads)[0][0])

    def _row_tile(self, ndim: int, elements_per_thread: int, inner_cap: int) -> tuple[int, ...]:
        elements = self.threads_per_block * elements_per_thread
        if ndim == 1:
            return (elements * 4,)
        tile = [1] * ndim
        inner = min(elements, inner_cap)
        tile[-1] = inner
        tile[-2] = max(1, elements // inner)
        return tuple(tile)


# --------------------------------------------------------------------------- #
# B200 engine plan
# --------------------------------------------------------------------------- #

B200_SMEM_PER_BLOCK = 227 * 1024
B200_SMEM_PER_SM = 228 * 1024
B200_SM_COUNT = 148
B200_MAX_THREADS_PER_SM = 2048
TMA_BOX_MAX = 256


@dataclass(frozen=True)
class EnginePlan:
    """Tile configuration of the streaming stencil engine.

    Arrays are viewed as 3-D ``(Z, Y, X)`` with X innermost (a 2-D array is
    ``(rows, 1, cols)``, a 1-D one ``(1, 1, n)``).  A work item is a column of
    ``tile_y x tile_x`` points that streams through ``zchunk`` output rows of
    Z, ``rows`` rows per step; each thread owns ``vec`` consecutive X points
    of ``units_per_thread`` positions per step.  Input rows arrive through a
    ring of ``nslot`` shared-memory chunks (``stages`` of them in flight).
    ``temporal`` > 1 chains that many stencil steps inside one pass.
    """

    ndim: int
    rows: int
    tile_y: int
    tile_x: int
    vec: int
    threads: int
    stages: int
    zchunk: int
    temporal: int = 1
    min_blocks: int = 1        # resident blocks per SM the launch bound asks for (fit_plan)
    occupancy: int = 0         # explicit min_blocks request (0: fit_plan chooses)
    waves: int = 0             # auto zchunk: work items per resident block (0: fit_plan chooses)
    rpy: int = 1               # Y rows per thread (3-D, single step): strips shared by rows

    @property
    def units_per_step(self) -> int:
        return self.rows * (self.tile_y // self.rpy) * (self.tile_x // self.vec)

    @property
    def units_per_thread(self) -> int:
        return max(1, self.units_per_step // self.threads)

    def tile_sizes(self) -> tuple[int, ...]:
        if self.ndim == 3:
            return (self.rows, self.tile_y, self.tile_x)
        if self.ndim == 2:
            return (self.rows, self.tile_x)
        return (self.tile_x,)

    def hints(self) -> dict:
        h = {"threads": self.threads, "vec": self.vec, "stages": self.stages,
             "zchunk": self.zchunk, "min_blocks": self.min_blocks, "waves": self.waves}
        if self.rpy != 1:
            h["rpy"] = self.rpy
        return h


def _align_up(x: int, a: int) -> int:
    return -(-x // a) * a


def engine_geometry(plan: EnginePlan, radius3: tuple[int, int, int], dtype_bytes: int,
                    num_inputs: int, periodic: bool = False) -> dict:
    """Derived sizes, identical to the constexprs of ``csd::Cfg`` (engine.cuh);
    ``periodic`` adds the periodic-X wrap buffer of fused periodic kernels.

    ``radius3`` is the radius of ONE stencil step per internal dimension
    (Z, Y, X); ``plan.temporal`` steps are chained.
    """
    rz, ry, rx = radius3
    T = plan.temporal
    align = 16 // dtype_bytes
    hc = -(-rz // plan.rows) if rz > 0 else 0
    if T == 1:
        pad_left = _align_up(rx, max(align, plan.vec))   # Cfg::PADL: a unit starts on a vector
        box_w = _align_up(pad_left + plan.tile_x + rx, align)
    else:
        pad_left = _align_up(T * rx + 2 * align - 2, align)
        box_w = _align_up(pad_left + plan.tile_x + T * rx + 2 * align - 2, align)
    box_h = plan.tile_y + 2 * T * ry
    nslot = 2 * hc + 1 + plan.stages
    nslot_i = 2 * hc + 2   # engine.cuh Cfg::NSLOT_I (chain skew on)
    per128 = 128 // dtype_bytes
    slot_elems = _align_up(plan.rows * box_h * box_w, per128)
    inter = num_inputs * sum(nslot_i * _align_up(plan.rows * (plan.tile_y + 2 * (T - s) * ry) * box_w,
                                                 per128)
                             for s in range(1, T))
    wrapw = _align_up(rx, align) + align
    pbuf_slot = (num_inputs * 2 * _align_up(plan.rows * box_h * wrapw, per128)
                 if (periodic and rx > 0) else 0)
    smem = ((num_inputs * nslot * slot_elems + inter + nslot * pbuf_slot) * dtype_bytes
            + 8 * nslot + 64 + 128)
    return {"align": align, "pad_left": pad_left, "box_w": box_w, "box_h": box_h,
            "halo_chunks": hc, "nslot": nslot, "slot_elems": slot_elems,
            "smem_bytes": smem}


def default_engine_plan(ndim: int, num_loads: int, dtype_bytes: int, radius: tuple[int, ...],
                        num_inputs: int = 1, num_outputs: int = 1) -> EnginePlan:
    """B200 starting point (the autotuner refines it per grid-size class)."""
    vec = 16 // dtype_bytes
    wide = num_loads > 16
    # zchunk 0 = sized at launch so the work items fill the resident CTAs in
    # one wave (csd_launch).  Measured on B200 (7-point 512^3): single-wave,
    # 8-9 resident 128-thread blocks per SM with one chunk in flight each beat
    # deeper per-block prefetch (FP64 385 vs 297 GPts/s for 1x8x64/256t/2 stages).
    if ndim == 3:
        if dtype_bytes == 8:
            plan = EnginePlan(3, rows=1, tile_y=4, tile_x=128, vec=vec, threads=128, stages=1,
                              zchunk=0)
        else:
            # autotuned on B200 (7-point 512^3 FP32): two rows per step over a
            # 4x128 tile, 711 GPts/s against 559 for one row over 8x128
            plan = EnginePlan(3, rows=2, tile_y=4, tile_x=128, vec=vec, threads=128, stages=1,
                              zchunk=0)
        if wide:
            plan = replace(plan, tile_y=4, tile_x=64)
            if (dtype_bytes == 8 and num_inputs == 1 and num_outputs == 1
                    and max(radius) <= 2):
                # measured on B200 (dense boxes, 512^3 FP64): a thread owning
                # several Y rows reads each staged strip once for all of them;
                # 27 points: 4 rows over 16x64, 136 -> 264 GPts/s; 125 points
                # (radius 2, more strips live): 2 rows over 2x4x128, 55 -> 87.
                # Wider footprints keep one row (their strips would spill).
                if max(radius) <= 1:
                    plan = replace(plan, rows=1, tile_y=16, tile_x=64, threads=128, rpy=4)
                else:
                    plan = replace(plan, rows=2, tile_y=4, tile_x=128, threads=128, rpy=2)
    elif ndim == 2:
        # short single-field bodies (5/9-point) over 8 x 128 tiles: FP32 runs
        # best with 128 threads (heat 4096^2: 671 vs 574 GPts/s with 256),
        # FP64 with 256 (351 vs 312: two 2-point units per thread instead
        # of four); multi-field flux bodies keep 256
        short = num_loads <= 8 and dtype_bytes == 4
        plan = EnginePlan(2, rows=4 if wide else 8, tile_y=1, tile_x=128, vec=vec,
                          threads=128 if short else 256, stages=1, zchunk=0)
        if dtype_bytes == 8 and num_inputs > 1 and not wide:
            # several FP64 fields: 64-wide chunks keep 4 blocks per SM
            # (Gray-Scott 4096^2 fused periodic step: 179.9 vs 168.8 GPts/s
            # for 8 x 128 at 3 blocks per SM)
            plan = replace(plan, tile_x=64)
        rz = radius[0]
        if rz > plan.rows:
            plan = replace(plan, rows=_align_up(rz, 4))
    else:
        plan = EnginePlan(1, rows=1, tile_y=1, tile_x=128, vec=vec, threads=256, stages=0,
                          zchunk=0)
    # waves stay unset: the caller's fit_plan derives them from the body size
    return replace(fit_plan(plan, radius, dtype_bytes, num_inputs), waves=0)


def radius3(ndim: int, radius: tuple[int, ...]) -> tuple[int, int, int]:
    """Stencil radius per array dim -> (Z, Y, X) of the engine's 3-D view."""
    if ndim == 3:
        return (radius[0], radius[1], radius[2])
    if ndim == 2:
        return (radius[0], 0, radius[1])
    return (0, 0, radius[0])


def fit_plan(plan: EnginePlan, radius: tuple[int, ...], dtype_bytes: int,
             num_inputs: int, body_ops: int = 0, periodic: bool = False) -> EnginePlan:
    """Shrink a plan until its TMA box and shared memory fit the B200 limits."""
    r3 = radius3(plan.ndim, radius)
    if plan.rpy != 1 and (plan.ndim != 3 or plan.temporal != 1 or plan.rpy < 1):
        raise ValueError("rows per thread > 1 needs a 3-D single-step stencil")
    if plan.vec != 16 // dtype_bytes and (plan.vec % (16 // dtype_bytes) or plan.vec <= 0
                                          or plan.temporal != 1 or plan.rpy != 1):
        raise ValueError(f"a {plan.vec}-point unit needs a multiple of {16 // dtype_bytes} points, "
                         "one step and one row per thread")
    for _ in range(64):
        g = engine_geometry(plan, r3, dtype_bytes, num_inputs, periodic)
        ok_box = g["box_w"] <= TMA_BOX_MAX and g["box_h"] <= TMA_BOX_MAX
        if ok_box and g["smem_bytes"] <= B200_SMEM_PER_BLOCK - 1024:
            break
        if plan.stages > 1:
            plan = replace(plan, stages=plan.stages - 1)
        elif plan.tile_x > 32 and (not ok_box or plan.tile_x >= plan.tile_y * 8):
            plan = replace(plan, tile_x=plan.tile_x // 2)
        elif plan.tile_y > plan.rpy:
            plan = replace(plan, tile_y=max(plan.rpy, plan.tile_y // 2))
        elif plan.rows > 1 and plan.rows // 2 >= 1:
            plan = replace(plan, rows=plan.rows // 2)
        else:
            raise ValueError(f"stencil footprint {radius} does not fit the B200 engine")
    if plan.tile_y % plan.rpy:
        raise ValueError(f"tile height {plan.tile_y} is not a multiple of {plan.rpy} rows per thread")
    units = plan.units_per_step
    threads = min(plan.threads, units)
    while units % threads:
        threads //= 2
    threads = max(32, threads)
    zchunk = 0 if plan.zchunk <= 0 else max(plan.rows, (plan.zchunk // plan.rows) * plan.rows)
    g = engine_geometry(plan, r3, dtype_bytes, num_inputs, periodic)
    # resident blocks the shared memory allows, capped so the register budget
    # stays >= 64 per thread (128 for long bodies such as flux stencils, which
    # otherwise spill); the launch bound is a hint to ptxas, not a floor
    regs = 128 if body_ops > 120 or plan.rpy > 1 else 64
    fit_blocks = max(1, min(B200_SMEM_PER_SM // max(1, g["smem_bytes"] + 1024),
                            B200_MAX_THREADS_PER_SM // threads))
    if plan.occupancy > 0:    # an explicit occupancy hint, capped by what fits
        min_blocks = min(plan.occupancy, fit_blocks)
    else:
        min_blocks = max(1, min(fit_blocks, 65536 // (threads * regs)))
    # Auto-sized items: a memory-bound body runs best as one wave of long
    # items (neighbouring columns stream the same planes together and share
    # halo rows in L2); a long body (flux stencils) is issue-bound and wants
    # several shorter items per resident block so that blocks finish together
    # (measured on B200, 2-D shallow water RK stage on 2048^2: 16-row items
    # 114 us vs one 128-row item per block 184 us).
    # Temporal chains are latency-bound the same way (measured on 512^3 FP64,
    # T=2, 8 x 64 tiles: one wave 308, eight waves 343 GPts/s).
    waves = plan.waves if plan.waves > 0 else (8 if body_ops > 60 or plan.temporal > 1 else 1)
    return replace(plan, threads=threads, zchunk=zchunk, min_blocks=min_blocks, waves=waves)


@dataclass(frozen=True)
class EngineTilingPass(ModulePass):
    """Attach the B200 engine plan (``engine_tile``, ``engine_hints``) to each apply."""

    name: ClassVar[str] = "engine-tiling"
    dtype_bytes: int = 8
    temporal_steps: int = 1
    num_inputs: int | None = None
    overrides: dict = field(default_factory=dict)

    def apply(self, ctx: Context, op: ModuleOp) -> None:
        for child in op.walk():
            if isinstance(child, ApplyOp) and "halo_widths" in child.attributes:
                halo = tuple(a.data for a in child.attributes["halo_widths"])
                nin = self.num_inputs or child.attributes["num_arrays"].data
                plan = default_engine_plan(len(halo), unique_access_count(child), self.dtype_bytes,
                                           halo, nin)
                if self.overrides or self.temporal_steps != 1:
                    if self.temporal_steps != 1:
                        plan = replace(plan, rpy=1)   # temporal chains: one row per thread
                    plan = fit_plan(replace(plan, temporal=self.temporal_steps, **self.overrides),
                                    halo, self.dtype_bytes, nin)
                child.attributes["engine_tile"] = ArrayAttr([IntAttr(t) for t in plan.tile_sizes()])
                child.attributes["engine_threads"] = IntAttr(plan.threads)
                child.attributes["engine_layout"] = StringAttr("flat")


__all__ = ["TilingPass", "EngineTilingPass", "EnginePlan", "unique_access_count",
           "default_engine_plan", "fit_plan", "engine_geometry", "radius3", "B200_SM_COUNT",
           "B200_SMEM_PER_BLOCK", "math"]
