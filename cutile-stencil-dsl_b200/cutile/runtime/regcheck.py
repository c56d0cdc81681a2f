"""Register and spill checks of candidate kernel configurations.

The reference (runtime/regcheck.py:41-306) captures cuTile's cubins and reads
their resource usage with ``cuobjdump -res-usage``, then keeps the first
candidate that neither spills nor exceeds the register budget of its
occupancy target, or the fastest measured one.  Here the kernels are this
project's own NVRTC builds, so the resources come from ptxas' own report of
the build (``-Xptxas -v``: registers, stack frame, spill stores) and, on a
GPU, from ``cudaFuncGetAttributes``-style queries (``csd_kernel_resources``).
No compiled code is read.

``Config`` / ``Resources`` / ``register_budget`` / ``select_config`` /
``select_fastest`` keep the reference's names and selection rules.
"""

from __future__ import annotations

import re
from dataclasses import dataclass, field
from typing import Callable, Optional, Sequence


@dataclass(frozen=True)
class Resources:
    """Per-thread resources of a compiled kernel, and optionally its measured
    time per launch (``ms``) on a probe domain."""

    registers: int
    stack_bytes: int
    ms: Optional[float] = None
    spill_bytes: int = 0

    @property
    def spills(self) -> bool:
        return self.spill_bytes > 0 or self.stack_bytes > 0


@dataclass(frozen=True)
class Config:
    """A candidate: tile sizes and kernel hints (``threads``, ``stages``,
    ``min_blocks``/``occupancy``, ``zchunk``, ``waves``), plus the register
    budget it must meet (``None``: the budget given to the selection)."""

    tile_sizes: tuple
    kernel_hints: dict = field(default_factory=dict)
    max_registers: Optional[int] = None
    temporal_steps: int = 1


def parse_ptxas_log(text: str, entry: str | None = None) -> Optional[Resources]:
    """Resources of ``entry`` (or of the first entry function) from a ptxas
    ``-v`` report: the worst of the function's own frame and spill counts."""
    blocks = re.split(r"Compiling entry function '", text)[1:]
    for blk in blocks:
        name = blk.split("'", 1)[0]
        if entry is not None and name != entry:
            continue
        regs = re.search(r"Used (\d+) registers", blk)
        # NVRTC prefixes the frame line with "ptxas ."; nvcc's report does not
        frame = re.search(r"Function properties for " + re.escape(name) +
                          r"\s*\n\s*(?:ptxas\s+\.\s+)?(\d+) bytes stack frame, "
                          r"(\d+) bytes spill stores", blk)
        if regs is None:
            continue
        stack = int(frame.group(1)) if frame else 0
        spill = int(frame.group(2)) if frame else 0
        return Resources(registers=int(regs.group(1)), stack_bytes=stack, spill_bytes=spill)
    return None


def register_budget(occupancy: int, threads_per_block: int = 128,
                    registers_per_sm: int = 65536) -> int:
    """Registers per thread that keep ``occupancy`` blocks resident per SM."""
    return registers_per_sm // (occupancy * threads_per_block)


def _budget(cfg: Config, max_registers: Optional[int]) -> Optional[int]:
    return cfg.max_registers if cfg.max_registers is not None else max_registers


def _fits(cfg: Config, res: Resources, max_registers: Optional[int]) -> bool:
    b = _budget(cfg, max_registers)
    return not res.spills and (b is None or res.registers <= b)


def select_config(configs: Sequence[Config], probe: Callable[[Config], Optional[Resources]],
                  max_registers: Optional[int] = None) -> Config:
    """The first configuration whose kernel fits (no spill, registers within
    its budget).  An unavailable probe (``None``) keeps the configuration
    under test; when none fits, the first that does not spill, else the last
    (most conservative) candidate."""
    if not configs:
        raise ValueError("no candidate configurations")
    seen = []
    for cfg in configs:
        res = probe(cfg)
        if res is None:
            return cfg
        if _fits(cfg, res, max_registers):
            return cfg
        seen.append((cfg, res))
    for cfg, res in seen:
        if not res.spills:
            return cfg
    return configs[-1]


def select_fastest(configs: Sequence[Config], probe: Callable[[Config], Optional[Resources]],
                   max_spill_bytes: int = 512, margin: float = 0.03,
                   max_registers: Optional[int] = None) -> Config:
    """Probe every configuration and keep the fastest measured one; kernels
    spilling more than ``max_spill_bytes`` are trusted only when nothing else
    was timed, and the earliest candidate within ``margin`` of the best time
    wins (the candidate order breaks near-ties).  Without timings the rule of
    :func:`select_config` applies; without any probe result, the first
    configuration."""
    if not configs:
        raise ValueError("no candidate configurations")
    probed = []
    for k, cfg in enumerate(configs):
        res = probe(cfg)
        if res is None:
            if k == 0:
                return cfg
            continue
        probed.append((cfg, res))
    if not probed:
        return configs[0]
    timed = [(c, r) for c, r in probed if r.ms is not None]
    if timed:
        pool = [(c, r) for c, r in timed if r.spill_bytes <= max_spill_bytes] or timed
        best = min(r.ms for _, r in pool)
        for c, r in pool:
            if r.ms <= best * (1.0 + margin):
                return c
    for c, r in probed:
        if _fits(c, r, max_registers):
            return c
    for c, r in probed:
        if not r.spills:
            return c
    return configs[-1]


def probe_build(stencil_fn, cfg: Config, *, dtype: str | None = None,
                align_halo: bool = True, entry_suffix: str = "_tma") -> Optional[Resources]:
    """Resources of ``stencil_fn`` built with ``cfg`` (NVRTC, no GPU)."""
    from cutile.runtime.launcher import compile as stencil_compile
    from cutile.runtime.native import compile_source

    hints = dict(cfg.kernel_hints)
    r = stencil_compile(stencil_fn, tile_sizes=tuple(cfg.tile_sizes), kernel_hints=hints,
                        temporal_steps=cfg.temporal_steps, dtype=dtype, align_halo=align_halo,
                        autotune=False)
    _, log = compile_source(r.cuda_source, ["-Xptxas=-v"])
    return parse_ptxas_log(log, r.name + entry_suffix)


__all__ = ["Resources", "Config", "parse_ptxas_log", "register_budget", "select_config",
           "select_fastest", "probe_build"]
