"""GPU presets and hardware specs (reference: cutile/config.py:16-247), with B200.

The B200 preset uses the dense, non-sparse datasheet figures; runtime code
that reports a roofline fraction takes its peak from a measured copy
bandwidth instead (``HardwareSpec.measured``).
"""

from __future__ import annotations

import json
import os
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple


@dataclass(frozen=True)
class GPUPreset:
    name: str
    peak_bandwidth_gbs: float
    shared_mem_bytes: int
    sm_count: int
    peak_gflops_fp64: float
    peak_gflops_fp32: float

    def peak_gflops(self, dtype: str = "float64") -> float:
        return self.peak_gflops_fp32 if dtype in ("float32", "fp32") else self.peak_gflops_fp64


B200 = GPUPreset("B200", peak_bandwidth_gbs=7700.0, shared_mem_bytes=227 * 1024, sm_count=148,
                 peak_gflops_fp64=37000.0, peak_gflops_fp32=75000.0)
H100_SXM = GPUPreset("H100_SXM", 3350.0, 232 * 1024, 132, 33500.0, 67000.0)
H100_PCIe = GPUPreset("H100_PCIe", 2039.0, 232 * 1024, 114, 24000.0, 48000.0)
A100_80GB = GPUPreset("A100_80GB", 2039.0, 164 * 1024, 108, 9746.0, 19492.0)
A100_40GB = GPUPreset("A100_40GB", 1555.0, 164 * 1024, 108, 9746.0, 19492.0)
V100 = GPUPreset("V100", 900.0, 96 * 1024, 80, 7066.0, 14131.0)
RTX4090 = GPUPreset("RTX4090", 1008.0, 100 * 1024, 128, 1290.0, 82580.0)
RTX_PRO_6000 = GPUPreset("RTX_PRO_6000", 1792.0, 228 * 1024, 188, 1953.0, 125000.0)

GPU_PRESETS: Dict[str, GPUPreset] = {p.name: p for p in (
    B200, H100_SXM, H100_PCIe, A100_80GB, A100_40GB, V100, RTX4090, RTX_PRO_6000)}


@dataclass
class HardwareSpec:
    """Hardware parameters used by analysis and code generation."""

    shared_mem_bytes: int = 49152
    dtype_bytes: int = 8
    peak_bandwidth_gbs: float = 900.0
    peak_gflops: float = 7066.0
    sm_count: int = 80

    @classmethod
    def from_preset(cls, name: str, dtype: str = "float64") -> "HardwareSpec":
        p = GPU_PRESETS[name]
        return cls(shared_mem_bytes=p.shared_mem_bytes,
                   dtype_bytes=4 if dtype in ("float32", "fp32") else 8,
                   peak_bandwidth_gbs=p.peak_bandwidth_gbs, peak_gflops=p.peak_gflops(dtype),
                   sm_count=p.sm_count)

    @classmethod
    def auto_detect(cls, dtype: str = "float64") -> "HardwareSpec":
        p = _auto_detect_gpu() or V100
        return cls(shared_mem_bytes=p.shared_mem_bytes,
                   dtype_bytes=4 if dtype in ("float32", "fp32") else 8,
                   peak_bandwidth_gbs=p.peak_bandwidth_gbs, peak_gflops=p.peak_gflops(dtype),
                   sm_count=p.sm_count)

    @staticmethod
    def measured_peak_gbs(path: Optional[str] = None) -> Optional[float]:
        """Measured copy bandwidth from a ``MEASURED_PEAKS.json`` (``hbm_gbs``)."""
        path = path or os.environ.get("CSD_MEASURED_PEAKS")
        if not path or not os.path.exists(path):
            return None
        with open(path) as f:
            return float(json.load(f).get("hbm_gbs"))


def _auto_detect_gpu() -> Optional[GPUPreset]:
    name = None
    try:
        import torch

        if torch.cuda.is_available():
            name = torch.cuda.get_device_name(0)
    except Exception:
        name = None
    if not name:
        return None
    up = name.upper()
    if "B200" in up:
        return B200
    for key, preset in GPU_PRESETS.items():
        if key.replace("_", " ") in up or key.replace("_", "") in up:
            return preset
    if "H100" in up:
        return H100_SXM if "SXM" in up else H100_PCIe
    if "A100" in up:
        return A100_80GB if "80" in up else A100_40GB
    return None


@dataclass
class TilingConfig:
    candidate_sizes: List[int] = field(default_factory=lambda: [32, 64, 128, 256, 512, 1024])
    max_temporal_steps: int = 16


@dataclass
class BenchmarkConfig:
    grid_sizes: Dict[int, Tuple[int, ...]] = field(default_factory=lambda: {
        1: (1024 * 1024,), 2: (1024, 1024), 3: (64, 64, 64)})
    warmup_iters: int = 5
    benchmark_iters: int = 20


DEFAULT_HW = HardwareSpec()
DEFAULT_TILING = TilingConfig()
DEFAULT_BENCHMARK = BenchmarkConfig()
