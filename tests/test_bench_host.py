"""bench.py's summaries of secondary workloads (no GPU): the compact entry
keeps value, roofline, clocks and the comparison figures, drops the serving
timeline, and a failed child process is reported, not raised."""

import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def test_summary_keeps_the_figures_and_drops_the_timeline():
    import bench

    line = {"metric": "m", "value": 1.5, "unit": "GPts/s", "steps": 3, "ms_per_step": 0.2,
            "config": {"workload": "w", "tile": [1, 8, 64], "temporal_steps": 2},
            "roofline": {"bound": "hbm", "achieved": 10.0, "peak": 20.0, "unit": "GB/s",
                         "frac": 0.5, "traffic": None, "algorithmic_bytes_per_launch": 8,
                         "peak_kind": "measured"},
            "e2e": {"value": 1.0, "unit": "GPts/s", "h2d_bytes_per_step": 4},
            "clocks": {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": [], "samples": 3},
            "gpu_launches": 3, "latency_ms": {"p50": 1.0},
            "comparison": {"server": {"timeline": [[1, 2, 3]], "launches": 7}, "x": 2}}
    s = bench._summary(line)
    assert s["value"] == 1.5 and s["unit"] == "GPts/s" and s["tile"] == [1, 8, 64]
    assert s["temporal_steps"] == 2 and s["roofline"]["frac"] == 0.5
    assert "peak_kind" not in s["roofline"]
    assert s["e2e"] == {"value": 1.0, "unit": "GPts/s"}
    assert s["clocks"] == {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": []}
    assert s["comparison"]["server"] == {"launches": 7} and s["comparison"]["x"] == 2
    json.dumps(s)


def test_secondary_reports_a_failing_child(monkeypatch):
    import subprocess

    import bench

    class Done:
        returncode = 1
        stdout = ""
        stderr = "Traceback\nRuntimeError: no device"

    monkeypatch.setattr(bench, "SECONDARY", (("broken", ["--workload", "wide"]),))
    monkeypatch.setattr(subprocess, "run", lambda *a, **k: Done())
    res = bench.run_secondary(budget_s=100)
    assert res["broken"]["error"].startswith("rc=1") and "no device" in res["broken"]["error"]


def test_traffic_records_match_the_algorithmic_bytes():
    """Each committed DRAM-traffic record (ncu at 320^3, scaled to 512^3) is
    within 10 % of one read and one write of the field per launch: the
    kernels re-read nothing, and a stale record would show here."""
    import bench

    for dtype, size in (("float64", 8), ("float32", 4)):
        for T in (1, 2, 4):
            for layout in ("flat", "bricked"):
                t = bench._profiled_traffic(dtype, T, layout)
                if t is None:
                    continue
                alg = 2 * size * 512 ** 3
                assert 0.9 * alg <= t <= 1.1 * alg, (dtype, T, layout, t / alg)
    assert bench._profiled_traffic("float64", 1) is not None
    assert bench._profiled_traffic("float64", 1, "bricked") is not None


def test_secondary_lines_cover_the_sweep_variants():
    """The 7-point configuration's variants: FP32, chains of 2, 4 and 8 steps
    in both dtypes, resident 8^3 bricks."""
    import bench

    args = {name: " ".join(extra) for name, extra in bench.SECONDARY}
    for dt in ("", "--dtype float32 "):
        for T in (2, 4, 8):
            assert any(a.startswith(f"{dt}--temporal {T} ") or a == f"{dt}--temporal {T}"
                       for a in args.values()), (dt, T)
    assert any("--layout bricked" in a for a in args.values())
    assert any(a.startswith("--dtype float32 --steps") for a in args.values())
