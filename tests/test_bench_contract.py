"""The benchmark contract: bench.py's reference arm (CPU: fr_sdg's own residual code,
oracle/_ref, on the host cores) and our arm (GPU, on a 64^2 version of the workload) each print one JSON
line with the keys of the contract."""
from __future__ import annotations

import json
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def test_reference_arm_line():
    res = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "2",
                          "--warmup", "1"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert res.returncode == 0, res.stderr[-2000:]
    lines = [ln for ln in res.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for key in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "higher_is_better", "scaling",
                "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference" and d["value"] > 0 and d["steps"] == 2 and d["warmup"] == 1
    assert d["e2e"]["value"] == d["value"] and d["e2e"]["h2d_bytes_per_step"] == 0
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] >= 1
    assert d["config"]["workload"].startswith("blast_vdw_1024x1024_p5")
    assert d["config"]["elements"] == [1024, 1024] and d["ms_per_step"] > 0
    # the reference arm runs the reference's code alone: the CUDA library is never loaded
    assert d["libraries_loaded"] == ["oracle/_ref/libfrsdg_ref.so"]


@pytest.mark.gpu
def test_our_arm_line_small(cuda):
    """Our arm on a 64^2 version of the workload: the contract keys, the roofline and clock
    records and a positive end-to-end figure."""
    res = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--elements", "64", "--steps", "3", "--warmup", "3",
                          "--no-t-end", "--no-cpu-baseline", "--e2e-steps", "2"],
                         capture_output=True, text=True, timeout=900, cwd=ROOT)
    assert res.returncode == 0, res.stderr[-2000:]
    lines = [ln for ln in res.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "clocks", "gpu_launches", "roofline", "e2e"):
        assert key in d, key
    assert d["n_gpus"] == 1 and d["steps"] == 3 and d["warmup"] >= 3 and d["gpu_launches"] == 3
    r = d["roofline"]
    assert r["bound"] == "hbm" and r["unit"] == "GB/s" and 0 < r["frac"] and r["achieved"] > 0
    e = d["e2e"]
    assert e["value"] > 0 and e["h2d_bytes_per_step"] == e["d2h_bytes_per_step"] > 0
    assert "sm_mhz" in d["clocks"] and "reasons" in d["clocks"]
