"""bench.py's GPU arm at a small grid keeps the JSON contract: the headline metric with a
roofline of the PCG kernel, the CPU baseline, the end-to-end figure through the host-buffer
entry point, the kernel launch count and the clocks seen during the timed region."""
import json
import subprocess
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent


def _line(*args):
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), *args], capture_output=True, text=True, timeout=900,
                       cwd=ROOT)
    assert r.returncode == 0, r.stderr[-3000:]
    lines = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    return lines[0]


def test_flip_line_contract():
    d = _line("--grid", "32", "--steps", "3", "--warmup", "3")
    assert d["metric"] == "particle-steps/s at 32^3 FLIP (1e-6 rel residual)" and d["value"] > 0
    assert d["n_gpus"] == 1 and d["steps"] == 3 and d["warmup"] == 3 and d["higher_is_better"] is True
    assert d["config"]["workload"] == "flip_dam_break_32"
    rf = d["roofline"]
    assert rf["bound"] == "hbm" and rf["unit"] == "GB/s" and rf["peak"] > 0
    assert abs(rf["frac"] - rf["achieved"] / rf["peak"]) < 1e-9 and rf["achieved"] > 0
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] > 0
    e2e = d["e2e"]
    assert 0 < e2e["value"] <= d["value"] * 1.05
    assert e2e["h2d_bytes_per_step"] == 24 * d["config"]["particles"] == e2e["d2h_bytes_per_step"]
    assert d["gpu_launches"] >= 3 * 20
    assert d["clocks"]["samples"] >= 0 and "reasons" in d["clocks"]


def test_pcg_line():
    d = _line("--workload", "pcg", "--steps", "50", "--warmup", "1")
    assert d["unit"] == "us/iteration" and d["value"] > 0 and d["steps"] == 50 and d["gpu_launches"] >= 1
