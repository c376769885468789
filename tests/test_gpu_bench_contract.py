"""`bench.py` on a small zoom box (N = 2^13): the JSON line carries every key of the benchmark
contract with sane values -- the metric and its unit, the roofline of the walk, the end-to-end figure
through host buffers with its copy volumes, the kernel launch count and the clock record."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_bench_json_line_small_case(cuda_lib):
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--log2-half", "12", "--steps", "2", "--warmup",
                          "3", "--no-cpu-baseline", "--no-serving"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "roofline", "e2e", "gpu_launches", "clocks"):
        assert k in line, k
    n = 1 << 13
    assert line["unit"] == "particles/s" and line["n_gpus"] == 1 and line["steps"] == 2 and line["warmup"] == 3
    assert line["value"] > 0 and abs(line["value"] * line["ms_per_step"] / 1e3 - n) < 1e-6 * n
    assert line["dtype"] == "f32" and line["config"]["n_particles"] == n
    r = line["roofline"]
    assert r["achieved"] > 0 and r["peak"] > 0 and abs(r["frac"] - r["achieved"] / r["peak"]) < 1e-9
    assert r["traffic"] > 0
    e = line["e2e"]
    assert e["value"] > 0 and e["unit"] == "particles/s"
    assert e["h2d_bytes_per_step"] >= n * 36 and e["d2h_bytes_per_step"] >= n * 36  # pos + mass + type + OldAcc; acc + pot + counts
    assert line["gpu_launches"] > 0
    assert set(line["clocks"]) >= {"sm_mhz", "sm_max_mhz", "reasons"}
    assert line["accuracy"]["rms_rel"] < 1e-3
