"""bench.py's output line: one JSON object with the keys the benchmark
protocol names (metric, value, unit, timing, config, roofline, e2e, clocks,
launch count), measured on the headline workload with the minimum warm-up.
"""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_quick_bench_line_has_the_protocol_keys():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--quick",
                        "--no-cpu-baseline", "--steps", "3", "--warmup", "3"],
                       cwd=ROOT, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True,
                       timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
              "roofline", "e2e", "clocks", "gpu_launches"):
        assert k in d, k
    assert d["n_gpus"] == 1 and d["steps"] == 3 and d["warmup"] == 3
    assert d["higher_is_better"] is True and d["value"] > 0
    assert "workload" in d["config"]
    roof = d["roofline"]
    for k in ("bound", "achieved", "peak", "unit", "frac", "traffic"):
        assert k in roof, k
    assert roof["bound"] == "hbm" and 0 < roof["frac"] < 2
    assert abs(roof["frac"] - roof["achieved"] / roof["peak"]) < 1e-9
    # the three tile passes of the complex64 3D step, each timed
    assert [p[0].split()[0] for p in roof["passes_us"]] == ["forward", "z", "inverse"]
    e2e = d["e2e"]
    assert e2e["unit"] == d["unit"] and 0 < e2e["value"] < d["value"]
    assert e2e["h2d_bytes_per_step"] == 256 ** 3 * 16
    assert e2e["d2h_bytes_per_step"] >= 256 ** 3 * 16
    assert d["gpu_launches"] >= 3 * 100 * 3  # three passes per time step
    assert d["plain_fp64"]["fused_fp32_over_plain_fp64"] > 1
