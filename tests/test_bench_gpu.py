"""bench.py end to end on a small workload: every leg of the default run
(device timing, end-to-end through the C ABI with host films, time to
relMSE for the plain and cached forms, the cache kernels' roofline, the
batched requests, the CPU baseline) runs and the JSON line carries the keys
the measurement contract names."""

import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.gpu
def test_bench_line_cornell():
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--workload", "cornell", "--steps", "2", "--warmup", "3",
           "--cpu-seconds", "1"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=900, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-3000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout[-2000:]
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "roofline", "cpu_baseline", "e2e", "gpu_launches", "clocks",
              "time_to_relmse", "cache_roofline", "batched"):
        assert k in d, k
    assert d["value"] > 0 and d["e2e"]["value"] > 0 and d["gpu_launches"] > 0
    assert d["config"]["workload"] == "cornell"
    assert d["roofline"]["bound"] == "hbm" and d["roofline"]["achieved"] > 0
    assert d["cpu_baseline"]["value"] > 0 and d["cpu_baseline"]["cores"] >= 1
    t = d["time_to_relmse"]
    assert t["cached"]["settings"]["warmup_calls"] >= 1 and t["plain"]["curve"] and t["cached"]["curve"]
    assert d["batched"]["mpaths_per_s"] > 0
