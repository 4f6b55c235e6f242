"""bench.py end to end on the GPU at small sizes: both workloads print one JSON
line with the contract's keys (the same code paths as a full run)."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

pytestmark = pytest.mark.gpu

KEYS = ["metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
        "vs_baseline", "dtype", "data", "config", "e2e", "roofline", "clocks", "gpu_launches", "cpu_baseline"]


@pytest.mark.parametrize("workload,extra", [("learned_band", ["--windows", "40", "--reads-per-window", "6"]),
                                            ("polishing", ["--windows", "300"])])
def test_bench_line(workload, extra):
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--workload", workload, "--steps", "1", "--warmup", "1",
           "--cpu-seconds", "3", "--plain-windows", "1"] + extra
    res = subprocess.run(cmd, capture_output=True, text=True, timeout=900, cwd=ROOT)
    assert res.returncode == 0, res.stderr[-3000:]
    line = json.loads(res.stdout.strip().splitlines()[-1])
    for k in KEYS:
        assert k in line, k
    assert line["value"] > 0 and line["e2e"]["value"] > 0
    assert line["roofline"]["bound"] == "int_alu" and 0 < line["roofline"]["frac"] < 2
    assert line["parity_sample"]["identical_consensus"] == line["parity_sample"]["windows"]
