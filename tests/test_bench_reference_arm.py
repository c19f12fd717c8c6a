"""bench.py --impl reference on the CPU: one JSON line with the contract's keys for the default
workload (the oracle timed on the host cores), and an `unavailable` line for the workloads the
reference has no counterpart of."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def bench_line(*args):
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", *args],
                       capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    return json.loads(lines[0])


def test_reference_arm_line():
    d = bench_line("--steps", "1", "--warmup", "3", "--cpu-budget", "0.5")
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["unit"] == "solves/s" and d["value"] > 0 and d["higher_is_better"]
    assert d["config"]["workload"] == "medium_cluster_2000" and d["config"]["spheres"] == 2000
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


@pytest.mark.parametrize("args", [["--precision", "mixed"], ["--workload", "serving"], ["--workload", "multi_rhs"]])
def test_reference_arm_unavailable(args):
    d = bench_line(*args)
    assert d["impl"] == "reference" and d["unavailable"]
