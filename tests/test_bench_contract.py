"""bench.py's reference arm runs on the host cores, so its JSON contract is
checked here without a GPU: one line with the metric, the CPU baseline
description and the end-to-end figure; the time-to-steady workload reports
itself unavailable on the CPU with a reason."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(*args):
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], capture_output=True, text=True,
                         cwd=ROOT, timeout=600, env={**os.environ, "OMP_NUM_THREADS": "2"})
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out.stdout
    return json.loads(lines[0])


@pytest.mark.parametrize("workload", ["cavity2d_128", "batch256"])
def test_reference_arm_line(workload):
    d = _run("--impl", "reference", "--workload", workload, "--steps", "2", "--warmup", "3")
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference" and d["metric"] == "MLUPS" and d["value"] > 0
    assert d["steps"] == 2 and d["warmup"] == 3 and d["higher_is_better"] is True
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"]["value"] == d["value"] and d["e2e"]["h2d_bytes_per_step"] == 0
    assert d["config"]["workload"] == workload


def test_reference_arm_of_the_steady_workload_is_unavailable():
    d = _run("--impl", "reference", "--workload", "steady", "--steps", "1", "--warmup", "3")
    assert d["impl"] == "reference" and "unavailable" in d and d["unavailable"]
