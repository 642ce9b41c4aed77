"""The reference arm of bench.py keeps the one-JSON-line contract (CPU only:
it times the reference library built from its sources on the host cores)."""
import json
import os
import subprocess
import sys

import pytest

from oracle import ref

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(*args):
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], cwd=ROOT,
                       capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, p.stdout[-2000:]
    return json.loads(lines[0])


@pytest.mark.skipif(not ref.available(), reason="reference library not built")
def test_reference_arm_prints_one_contract_line():
    line = _run("--impl", "reference", "--workload", "laplace128", "--steps", "2", "--warmup", "1",
                "--cpu-sample", "16")
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference"
    assert line["steps"] == 2 and line["warmup"] == 1 and line["n_gpus"] == 1
    assert line["value"] > 0 and line["higher_is_better"] is True
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert "workload" in line["config"]


@pytest.mark.skipif(not ref.available(), reason="reference library not built")
def test_reference_arm_of_batched_workload():
    line = _run("--impl", "reference", "--workload", "batched512", "--steps", "1", "--warmup", "1")
    assert line["impl"] == "reference" and line["unit"] == "problems/s" and line["value"] > 0
    assert line["cpu_baseline"]["value"] == line["value"]
    assert "6 problems" in line["cpu_baseline"]["sample"]


@pytest.mark.skipif(not ref.available(), reason="reference library not built")
def test_reference_arm_of_learned_seed_workload_needs_no_gpu():
    line = _run("--impl", "reference", "--workload", "wells256", "--steps", "1", "--warmup", "1")
    assert line["impl"] == "reference" and line["unit"] == "solves/s" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "reference"
