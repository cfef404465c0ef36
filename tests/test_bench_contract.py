"""The bench's reference arm on the CPU: the JSON line a driver parses.

The reference arm runs the reference's own OpenMP build (oracle/_ref, built
from the reference sources by oracle/Makefile) on the host cores, so it needs
no GPU; a small mesh keeps it to a second or two.
"""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "phg_dump_omp")

pytestmark = pytest.mark.skipif(not os.path.exists(REF_BIN), reason="reference build absent (oracle/_ref)")


def run_bench(env_extra=None):
    env = dict(os.environ)
    env.update(env_extra or {})
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--m", "6",
                          "--steps", "2", "--warmup", "1"], capture_output=True, text=True, env=env, timeout=600,
                         cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    return [line for line in out.stdout.splitlines() if line.startswith("{")]


def test_reference_arm_prints_one_contract_line():
    lines = run_bench()
    assert len(lines) == 1
    rec = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in rec, key
    assert rec["impl"] == "reference"
    assert rec["steps"] == 2 and rec["warmup"] == 1 and rec["n_gpus"] == 1
    assert rec["unit"] == "ms" and rec["higher_is_better"] is False
    assert rec["value"] > 0 and rec["value"] == rec["ms_per_step"]
    cb = rec["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == rec["value"] and cb["sample"]
    e2e = rec["e2e"]
    assert e2e["value"] == rec["value"] and e2e["unit"] == rec["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
    assert "workload" in rec["config"] and rec["config"]["dofs"] > 0
    # the reference's own PCG reaches the stopping rule in a positive number of iterations
    assert rec["reference_nits"] > 0

