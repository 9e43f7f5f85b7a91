"""The reference arm of bench.py (`--impl reference`), run for real on a tiny
batch: the reference's own OpenMP code times the same metric and prints the
same JSON line, marked as the reference, with no host-device traffic."""
import json
import os
import subprocess
import sys

import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(not oracle.reference_available(), reason="reference driver not built (no reference tree)")
def test_reference_arm_prints_the_contract_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--nsys", "2",
                          "--steps", "1", "--warmup", "1"], capture_output=True, text=True, timeout=300,
                         cwd=ROOT, check=True).stdout
    line = json.loads([x for x in out.splitlines() if x.startswith("{")][-1])
    assert line["impl"] == "reference"
    assert line["metric"] == "particle-steps/s (batched polymer systems)" and line["unit"] == "particle-steps/s"
    assert line["value"] > 0 and line["higher_is_better"] is True
    assert line["steps"] == 1 and line["warmup"] == 1 and line["n_gpus"] == 1
    assert line["e2e"] == {"value": line["value"], "unit": "particle-steps/s",
                           "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    cb = line["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["value"] == line["value"] and cb["cores"] >= 1
    assert line["config"]["systems"] == 2
