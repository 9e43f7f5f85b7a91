"""The reference arm of bench.py (`--impl reference`), run for real on a tiny
batch: the reference's own OpenMP code times the same metric on the same
workload config and prints the same JSON line, marked as the reference, with
no host-device traffic, and without loading the product library."""
import json
import os
import subprocess
import sys

import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# runs bench.py's main in this process, then reports whether the product
# library was mapped into it
RUNNER = """
import runpy, sys
sys.argv = ["bench.py", "--impl", "reference", "--nsys", "2", "--steps", "1", "--warmup", "1"]
runpy.run_path("bench.py", run_name="__main__")
maps = open("/proc/self/maps").read()
print("PRODUCT_LIBRARY_LOADED" if "libmjolnir_b200" in maps else "PRODUCT_LIBRARY_ABSENT")
"""


@pytest.mark.skipif(not oracle.reference_available(), reason="reference driver not built (no reference tree)")
def test_reference_arm_prints_the_contract_line():
    out = subprocess.run([sys.executable, "-c", RUNNER], capture_output=True, text=True, timeout=600,
                         cwd=ROOT, check=True).stdout
    assert "PRODUCT_LIBRARY_ABSENT" in out, "the reference arm loaded libmjolnir_b200.so"
    line = json.loads([x for x in out.splitlines() if x.startswith("{")][-1])
    assert line["impl"] == "reference"
    assert line["metric"] == "particle-steps/s (batched polymer systems)" and line["unit"] == "particle-steps/s"
    assert line["value"] > 0 and line["higher_is_better"] is True
    assert line["steps"] == 1 and line["warmup"] == 1 and line["n_gpus"] == 1
    assert line["e2e"] == {"value": line["value"], "unit": "particle-steps/s",
                           "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    cb = line["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["value"] == line["value"] and cb["cores"] >= 1
    # the same config dict as the B200 arm's line, built from the same systems
    sys.path.insert(0, ROOT)
    import bench
    assert line["config"] == bench.workload_config(bench.build_batch(2))
    assert line["config"]["md_steps_per_bench_step"] == bench.CHUNK
