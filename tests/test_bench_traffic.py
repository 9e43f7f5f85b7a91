"""bench.py's roofline traffic: the DRAM bytes of the committed ncu captures
(profiles/ncu_traffic.json) are reported only for the kernel, schedule and
list form they were captured with, scaled by the launch's slots."""
import importlib.util
import json
import os

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("bench_module", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="module")
def records():
    with open(os.path.join(ROOT, "profiles", "ncu_traffic.json")) as f:
        return json.load(f)


def test_every_record_names_its_capture(records):
    for key, r in records.items():
        assert {"kernel", "schedule", "half_lists", "slots", "dram_read_bytes", "dram_write_bytes",
                "workload"} <= set(r), key
        assert r["slots"] > 0 and r["dram_read_bytes"] > 0 and r["dram_write_bytes"] >= 0


def test_matching_capture_is_scaled_by_slots(bench, records):
    r = records["batch256_exv"]
    per_slot = (r["dram_read_bytes"] + r["dram_write_bytes"]) / r["slots"]
    b, src = bench.ncu_traffic("batch256_exv", r["schedule"], 2 * r["slots"], r["half_lists"])
    assert b == pytest.approx(2 * per_slot * r["slots"])
    assert "ncu" in src and r["kernel"] in src


def test_other_schedule_list_form_or_kernel_reports_none(bench, records):
    r = records["batch256_exv"]
    b, why = bench.ncu_traffic("batch256_exv", r["schedule"] + 1, r["slots"], r["half_lists"])
    assert b is None and "schedule" in why
    b, why = bench.ncu_traffic("batch256_exv", r["schedule"], r["slots"], not r["half_lists"])
    assert b is None and "lists" in why
    b, why = bench.ncu_traffic("no_such_kernel", 0, 1, False)
    assert b is None


def test_clock_summary_keeps_the_timed_span(bench):
    """The clock summary uses only the samples taken between mark_start and
    mark_end, and reports any throttle reason seen there."""
    c = bench.ClockSampler(0)
    row = "0, {sm}, 1965, 700.0, 0x0, Not Active, Not Active, {therm}, Not Active"
    c.lines = [row.format(sm=1000, therm="Active")]                     # warm-up, throttled
    c.span[0] = len(c.lines)
    c.lines += [row.format(sm=1965, therm="Not Active") for _ in range(5)]
    c.span[1] = len(c.lines)
    c.lines += [row.format(sm=900, therm="Active")]                     # after the timed steps
    s = c.summary()
    assert s == {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": [], "samples": 5}
    c.lines[2] = row.format(sm=1500, therm="Active")
    assert c.summary()["reasons"] == ["sw_thermal_slowdown"]
