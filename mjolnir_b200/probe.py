"""Fixed workloads for profiling the kernels (ncu, CUDA-event timings).

    python -m mjolnir_b200.probe batch            # the 256-system polymer batch, mixed form
    python -m mjolnir_b200.probe fluid [--precision fp64] [--n 1048576]
    python -m mjolnir_b200.probe lj [--precision fp64]   # the 4,096-particle Lennard-Jones fluid

`batch` builds the benchmark's 256 independent polymer melts with the launch
shapes the autotuner picks for them (ExcludedVolume: margin 0.25, half lists,
block-vector schedule with length-sorted threads, 2-word blocks; DebyeHuckel:
margin 0.1, full lists, 2 threads per slot with length-sorted groups), steps
300 MD steps, then times
each kernel alone.  `fluid` builds the periodic EXV + DebyeHuckel bead fluid
(0.003 per cubic A, margins 0.3 / 0.1) with its tuned shapes (ExcludedVolume:
block-vector schedule, 2-word blocks; DebyeHuckel: slot-major lists, 8
threads per slot).  Each timing runs inside an NVTX range
named probe_<term> (probe_step: 2 MD steps; probe_steps20: 20 MD steps) so that
a profiler can select those launches.  Prints one JSON object.
"""
from __future__ import annotations

import argparse
import json

import torch

from . import systems as S
from .engine import Engine

BATCH_SHAPES = {"exv": dict(margin=0.25, schedule=3, tpp=2, unroll=1, lanes=8, half=True),
                "dh": dict(margin=0.1, schedule=4, tpp=2, unroll=1, lanes=16)}
FLUID_SHAPES = {"exv": dict(schedule=2, tpp=2, unroll=1),
                "dh": dict(schedule=5, tpp=8, unroll=1)}


def _shape(e, shapes):
    for t, c in shapes.items():
        if "margin" in c:
            e.set_margin(t, c["margin"])
        if e.precision == "mixed":
            e.set_half_lists(t, c.get("half", False))
        e.set_pair_schedule(t, c["schedule"])
        e.set_threads_per_particle(t, c["tpp"])
        e.set_pair_unroll(t, c["unroll"])
        if "lanes" in c:
            e.set_build_lanes(t, c["lanes"])


def _steps_ms(e, n):
    st = torch.cuda.ExternalStream(e.stream_handle())
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(st)
    e.step(n)
    b.record(st)
    b.synchronize()
    return a.elapsed_time(b) / n


def _ranges(e, out, terms):
    for t in terms:
        torch.cuda.nvtx.range_push(f"probe_{t}")
        out[f"{t}_ms"] = e.time_kernel(t, reps=10)
        torch.cuda.nvtx.range_pop()
        if t in ("exv", "dh", "lj"):
            out[f"{t}_pairs_in_cutoff"] = e.pair_count(-1, t)
    for name, n in (("probe_step", 2), ("probe_steps20", 20)):
        torch.cuda.nvtx.range_push(name)
        e.step(n)
        e.synchronize()
        torch.cuda.nvtx.range_pop()


def batch(device: int = 0) -> dict:
    descs = S.polymer_batch(nsys=256, seed=4)
    e = Engine("mixed", device=device)
    for d in descs:
        e.add_system(d)
    e.commit()
    _shape(e, BATCH_SHAPES)
    e.step(100)
    out = {"workload": "256 polymer melts, mixed form", "particles": sum(d.n for d in descs)}
    out["ms_per_md_step"] = _steps_ms(e, 200)
    _ranges(e, out, ("exv", "dh", "bond", "angle", "dihedral"))
    e.close()
    return out


def fluid(precision: str = "mixed", n: int = 1 << 20, device: int = 0) -> dict:
    d = S.bead_fluid(n=n, density=0.003, seed=3)
    d.exv.margin = 0.3
    d.dh.margin = 0.1
    e = Engine(precision, device=device)
    e.add_system(d)
    e.commit()
    _shape(e, FLUID_SHAPES)
    e.step(20)
    out = {"workload": f"{n}-bead periodic EXV + DebyeHuckel fluid, {precision} form", "particles": n}
    out["ms_per_md_step"] = _steps_ms(e, 100)
    _ranges(e, out, ("exv", "dh"))
    e.close()
    return out


def lj(precision: str = "mixed", device: int = 0) -> dict:
    d = S.lj_fluid(n=4096, density=0.8, margin=0.2, seed=1)
    e = Engine(precision, device=device)
    e.add_system(d)
    e.commit()
    e.step(200)
    out = {"workload": f"4,096-particle Lennard-Jones fluid, {precision} form", "particles": d.n}
    out["ms_per_md_step"] = _steps_ms(e, 2000)
    out["rebuilds"] = e.rebuild_count(0, "lj")
    _ranges(e, out, ("lj",))
    e.close()
    return out


def main():
    ap = argparse.ArgumentParser(prog="python -m mjolnir_b200.probe")
    ap.add_argument("workload", choices=["batch", "fluid", "lj"])
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--n", type=int, default=1 << 20)
    a = ap.parse_args()
    res = batch() if a.workload == "batch" else (fluid(a.precision, a.n) if a.workload == "fluid"
                                                 else lj(a.precision))
    print(json.dumps(res))


if __name__ == "__main__":
    main()
