"""Precision at scale: a mixed-form trajectory (FP32 pair math, 64-bit
fixed-point force sums, FP64 state) checked against the FP64 form on its own
coordinates.

    python -m mjolnir_b200.precision [--n 1048576] [--steps 20000] [--every 1000]

The system is the periodic bead fluid (ExcludedVolume on every bead,
DebyeHuckel on 30 % of them with zero net charge, I = 0.15 M, T = 300 K, BAOAB
dt = 0.3).  Every ``every`` steps the mixed engine's coordinates are loaded
into an FP64 engine holding the same system, and per term the forces (relative
RMS error, sqrt(sum |dF|^2 / sum |F|^2)) and energies (relative error) of the
two forms are compared.  The FP64 form itself matches the CPU restatement of
the reference to 1e-12 (tests/test_gpu_parity.py), so it stands in for the
reference's double-precision path on coordinates no CPU run could reach in
reasonable time.  Prints one JSON object.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import systems as S
from .engine import Engine

TERMS = ("exv", "dh")


def _rel_rms(a: np.ndarray, b: np.ndarray) -> float:
    den = float(np.sum(b * b))
    return float(np.sqrt(np.sum((a - b) ** 2) / den)) if den > 0 else 0.0


def compare(mixed: Engine, fp64: Engine, sid: int) -> dict:
    """Loads the mixed engine's coordinates into the FP64 engine and compares
    forces and energies term by term."""
    pos, vel, _ = mixed.state(sid)
    fp64.set_state(sid, pos, vel)
    out = {}
    f_tot_m = np.zeros_like(pos)
    f_tot_d = np.zeros_like(pos)
    for t in TERMS:
        fm, em = mixed.term_force(sid, t)
        fd, ed = fp64.term_force(sid, t)
        f_tot_m += fm
        f_tot_d += fd
        out[t] = {"force_rel_rms": _rel_rms(fm, fd),
                  "energy_rel": abs(em - ed) / abs(ed) if ed != 0 else abs(em - ed),
                  "energy_fp64": ed}
    out["total_force_rel_rms"] = _rel_rms(f_tot_m, f_tot_d)
    return out


def run(n: int = 1 << 20, steps: int = 20000, every: int = 1000, seed: int = 3,
        margin: float = 0.2, device: int = 0, log=None) -> dict:
    desc = S.bead_fluid(n=n, density=0.003, seed=seed, margin=margin)
    mixed = Engine("mixed", device=device)
    sid = mixed.add_system(desc)
    mixed.commit()
    fp64 = Engine("fp64", device=device)
    assert fp64.add_system(desc) == sid
    fp64.commit()
    frames = []
    t0 = time.perf_counter()
    done = 0
    while True:
        frame = {"step": done, **compare(mixed, fp64, sid)}
        frames.append(frame)
        if log:
            log(json.dumps(frame))
        if done >= steps:
            break
        k = min(every, steps - done)
        mixed.step(k)
        done += k
    wall = time.perf_counter() - t0
    worst = {t: max(f[t]["force_rel_rms"] for f in frames) for t in TERMS}
    worst_e = {t: max(f[t]["energy_rel"] for f in frames) for t in TERMS}
    res = {"beads": n, "steps": steps, "every": every, "margin": margin, "seed": seed,
           "worst_force_rel_rms": worst, "worst_energy_rel": worst_e,
           "worst_total_force_rel_rms": max(f["total_force_rel_rms"] for f in frames),
           "rebuilds": {t: mixed.rebuild_count(sid, t) for t in TERMS},
           "wall_s": wall, "frames": frames}
    mixed.close()
    fp64.close()
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=1 << 20)
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--every", type=int, default=1000)
    ap.add_argument("--seed", type=int, default=3)
    ap.add_argument("--margin", type=float, default=0.2)
    a = ap.parse_args()
    import sys
    res = run(a.n, a.steps, a.every, a.seed, a.margin, log=lambda m: print(m, file=sys.stderr))
    print(json.dumps(res))


if __name__ == "__main__":
    main()
