"""Autotuner of the per-term launch shape and Verlet skin.

For every global term of an :class:`~mjolnir_b200.engine.Engine` it picks
  * the relative margin (list radius cutoff * (1 + margin), hence the cell size
    and the rebuild interval) from a candidate set, by timing whole MD steps --
    a thinner skin makes shorter lists but more frequent rebuilds;
  * the number of threads that cooperate on one particle's list in the pair
    kernel (1, 2, 4, 8, 16), by timing the pair kernel alone.
In the mixed form neither choice changes a result: the fixed-point force sums
do not depend on list order or length.  The engine's systems keep stepping
while the tuner measures (the tuning run is part of the warm-up).
"""
from __future__ import annotations

import torch


def _time_steps(eng, nsteps: int) -> float:
    stream = torch.cuda.ExternalStream(eng.stream_handle())
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(stream)
    eng.step(nsteps)
    b.record(stream)
    b.synchronize()
    return a.elapsed_time(b) / nsteps


def tune(eng, terms=("exv", "dh", "lj"), margins=(0.1, 0.2, 0.3, 0.5),
         tpps=(1, 2, 4, 8, 16), steps: int = 60, warm: int = 20, log=None) -> dict:
    present = []
    for t in terms:
        try:
            eng.get_threads_per_particle(t)
            present.append(t)
        except Exception:
            continue
    choice = {}
    for t in present:
        best = None
        for m in margins:
            eng.set_margin(t, m)
            best_tpp = _tune_tpp(eng, t, tpps)
            eng.set_threads_per_particle(t, best_tpp)
            eng.step(warm)
            ms = _time_steps(eng, steps)
            if log:
                log(f"autotune {t}: margin {m} tpp {best_tpp}: {ms:.4f} ms/step")
            if best is None or ms < best[0]:
                best = (ms, m, best_tpp)
        eng.set_margin(t, best[1])
        eng.set_threads_per_particle(t, best[2])
        choice[t] = {"margin": best[1], "threads_per_particle": best[2], "ms_per_step": best[0]}
    return choice


def _tune_tpp(eng, term, tpps) -> int:
    best = None
    for p in tpps:
        eng.set_threads_per_particle(term, p)
        ms = eng.time_kernel(term, reps=10)
        if best is None or ms < best[0]:
            best = (ms, p)
    return best[1]
