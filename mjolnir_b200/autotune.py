"""Autotuner of the per-term launch shape and Verlet skin.

For every global term of an :class:`~mjolnir_b200.engine.Engine` it picks
  * the relative margin (list radius cutoff * (1 + margin), hence the cell size
    and the rebuild interval) from a candidate set, by timing whole MD steps --
    a thinner skin makes shorter lists but more frequent rebuilds;
  * the pair kernel's launch shape, by timing the kernel alone: the schedule
    (one particle per group of threads; warp-balanced over the lists of a
    warp's 32 particles, mixed form only; or one thread per particle reading
    its list in blocks with vector loads; the first and last optionally with
    each block's threads ordered by list length; or the first on lists stored
    slot by slot, each brought to L2 by one bulk prefetch), the threads per
    particle / list block (1, 2, 4, 8, 16, 32), the partners each thread
    requests per batch (1, 2, 4) and, in the mixed form, full or half lists;
  * the lanes per particle of the list build (4, 8, 16, 32), by timing whole
    steps at the chosen margin and shape.
In the mixed form none of the choices changes a result: the fixed-point force
sums do not depend on list order or length, and the lists are the same.  The engine's systems keep stepping
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


def tune(eng, terms=("exv", "dh", "lj"), margins=(0.1, 0.15, 0.2, 0.25, 0.3, 0.4, 0.5),
         tpps=(1, 2, 4, 8, 16, 32), unrolls=(1, 2, 4), schedules=(0, 1, 2, 3, 4, 5), steps: int = 200,
         warm: int = 300, log=None, build_lanes=(4, 8, 16, 32)) -> dict:
    """`warm` steps after each change before `steps` timed ones: a new margin
    rebuilds every list at once, and the rebuilds only spread out to their
    steady rate after a few rebuild intervals -- a short window after the
    change sees too few of them and favours wide margins.  Among margins
    within 1 % of the fastest the narrowest is kept (shorter lists, less
    memory)."""
    present = []
    for t in terms:
        try:
            eng.get_threads_per_particle(t)
            present.append(t)
        except Exception:
            continue
    choice = {}
    for t in present:
        cands = []
        for m in margins:
            eng.set_margin(t, m)
            shape = _tune_shape(eng, t, tpps, unrolls,
                                tuple(x for x in schedules if eng.precision == "mixed" or x != 1))
            _apply(eng, t, shape)
            eng.step(warm)
            ms = _time_steps(eng, steps)
            if log:
                log(f"autotune {t}: margin {m} schedule {shape[0]} tpp {shape[1]} unroll {shape[2]} "
                    f"half lists {shape[3]}: {ms:.4f} ms/step")
            cands.append((ms, m, shape))
        fastest = min(c[0] for c in cands)
        best = min((c for c in cands if c[0] <= 1.01 * fastest), key=lambda c: c[1])
        eng.set_margin(t, best[1])
        _apply(eng, t, best[2])
        # lanes per particle of the list build, at the chosen margin and shape
        lanes_best = None
        for lanes in build_lanes:
            eng.set_build_lanes(t, lanes)
            eng.step(warm)
            ms = _time_steps(eng, steps)
            if log:
                log(f"autotune {t}: list build with {lanes} lanes: {ms:.4f} ms/step")
            if lanes_best is None or ms < lanes_best[0]:
                lanes_best = (ms, lanes)
        eng.set_build_lanes(t, lanes_best[1])
        choice[t] = {"margin": best[1], "schedule": best[2][0], "threads_per_particle": best[2][1],
                     "unroll": best[2][2], "half_lists": best[2][3], "build_lanes": lanes_best[1],
                     "ms_per_step": min(best[0], lanes_best[0])}
    return choice


def _apply(eng, term, shape):
    if eng.precision == "mixed":
        eng.set_half_lists(term, shape[3])
    eng.set_pair_schedule(term, shape[0])
    eng.set_threads_per_particle(term, shape[1])
    eng.set_pair_unroll(term, shape[2])


def _tune_shape(eng, term, tpps, unrolls, schedules):
    best = None
    # half lists (mixed form): half the list words and pair evaluations, plus
    # integer atomics for the partners' shares -- a gain where few listed
    # pairs are inside the cutoff, a loss where most are
    for half in ((False, True) if eng.precision == "mixed" else (False,)):
        if eng.precision == "mixed":
            eng.set_half_lists(term, half)
        for sch in schedules:
            eng.set_pair_schedule(term, sch)
            for p in tpps:
                if sch in (2, 3) and p in (1, 32):
                    continue                  # the same launch as schedule 0
                if sch == 5 and p < 8:
                    continue                  # slot-major lists want whole 32-byte sectors per group
                eng.set_threads_per_particle(term, p)
                for u in (unrolls if sch not in (2, 3) else (1,)):
                    eng.set_pair_unroll(term, u)
                    ms = eng.time_kernel(term, reps=10)
                    if best is None or ms < best[0]:
                        best = (ms, (sch, p, u, half))
    return best[1]


def tune_shapes(eng, terms=("exv", "dh", "lj"), tpps=(1, 2, 4, 8, 16, 32), unrolls=(1, 2, 4),
                schedules=(0, 1, 2, 3, 4, 5)) -> dict:
    """Launch shape only (margins as committed): for a single large system,
    where the margin is fixed by the input."""
    out = {}
    for t in terms:
        try:
            eng.get_threads_per_particle(t)
        except Exception:
            continue
        shape = _tune_shape(eng, t, tpps, unrolls,
                            tuple(x for x in schedules if eng.precision == "mixed" or x != 1))
        _apply(eng, t, shape)
        out[t] = {"schedule": shape[0], "threads_per_particle": shape[1], "unroll": shape[2],
                  "half_lists": shape[3]}
    return out
