"""Simulated annealing: a linear temperature schedule over the Langevin
integrator (core/SimulatedAnnealingSimulator.hpp).

The temperature starts at ``first`` (the reference sets the system's
temperature attribute to ``current(0)`` before the force field and the
integrator are initialised, :108-119) and, every ``each_step`` steps, becomes
``current(step * (1 / total_step))`` with ``current(r) = first (1 - r) +
last r`` (:28-32, :144-154); only the integrator's noise follows it, the
DebyeHuckel screening keeps the initial temperature, as in the reference.
Every system of the engine that is listed is annealed together, each on its
own schedule.
"""
from __future__ import annotations


def current(first: float, last: float, ratio: float) -> float:
    """LinearScheduler::current (core/SimulatedAnnealingSimulator.hpp:28-32)."""
    return first * (1.0 - ratio) + last * ratio


def run(engine, schedules: dict, total_step: int, each_step: int, on_step=None):
    """Advances the engine `total_step` steps, updating the temperature of
    every system in `schedules` ({sid: (first, last)}) each `each_step` steps.
    The systems must have been committed with temperature `first`.
    `on_step(step)` is called after every temperature update."""
    if each_step <= 0 or total_step < 0:
        raise ValueError("each_step must be positive and total_step non-negative")
    r_total = 1.0 / total_step if total_step else 0.0
    done = 0
    while done < total_step:
        k = min(each_step - done % each_step, total_step - done)
        engine.step(k)
        done += k
        if done % each_step == 0:
            for sid, (first, last) in schedules.items():
                engine.set_temperature(sid, current(first, last, done * r_total))
            if on_step:
                on_step(done)
    return done
