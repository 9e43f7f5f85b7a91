"""Langevin runs on the GPU against the reference's own Langevin runs.

The GPU's BAOAB draws its noise from a counter-based Philox stream, the
reference's from mt19937 (core/RandomNumberGenerator.hpp:77-78), so the two
trajectories differ from the first step and are compared as distributions:
kinetic temperature and every term's potential energy sampled along the
same schedule as the reference's runs in tests/golden/langevin_ref.npz
(tests/golden/make_langevin.py: the 4,096-particle Lennard-Jones fluid at
kT = 1 and a 1,000-bead polymer melt at 300 K), both forms, by the block-mean,
width and Kolmogorov-Smirnov criteria of tests/langevin_stats.py.  A run at a
temperature 2 % off must fail the same comparison.
"""
import numpy as np
import pytest

from langevin_stats import compare
from mjolnir_b200.engine import Engine
from test_oracle_langevin_reference import FAST, MOD, REF

pytestmark = pytest.mark.gpu


def sample_gpu(d, precision, settle, every, count):
    e = Engine(precision)
    sid = e.add_system(d)
    e.commit()
    e.step(settle)
    terms = MOD.terms_of(d)
    s = {k: [] for k in ("T", *terms)}
    for _ in range(count):
        e.step(every)
        _p, v, _f = e.state(sid)
        s["T"].append(MOD.kinetic_temperature(v, d.mass))
        E = e.energies(sid)
        for t in terms:
            s[t].append(E[t])
    e.close()
    return {k: np.array(v) for k, v in s.items()}


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", sorted(MOD.cases()))
def test_gpu_langevin_matches_reference_distributions(name, precision):
    d, settle, every, count = MOD.cases()[name]
    s = sample_gpu(d, precision, settle, every, count)
    bad = {}
    for k, v in s.items():
        ok, rep = compare(v, REF[f"{name}_{k}"], fast=k in FAST[name])
        if not ok:
            bad[k] = rep
    assert not bad, (name, precision, bad)


def test_comparison_detects_a_temperature_error():
    d, settle, every, count = MOD.cases()["lj4096"]
    d = d.copy()
    d.temperature *= 1.02
    s = sample_gpu(d, "fp64", settle, every, count)
    ok, rep = compare(s["T"], REF["lj4096_T"], fast=True)
    assert not ok, rep
