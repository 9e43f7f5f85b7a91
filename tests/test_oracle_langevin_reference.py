"""The oracle's BAOAB (the C restatement, driven by the Philox stream the GPU
uses) against the reference's own BAOAB runs with their mt19937 noise
(tests/golden/langevin_ref.npz, tests/golden/make_langevin.py): kinetic
temperature and per-term potential energy distributions agree
(tests/langevin_stats.py).  This pins the statistical comparison that
tests/test_gpu_langevin_reference.py applies to the GPU.  CPU only."""
import importlib.util
import os

import numpy as np
import pytest

import oracle
from langevin_stats import compare

HERE = os.path.dirname(os.path.abspath(__file__))


def load_cases():
    spec = importlib.util.spec_from_file_location("make_langevin", os.path.join(HERE, "golden", "make_langevin.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod, dict(np.load(os.path.join(HERE, "golden", "langevin_ref.npz")))


MOD, REF = load_cases()
# observables sampled further apart than their relaxation time
FAST = {"lj4096": ("T", "lj"), "melt1000": ("T", "bond", "angle")}


@pytest.mark.parametrize("name", sorted(MOD.cases()))
def test_oracle_philox_matches_reference_distributions(name):
    d, settle, every, count = MOD.cases()[name]
    o = oracle.Oracle(d)
    o.init_dynamics()
    o.run(settle)
    terms = MOD.terms_of(d)
    s = {k: [] for k in ("T", *terms)}
    for _ in range(count):
        o.run(every)
        p, v, _ = o.state()
        s["T"].append(MOD.kinetic_temperature(v, d.mass))
        for t in terms:
            s[t].append(o.term_energy(t, p))
    o.close()
    bad = {}
    for k, v in s.items():
        ok, rep = compare(np.array(v), REF[f"{name}_{k}"], fast=k in FAST[name])
        if not ok:
            bad[k] = rep
    assert not bad, bad
