"""Generates tests/golden/langevin_ref.npz: samples of the reference's own
Langevin dynamics (BAOABLangevinIntegrator, core/BAOABLangevinIntegrator.hpp
:170-240, with its mt19937 + std::normal_distribution noise,
core/RandomNumberGenerator.hpp:77-78), run through oracle/_ref from the
unmodified reference headers, for the distribution test of the GPU's Philox
runs (tests/test_gpu_langevin_reference.py).

  lj4096     the 4,096-particle Lennard-Jones fluid at kT = 1 (reduced density
             0.8, cutoff 2.5, margin 0.2, gamma 1, dt 0.005): 1,000 steps to
             settle from the lattice, then a sample every 50 steps for 10,000
             steps (200 samples, 2.5 time units apart at the thermostat's
             relaxation time of 1)
  melt1000   a polymer melt of 20 chains x 50 beads (the melt's composition:
             bonds, angles, dihedrals, ExcludedVolume, DebyeHuckel) at 300 K,
             gamma 1, dt 0.01: 2,000 steps to settle, then a sample every 50
             steps for 20,000 steps (400 samples)

Each sample holds the kinetic temperature (2 KE / (3 N kB)) and every term's
potential energy (calc_energy).

    MJOLNIR_REFERENCE_ROOT=<reference tree> python tests/golden/make_langevin.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from mjolnir_b200 import systems as S  # noqa: E402

TERMS = ("bond", "angle", "dihedral", "exv", "dh", "lj")


def cases():
    """{name: (SystemDesc, settle steps, sample every, samples)}"""
    lj = S.lj_fluid(n=4096, density=0.8, margin=0.2, seed=1)
    melt = S.polymer_melt(nchains=20, nbeads=50, radius=300.0 * (1000 / 10000) ** (1 / 3), seed=21)
    return {"lj4096": (lj, 1000, 50, 200), "melt1000": (melt, 2000, 50, 400)}


def terms_of(d):
    out = []
    if d.bonds is not None:
        out.append("bond")
    if d.angles is not None:
        out.append("angle")
    if d.dihedrals is not None:
        out.append("dihedral")
    out += [t for t, p in (("exv", d.exv), ("dh", d.dh), ("lj", d.lj)) if p is not None]
    return out


def kinetic_temperature(vel, mass):
    return float(np.sum(mass[:, None] * vel * vel)) / (3 * len(mass) * S.KB_KCAL)


def sample_reference(d, settle, every, count):
    r = oracle.Reference(d)
    r.initialize()
    r.run(settle)
    terms = terms_of(d)
    out = {"T": []}
    out.update({t: [] for t in terms})
    for _ in range(count):
        r.run(every)
        out["T"].append(kinetic_temperature(r.state()[1], d.mass))
        for t in terms:
            out[t].append(r.term_energy(t))
    r.close()
    return {k: np.array(v) for k, v in out.items()}


if __name__ == "__main__":
    oracle.build(os.environ.get("MJOLNIR_REFERENCE_ROOT"))
    rec = {}
    for name, (d, settle, every, count) in cases().items():
        s = sample_reference(d, settle, every, count)
        for k, v in s.items():
            rec[f"{name}_{k}"] = v
            print(name, k, f"mean {v.mean():.6g} std {v.std():.4g}")
    np.savez_compressed(os.path.join(HERE, "langevin_ref.npz"), **rec)
