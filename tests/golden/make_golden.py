"""Generates the golden fixtures of tests/golden/ by running the REFERENCE's own
code (oracle/_ref/libmjolnir_ref.so, compiled from the unmodified Mjolnir
headers by oracle/Makefile) on small seeded systems.

    python tests/golden/make_golden.py        # needs the reference tree to build _ref

Each fixture holds the input coordinates and the reference's outputs:
half neighbour lists (SpatialPartition::neighbors), per-term forces and
energies of calc_force_and_energy, per-term calc_energy, and the final state
of a noise-free velocity-Verlet run.  The GPU box has no reference tree; the
tests read these files there.
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

TERMS = ["bond", "angle", "dihedral", "exv", "dh", "lj"]


def cases():
    out = {}
    # 1. polymer melt in unbounded space (EXV + DH + bonded), jittered so that
    #    every bonded term carries force
    d = S.polymer_melt(nchains=6, nbeads=60, radius=60.0, seed=5)
    d.pos = d.pos + np.random.default_rng(11).normal(0, 0.15, d.pos.shape)
    out["polymer_small"] = (d, 300)
    # 2. Lennard-Jones fluid, periodic (dims 4 x 4 x 4 cell grid)
    d = S.lj_fluid(n=1000, density=0.8, margin=0.2, seed=3)
    out["lj_small"] = (d, 200)
    # 3. periodic EXV + DH bead fluid, DH list radius > L/2 (3 x 3 x 3 grid)
    d = S.bead_fluid(n=1500, density=0.003, seed=7, dt=0.3)
    out["fluid_small"] = (d, 0)
    # 4. edge cases: ignore.molecule = "Self" (DH and EXV only between
    #    chains), per-bead radii, participants that skip particles.  (The
    #    reference requires participants in increasing order: NeighborList::
    #    add_list_for asserts it, core/NeighborList.hpp:215.)
    d = S.polymer_melt(nchains=4, nbeads=30, radius=40.0, seed=9)
    rng = np.random.default_rng(9)
    d.pos = d.pos + rng.normal(0, 0.1, d.pos.shape)
    d.exv.param0 = rng.uniform(1.5, 2.5, d.n)
    keep = np.sort(rng.choice(d.n, size=d.n - 17, replace=False))
    d.exv.idx = d.exv.idx[keep]
    d.exv.param0 = d.exv.param0[keep]
    d.ignore_molecule = "Self"
    out["edge_self_subset"] = (d, 100)
    return out


def make(name, d, vv_steps):
    ref = oracle.Reference(d)
    rec = {"pos": d.pos, "vel": d.vel}
    for t in TERMS:
        try:
            f, e = ref.term_force(t)
        except RuntimeError:
            continue
        rec[f"force_{t}"] = f
        rec[f"energy_{t}"] = np.array(e)
        rec[f"calc_energy_{t}"] = np.array(ref.term_energy(t))
        if t in ("exv", "dh", "lj"):
            rec[f"pairs_{t}"] = ref.neighbors(t).astype(np.int32)
    if vv_steps:
        dv = d.copy()
        dv.integrator = "VelocityVerlet"
        dv.dt = 0.002 if d.lj is not None else 0.005
        r = oracle.Reference(dv)
        r.initialize()
        r.run(vv_steps)
        p, v, f = r.state()
        rec["vv_steps"] = np.array(vv_steps)
        rec["vv_dt"] = np.array(dv.dt)
        rec["vv_pos"], rec["vv_vel"], rec["vv_force"] = p, v, f
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **rec)
    return rec


if __name__ == "__main__":
    oracle.build()
    for name, (d, vv) in cases().items():
        rec = make(name, d, vv)
        print(name, d.n, {k: v.shape for k, v in rec.items() if k.startswith("pairs")})
