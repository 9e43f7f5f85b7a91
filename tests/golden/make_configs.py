"""Generates the configuration-size golden fixtures of tests/golden/ by running
the REFERENCE's own code (oracle/_ref/libmjolnir_ref.so, the unmodified Mjolnir
headers compiled by oracle/Makefile) on the benchmark's single-system
configurations at their own sizes:

  config1_lj4096      Lennard-Jones fluid, 4,096 particles, reduced density 0.8,
                      cutoff 2.5 sigma, margin 0.2 (= 0.5 sigma absolute),
                      PeriodicGridCellList, velocity Verlet dt = 0.005
  config2_melt10000   polymer melt, 50 chains x 200 beads in a 300 A sphere,
                      bonds / angles / dihedrals, ExcludedVolume, DebyeHuckel
                      (I = 0.1 M, 300 K), UnlimitedGridCellList (8^3 hashed
                      grid), velocity Verlet dt = 0.01
  config3_fluid32768  cut of the 1,048,576-bead fluid: 32,768 beads at
                      0.003 per cubic A (the same density, so the 42.3 A
                      DebyeHuckel cutoff and the cell widths are the real
                      ones), ExcludedVolume on all beads, DebyeHuckel on 30 %
                      (I = 0.15 M, 300 K), margins 0.3 / 0.1,
                      PeriodicGridCellList, velocity Verlet dt = 0.3

    MJOLNIR_REFERENCE_ROOT=<reference tree> python tests/golden/make_configs.py

The inputs are not stored: the tests rebuild each system with the same seeded
builders and check the SHA-256 of its coordinates against the stored one.
Stored per fixture:
  * the half neighbour list of each pair term (SpatialPartition::neighbors, the
    reference's CSR order) as its pair count and the SHA-256 of the int64
    (i, j) array -- lists are compared bit for bit through the hash;
  * the forces of every pair term and the total force (calc_force_and_energy),
    every term's energy and calc_energy;
  * a 1,000-step noise-free velocity-Verlet run (VelocityVerletIntegrator):
    the potential and kinetic energy every 100 steps and the final positions
    and velocities (for config 3, of its first 4,096 particles).
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from mjolnir_b200 import systems as S  # noqa: E402

VV_STEPS = 1000
VV_EVERY = 100
SUBSET = 4096          # particles of config 3 whose final VV state is stored


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def cases(synth=None):
    """{name: (SystemDesc, vv_dt, state subset or None)}; `synth` selects the
    library of the seeded builders (default the product library)."""
    out = {}
    d = S.lj_fluid(n=4096, density=0.8, margin=0.2, seed=1)
    out["config1_lj4096"] = (d, 0.005, None)
    d = S.polymer_melt(nchains=50, nbeads=200, radius=300.0, seed=2, synth=synth)
    out["config2_melt10000"] = (d, 0.01, None)
    d = S.bead_fluid(n=32768, density=0.003, seed=31, synth=synth)
    d.exv.margin = 0.3
    d.dh.margin = 0.1
    out["config3_fluid32768"] = (d, 0.3, SUBSET)
    return out


def kinetic(vel, mass):
    return 0.5 * float(np.sum(mass[:, None] * vel * vel))


def make(name, d, vv_dt, subset):
    ref = oracle.Reference(d)
    rec = {"pos_sha": np.array(sha(d.pos)), "vel_sha": np.array(sha(d.vel)), "n": np.array(d.n)}
    tot = np.zeros((d.n, 3))
    for t in ("bond", "angle", "dihedral", "exv", "dh", "lj"):
        try:
            f, e = ref.term_force(t)
        except RuntimeError:
            continue
        tot += f
        if t in ("exv", "dh", "lj"):
            rec[f"force_{t}"] = f
            pairs = ref.neighbors(t).astype(np.int64)
            rec[f"pairs_count_{t}"] = np.array(len(pairs))
            rec[f"pairs_sha_{t}"] = np.array(sha(pairs))
        rec[f"energy_{t}"] = np.array(e)
        rec[f"calc_energy_{t}"] = np.array(ref.term_energy(t))
    rec["force_total"] = tot
    ref.close()

    dv = d.copy()
    dv.integrator = "VelocityVerlet"
    dv.dt = vv_dt
    r = oracle.Reference(dv)
    r.initialize()
    pot, kin = [r.total_energy()], [kinetic(r.state()[1], d.mass)]
    for _ in range(VV_STEPS // VV_EVERY):
        r.run(VV_EVERY)
        pot.append(r.total_energy())
        kin.append(kinetic(r.state()[1], d.mass))
    p, v, _ = r.state()
    r.close()
    k = subset or d.n
    rec.update(vv_dt=np.array(vv_dt), vv_steps=np.array(VV_STEPS), vv_every=np.array(VV_EVERY),
               vv_potential=np.array(pot), vv_kinetic=np.array(kin), vv_pos=p[:k], vv_vel=v[:k])
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **rec)
    return rec


if __name__ == "__main__":
    import time
    oracle.build(os.environ.get("MJOLNIR_REFERENCE_ROOT"))
    for name, (d, dt, sub) in cases().items():
        t0 = time.time()
        rec = make(name, d, dt, sub)
        e = rec["vv_potential"] + rec["vv_kinetic"]
        print(name, d.n, {k: int(v) for k, v in rec.items() if k.startswith("pairs_count")},
              f"VV total energy {e[0]:.6g} -> {e[-1]:.6g}", f"{time.time() - t0:.1f} s")
