"""Generates tests/golden/integrators.npz by running the REFERENCE's own
integrators (oracle/_ref/libmjolnir_ref.so, compiled from the unmodified
Mjolnir headers by oracle/Makefile) where their noise vanishes:
BAOABLangevin, UnderdampedLangevin, G-JFLangevin and g-BAOABLangevin (no
constraints) on a small polymer melt, (1) without friction, with every term
of the path, and (2) with friction at temperature 0 (per-particle frictions,
no DebyeHuckel term, whose Debye length needs a temperature), which exercises
every friction factor of each scheme.  The final positions and velocities let
the GPU box, which has no reference tree, compare each integrator's
trajectory with the reference's.

    python tests/golden/make_integrators.py      # needs the reference tree to build _ref
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

INTEGRATORS = ["BAOAB", "UnderdampedLangevin", "G-JFLangevin", "g-BAOABLangevin"]
STEPS = 400


def system(integrator, cold_friction=False):
    d = S.polymer_melt(nchains=5, nbeads=40, radius=45.0, seed=17)
    d.pos = d.pos + np.random.default_rng(17).normal(0, 0.1, d.pos.shape)
    d.integrator = integrator
    d.gamma = np.zeros(d.n)
    d.dt = 0.005
    if cold_friction:
        d.gamma = np.random.default_rng(18).uniform(0.2, 2.0, d.n)   # G-JFLangevin: alpha
        d.temperature = 0.0
        d.dh = None
    return d


def main():
    if not oracle.reference_available():
        raise SystemExit("the reference driver is not built")
    out = {"steps": np.array(STEPS)}
    for integ in INTEGRATORS:
        for cold, tag in ((False, ""), (True, "_cold")):
            d = system(integ, cold)
            r = oracle.Reference(d)
            r.initialize()
            r.run(STEPS)
            p, v, _ = r.state()
            r.close()
            out[f"{integ}{tag}_pos"] = p
            out[f"{integ}{tag}_vel"] = v
    np.savez_compressed(os.path.join(HERE, "integrators.npz"), **out)


if __name__ == "__main__":
    main()
