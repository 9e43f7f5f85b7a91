"""Sampling tests of the Langevin noise (Philox in place of the reference's
mt19937, so parity with the reference's noise is statistical): the bond
lengths of independent harmonic dimers follow the Boltzmann distribution.
A Kolmogorov-Smirnov distance well inside three times its sampling noise
passes; the reference's own check of its integrators is the same kind of
comparison of a sampled histogram with the Boltzmann curve
(test/integration/test_BAOABIntegrator)."""
import numpy as np
import pytest

import oracle
from mjolnir_b200 import systems as S

INTEGRATORS = ["BAOAB", "UnderdampedLangevin", "G-JFLangevin", "g-BAOABLangevin"]


def ks_distance(samples, d):
    s = np.sort(np.concatenate(samples))
    emp = np.arange(1, s.size + 1) / s.size
    k, r0 = float(d.bonds[1][0]), float(d.bonds[2][0])
    return float(np.max(np.abs(emp - S.dimer_length_cdf(s, k, r0, d.temperature)))), s.size


def bond_lengths(p):
    return np.linalg.norm(p[1::2] - p[0::2], axis=1)


@pytest.mark.parametrize("integrator", INTEGRATORS)
def test_oracle_dimer_bond_lengths_are_boltzmann(integrator):
    d = S.dimers(n=2000, integrator=integrator)
    o = oracle.Oracle(d)
    o.init_dynamics()
    o.run(400)
    samples = []
    for _ in range(60):
        o.run(100)
        samples.append(bond_lengths(o.state()[0]))
    ks, n = ks_distance(samples, d)
    assert ks < 3 * 0.87 / np.sqrt(n), ks


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("integrator", INTEGRATORS)
def test_gpu_dimer_bond_lengths_are_boltzmann(integrator, precision):
    from mjolnir_b200.engine import Engine
    d = S.dimers(n=20000, integrator=integrator, seed=7)
    e = Engine(precision)
    sid = e.add_system(d)
    e.commit()
    e.step(400)
    samples = []
    for _ in range(60):
        e.step(100)
        samples.append(bond_lengths(e.positions(sid)))
    e.close()
    ks, n = ks_distance(samples, d)
    assert ks < 3 * 0.87 / np.sqrt(n), ks
