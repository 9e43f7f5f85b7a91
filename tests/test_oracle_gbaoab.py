"""The oracle's g-BAOAB Langevin integrator against the reference's own
(core/gBAOABLangevinIntegrator.hpp, omp/gBAOABLangevinIntegrator.hpp) on
systems without constraints, where it is BAOAB with each half drift applied to
the position and the displacement taken as new minus old position.

The reference draws its noise from mt19937 and the oracle from Philox, so the
trajectories are compared where the noise term vanishes: gamma = 0 (no
friction, no noise) and temperature 0 (friction, no noise).  Those two cases
fix every rounding step of the update; the noise itself is checked by its
statistics (equipartition)."""
import numpy as np
import pytest

import oracle
from mjolnir_b200 import systems as S

needs_ref = pytest.mark.skipif(not oracle.reference_available(),
                               reason="reference driver not built (no reference tree)")


def _run_both(d, steps):
    r = oracle.Reference(d)
    o = oracle.Oracle(d)
    r.initialize()
    o.init_dynamics()
    r.run(steps)
    o.run(steps)
    return r.state(), o.state()


@needs_ref
def test_frictionless_trajectory_bit_exact():
    d = S.polymer_melt(nchains=4, nbeads=40, radius=40.0, seed=31)
    d.integrator = "g-BAOABLangevin"
    d.gamma = np.zeros(d.n)
    d.dt = 0.005
    (pr, vr, fr), (po, vo, fo) = _run_both(d, 800)
    assert np.array_equal(pr, po) and np.array_equal(vr, vo) and np.array_equal(fr, fo)


@needs_ref
@pytest.mark.parametrize("periodic", [False, True])
def test_cold_friction_trajectory_bit_exact(periodic):
    """gamma > 0 at temperature 0: the friction factors of both half steps."""
    if periodic:
        d = S.bead_fluid(n=1500, density=0.003, seed=32, dt=0.3)
        d.gamma = np.random.default_rng(2).uniform(0.1, 0.9, d.n)
    else:
        d = S.polymer_melt(nchains=4, nbeads=40, radius=40.0, seed=33)
        d.gamma = np.random.default_rng(3).uniform(0.5, 2.0, d.n)
    d.integrator = "g-BAOABLangevin"
    d.temperature = 0.0
    d.dh = None                       # the Debye length needs a temperature
    (pr, vr, _), (po, vo, _) = _run_both(d, 600)
    assert np.array_equal(pr, po) and np.array_equal(vr, vo)


def test_equipartition():
    """BAOAB's O step keeps the Maxwell-Boltzmann velocity distribution
    exactly for a free particle: m <v^2> = kB T."""
    d = S.bead_fluid(n=1200, density=0.002, seed=34, dt=0.1, gamma=0.5)
    d.integrator = "g-BAOABLangevin"
    d.vel = np.zeros_like(d.vel)
    o = oracle.Oracle(d)
    o.init_dynamics()
    o.run(600)
    kin = []
    for _ in range(40):
        o.run(25)
        v = o.state()[1]
        kin.append(0.5 * float(np.sum(d.mass[:, None] * v * v)))
    assert np.mean(kin) == pytest.approx(1.5 * d.n * S.KB_KCAL * d.temperature, rel=0.02)
