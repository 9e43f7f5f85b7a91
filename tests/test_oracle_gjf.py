"""The oracle's G-JF Langevin integrator against the reference's own
(core/GJFNVTLangevinIntegrator.hpp, omp/GJFNVTLangevinIntegrator.hpp).

As for the other Langevin integrators the noise streams differ (mt19937 in
the reference, Philox here), so trajectories are compared bit for bit where
the noise vanishes: alpha = 0, and temperature 0 with alpha > 0 (every
friction factor a, b of the update).  The noise is checked by equipartition."""
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
    d = S.polymer_melt(nchains=4, nbeads=40, radius=40.0, seed=51)
    d.integrator = "G-JFLangevin"
    d.gamma = np.zeros(d.n)
    d.dt = 0.005
    (pr, vr, fr), (po, vo, fo) = _run_both(d, 800)
    assert np.array_equal(pr, po) and np.array_equal(vr, vo) and np.array_equal(fr, fo)


@needs_ref
@pytest.mark.parametrize("periodic", [False, True])
def test_cold_friction_trajectory_bit_exact(periodic):
    if periodic:
        d = S.bead_fluid(n=1500, density=0.003, seed=52, dt=0.3)
        d.gamma = np.random.default_rng(4).uniform(0.1, 0.9, d.n) * d.mass
    else:
        d = S.polymer_melt(nchains=4, nbeads=40, radius=40.0, seed=53)
        d.gamma = np.random.default_rng(5).uniform(0.5, 2.0, d.n) * d.mass
    d.integrator = "G-JFLangevin"
    d.temperature = 0.0
    d.dh = None
    (pr, vr, _), (po, vo, _) = _run_both(d, 600)
    assert np.array_equal(pr, po) and np.array_equal(vr, vo)


def stationary_kT(d):
    """kB T times the stationary m <v^2> / kB T of the scheme's velocity for a
    free particle.  With f = 0 the update is v' = a v + (b/m) beta,
    beta ~ N(0, 2 alpha kB T dt), a = (1 - x) / (1 + x), b = 1 / (1 + x),
    x = alpha dt / 2m, so m <v^2> = (b^2 / m) 2 alpha kB T dt / (1 - a^2)
    = kB T: no bias, unlike the UnderdampedLangevin scheme."""
    return S.KB_KCAL * d.temperature


def test_equipartition():
    d = S.bead_fluid(n=1200, density=0.002, seed=54, dt=0.1, gamma=0.5)
    d.gamma = d.gamma * d.mass                 # alpha = m gamma
    d.integrator = "G-JFLangevin"
    d.vel = np.zeros_like(d.vel)
    o = oracle.Oracle(d)
    o.init_dynamics()
    o.run(600)
    kin = []
    for _ in range(40):
        o.run(25)
        v = o.state()[1]
        kin.append(0.5 * float(np.sum(d.mass[:, None] * v * v)))
    assert np.mean(kin) == pytest.approx(1.5 * d.n * stationary_kT(d), rel=0.015)
