"""Every integrator against the reference's own trajectory where its noise
vanishes -- without friction, and with friction at temperature 0 -- from
tests/golden/integrators.npz (made by tests/golden/make_integrators.py from
the reference): the oracle bit for bit on the CPU, the GPU within its forms'
tolerances."""
import os
import sys

import numpy as np
import pytest

import oracle

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
from make_integrators import INTEGRATORS, system  # noqa: E402

GOLD = np.load(os.path.join(HERE, "golden", "integrators.npz"))
STEPS = int(GOLD["steps"])


@pytest.mark.parametrize("cold", [False, True])
@pytest.mark.parametrize("integrator", INTEGRATORS)
def test_oracle_reproduces_reference_trajectory(integrator, cold):
    tag = "_cold" if cold else ""
    o = oracle.Oracle(system(integrator, cold))
    o.init_dynamics()
    o.run(STEPS)
    p, v, _ = o.state()
    assert np.array_equal(p, GOLD[f"{integrator}{tag}_pos"]) and np.array_equal(v, GOLD[f"{integrator}{tag}_vel"])


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-9), ("mixed", 1e-4)])
@pytest.mark.parametrize("cold", [False, True])
@pytest.mark.parametrize("integrator", INTEGRATORS)
def test_gpu_follows_reference_trajectory(integrator, cold, precision, tol):
    from mjolnir_b200.engine import Engine
    tag = "_cold" if cold else ""
    d = system(integrator, cold)
    e = Engine(precision)
    sid = e.add_system(d)
    e.commit()
    e.step(STEPS)
    p, v, _ = e.state(sid)
    e.close()
    assert np.abs(p - GOLD[f"{integrator}{tag}_pos"]).max() <= tol, (integrator, cold, precision)
    assert np.abs(v - GOLD[f"{integrator}{tag}_vel"]).max() <= 10 * tol, (integrator, cold, precision)
