"""B200Simulator -- the reference-side binding (tests/binding/B200Simulator.hpp,
a SimulatorBase a maintainer adds to the reference tree) -- on the GPU.

A System and a ForceField built by the reference's own code are handed to
B200Simulator, which reads the reference's objects (particles, boundary,
attributes, bonded interactions and their topology, pair potentials and
partitions, the velocity-Verlet integrator) and drives this library's C ABI;
initialize(), step() until it returns false, finalize() write the GPU state
back into the reference System.  After 1,000 steps of the 4,096-particle
Lennard-Jones fluid and of the 10,000-bead melt the positions are compared
with those of the reference's own MolecularDynamicsSimulator on the same
objects (equal bit for bit to the configuration fixtures,
tests/test_binding_reference.py), within the bounds of
tests/test_gpu_configs.py, and the total energy with the reference's."""
import numpy as np
import pytest

import binding_lib as B
from conftest import config_cases
from test_gpu_configs import VV_ENERGY_TOL, VV_POS_TOL

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not B.available(), reason="binding library not built (no reference tree)")]

CASES = config_cases()


@pytest.mark.parametrize("name", ["config1_lj4096", "config2_melt10000"])
def test_b200_simulator_follows_reference_simulator(name, tmp_path):
    d, dt, _sub, fx = CASES[name]
    d = d.copy()
    d.dt = dt
    steps = int(fx["vv_steps"])
    e_ref = float(fx["vv_potential"][-1] + fx["vv_kinetic"][-1])
    scale = max(abs(float(fx["vv_potential"][0])), float(fx["vv_kinetic"][0]))
    p, _v, e = B.run(d, B.B200, steps, str(tmp_path / "gpu"), precision=0)
    dp = p - fx["vv_pos"]
    if d.periodic:
        L = np.array(d.upper) - np.array(d.lower)
        dp -= L * np.round(dp / L)
    assert np.abs(dp).max() <= VV_POS_TOL[name], (name, np.abs(dp).max())
    assert abs(e - e_ref) <= VV_ENERGY_TOL[name]["fp64"] * scale, (name, e, e_ref)
    # the mixed form through the same binding
    p, _v, e = B.run(d, B.B200, steps, str(tmp_path / "gpu_mixed"), precision=1)
    assert np.isfinite(p).all()
    assert abs(e - e_ref) <= VV_ENERGY_TOL[name]["mixed"] * scale, (name, e, e_ref)
