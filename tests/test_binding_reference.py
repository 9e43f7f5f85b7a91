"""The reference side of the binding test on the CPU: the reference's own
MolecularDynamicsSimulator, behind SimulatorBase in the binding library, runs
the 4,096-particle Lennard-Jones fluid's 1,000 velocity-Verlet steps bit for
bit as the configuration fixture recorded them (tests/golden/make_configs.py),
so that tests/test_gpu_binding.py compares B200Simulator with the reference's
simulator itself."""
import numpy as np
import pytest

import binding_lib as B
from conftest import config_cases


@pytest.mark.skipif(not B.available(), reason="binding library not built (no reference tree)")
def test_reference_simulator_matches_fixture(tmp_path):
    d, dt, _sub, fx = config_cases()["config1_lj4096"]
    d = d.copy()
    d.dt = dt
    p, v, _e = B.run(d, B.REFERENCE_MD, int(fx["vv_steps"]), str(tmp_path / "ref"))
    assert np.array_equal(p, fx["vv_pos"]) and np.array_equal(v, fx["vv_vel"])
