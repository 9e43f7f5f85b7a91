"""The oracle (oracle.c, the C restatement) against the reference's own output
at the benchmark configurations' sizes (tests/golden/make_configs.py):
neighbour lists bit for bit through their hash, per-term forces and energies
to the last bits, and for the 4,096-particle Lennard-Jones fluid the whole
1,000-step velocity-Verlet run bit for bit.  CPU only."""
import numpy as np
import pytest

import oracle
from conftest import config_cases, sha256

CASES = config_cases()


@pytest.mark.parametrize("name", sorted(CASES))
def test_lists_forces_energies_match_reference(name):
    d, _dt, _sub, fx = CASES[name]
    o = oracle.Oracle(d)
    for t in ("exv", "dh", "lj"):
        if f"pairs_sha_{t}" not in fx:
            continue
        pairs = o.neighbors(t, d.pos).astype(np.int64)
        assert len(pairs) == int(fx[f"pairs_count_{t}"]), (name, t)
        assert sha256(pairs) == str(fx[f"pairs_sha_{t}"]), (name, t)
        f, e = o.term_force(t, d.pos)
        ref = fx[f"force_{t}"]
        assert np.abs(f - ref).max() <= 1e-14 * np.abs(ref).max(), (name, t)
        assert e == pytest.approx(float(fx[f"energy_{t}"]), rel=1e-14, abs=1e-300), (name, t)
        assert o.term_energy(t, d.pos) == pytest.approx(float(fx[f"calc_energy_{t}"]), rel=1e-14), (name, t)
    o.close()


def test_lj4096_velocity_verlet_1000_steps_bit_exact():
    d, dt, _sub, fx = CASES["config1_lj4096"]
    dv = d.copy()
    dv.integrator = "VelocityVerlet"
    dv.dt = dt
    o = oracle.Oracle(dv)
    o.init_dynamics()
    o.run(int(fx["vv_steps"]))
    p, v, _ = o.state()
    assert np.array_equal(p, fx["vv_pos"]) and np.array_equal(v, fx["vv_vel"])
    o.close()
