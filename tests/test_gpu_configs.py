"""Parity of the CUDA path with the reference at the benchmark configurations'
own sizes (fixtures of tests/golden/make_configs.py, written by the reference's
code): the 4,096-particle Lennard-Jones fluid, the 10,000-bead polymer melt in
unbounded space and a 32,768-bead cut of the periodic EXV + DebyeHuckel fluid
at the 1,048,576-bead fluid's density and cutoffs.

Bounds (force error = relative RMS over all particles):
  lists        both forms, bit for bit (pair count and SHA-256 of the pairs)
  forces       FP64 <= 1e-12; mixed <= 1e-5
  energies     FP64 <= 1e-12; mixed <= 1e-7 relative
  1,000 velocity-Verlet steps
               the total energy every 100 steps against the reference's own
               trace, relative to the system's energy scale (the largest
               |term energy| or kinetic energy seen), within VV_ENERGY_TOL;
               FP64 final positions within VV_POS_TOL of the reference's.
               Velocity Verlet is chaotic: a 1e-13 A perturbation of the
               start grows in 1,000 steps to 9e-3 A in the Lennard-Jones
               fluid, 5e-8 A in the melt and 5e-7 A in the fluid cut (the
               oracle, tests/test_oracle_configs.py, follows the reference bit
               for bit), so FP64 positions differ from the reference's by the
               amplified rounding of a different summation order (measured on
               B200: 1.2e-4, 2.2e-8, 1.2e-8 A) and the mixed form's by the
               amplified FP32 force error (2.2, 9e-3, 6e-2 A).  The energy
               trace is the drift statement: measured, FP64 2.2e-8 / 1e-14 /
               5e-15 and mixed 2.9e-5 / 3.9e-8 / 2.5e-8 of the scale, the
               mixed Lennard-Jones figure a third of the reference's own
               1,000-step drift (1.5 of 12,463 kcal/mol).
"""
import numpy as np
import pytest

from conftest import config_cases, rel_rms, sha256
from mjolnir_b200.engine import Engine

pytestmark = pytest.mark.gpu

CASES = config_cases()
FORCE_TOL = {"fp64": 1e-12, "mixed": 1e-5}
ENERGY_TOL = {"fp64": 1e-12, "mixed": 1e-7}
VV_ENERGY_TOL = {"config1_lj4096": {"fp64": 2e-7, "mixed": 1e-4},
                 "config2_melt10000": {"fp64": 1e-12, "mixed": 1e-6},
                 "config3_fluid32768": {"fp64": 1e-12, "mixed": 1e-6}}
VV_POS_TOL = {"config1_lj4096": 2e-3, "config2_melt10000": 1e-6, "config3_fluid32768": 1e-6}
TERMS = ("bond", "angle", "dihedral", "exv", "dh", "lj")


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", sorted(CASES))
def test_config_lists_forces_energies(name, precision):
    d, _dt, _sub, fx = CASES[name]
    e = Engine(precision)
    sid = e.add_system(d)
    e.commit()
    total = np.zeros((d.n, 3))
    for t in TERMS:
        if f"energy_{t}" not in fx:
            continue
        if f"pairs_sha_{t}" in fx:
            pairs = e.neighbors(sid, t)
            assert len(pairs) == int(fx[f"pairs_count_{t}"]), (name, t)
            assert sha256(pairs.astype(np.int64)) == str(fx[f"pairs_sha_{t}"]), (name, t)
        f, en = e.term_force(sid, t)
        total += f
        if f"force_{t}" in fx:
            err = rel_rms(f, fx[f"force_{t}"])
            assert err <= FORCE_TOL[precision], (name, precision, t, err)
        ref = float(fx[f"energy_{t}"])
        assert abs(en - ref) <= ENERGY_TOL[precision] * max(abs(ref), 1e-12), (name, precision, t, en, ref)
    assert rel_rms(total, fx["force_total"]) <= FORCE_TOL[precision], (name, precision)
    E = e.energies(sid)
    for t in TERMS:
        if f"calc_energy_{t}" in fx:
            ref = float(fx[f"calc_energy_{t}"])
            assert abs(E[t] - ref) <= ENERGY_TOL[precision] * max(abs(ref), 1e-12), (name, precision, t, E[t], ref)
    e.close()


def vv_run(d, dt, precision, steps, every):
    """Potential + kinetic energy every `every` steps of a velocity-Verlet run,
    and the final state."""
    dv = d.copy()
    dv.integrator = "VelocityVerlet"
    dv.dt = dt
    e = Engine(precision)
    sid = e.add_system(dv)
    e.commit()
    trace, scale = [], 0.0

    def sample():
        nonlocal scale
        E = e.energies(sid)
        _p, v, _f = e.state(sid)
        kin = 0.5 * float(np.sum(d.mass[:, None] * v * v))
        pot = sum(E[t] for t in TERMS)
        scale = max(scale, kin, *(abs(E[t]) for t in TERMS))
        trace.append(pot + kin)

    sample()
    for _ in range(steps // every):
        e.step(every)
        sample()
    p, v, _ = e.state(sid)
    e.close()
    return np.array(trace), scale, p, v


@pytest.mark.parametrize("name", sorted(CASES))
def test_config_velocity_verlet_1000_steps(name):
    d, dt, sub, fx = CASES[name]
    ref = fx["vv_potential"] + fx["vv_kinetic"]
    steps, every = int(fx["vv_steps"]), int(fx["vv_every"])
    for precision in ("fp64", "mixed"):
        trace, scale, p, _v = vv_run(d, dt, precision, steps, every)
        drift = np.abs(trace - ref).max() / scale
        assert drift <= VV_ENERGY_TOL[name][precision], (name, precision, drift)
        if precision == "fp64":
            k = sub or d.n
            dp = p[:k] - fx["vv_pos"]
            if d.periodic:
                L = np.array(d.upper) - np.array(d.lower)
                dp -= L * np.round(dp / L)
            assert np.abs(dp).max() <= VV_POS_TOL[name], (name, np.abs(dp).max())


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_config_slot_major_lists(precision):
    """The slot-major list layout (schedule 5) on the fluid cut: the same
    lists bit for bit, the reference's forces within the form's tolerance,
    and in the mixed form the same forces as the default layout bit for bit."""
    d, _dt, _sub, fx = CASES["config3_fluid32768"]
    e = Engine(precision)
    sid = e.add_system(d)
    e.commit()
    base = {t: e.term_force(sid, t)[0] for t in ("exv", "dh")}
    for t in ("exv", "dh"):
        e.set_pair_schedule(t, 5)
        e.set_threads_per_particle(t, 8)
    for t in ("exv", "dh"):
        pairs = e.neighbors(sid, t)
        assert sha256(pairs.astype(np.int64)) == str(fx[f"pairs_sha_{t}"]), t
        f, _ = e.term_force(sid, t)
        assert rel_rms(f, fx[f"force_{t}"]) <= FORCE_TOL[precision], (precision, t)
        if precision == "mixed":
            assert np.array_equal(f, base[t]), t
    e.close()
