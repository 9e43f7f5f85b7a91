"""The oracle (oracle/oracle.c) pinned against the reference.

Golden fixtures (tests/golden/*.npz) were produced by the reference's own code
(oracle/_ref, see tests/golden/make_golden.py).  The C restatement must
reproduce them bit for bit: it keeps the reference's operation order, list
order and rebuild schedule.  When the reference driver is built (only where
the reference tree exists) the same comparisons also run live on fresh
systems.
"""
import numpy as np
import pytest

import oracle
from conftest import golden_cases

CASES = golden_cases()


@pytest.mark.parametrize("name", sorted(CASES))
def test_lists_match_reference(name):
    d, fx = CASES[name]
    o = oracle.Oracle(d)
    for t in ("exv", "dh", "lj"):
        if f"pairs_{t}" not in fx:
            continue
        got = o.neighbors(t, d.pos)
        assert np.array_equal(got, fx[f"pairs_{t}"].astype(np.int64)), (name, t)


@pytest.mark.parametrize("name", sorted(CASES))
def test_forces_energies_match_reference(name):
    d, fx = CASES[name]
    o = oracle.Oracle(d)
    for t in ("bond", "angle", "dihedral", "exv", "dh", "lj"):
        if f"force_{t}" not in fx:
            continue
        f, e = o.term_force(t, d.pos)
        ref_f = fx[f"force_{t}"]
        scale = max(np.abs(ref_f).max(), 1e-300)
        assert np.abs(f - ref_f).max() <= 1e-14 * scale, (name, t)
        assert e == pytest.approx(float(fx[f"energy_{t}"]), rel=1e-14, abs=1e-300), (name, t)
        ce = o.term_energy(t, d.pos)
        assert ce == pytest.approx(float(fx[f"calc_energy_{t}"]), rel=1e-14, abs=1e-300), (name, t)


@pytest.mark.parametrize("name", [n for n in sorted(CASES) if "vv_pos" in CASES[n][1]])
def test_velocity_verlet_trajectory_matches_reference(name):
    d, fx = CASES[name]
    d = d.copy()
    d.integrator = "VelocityVerlet"
    d.dt = float(fx["vv_dt"])
    o = oracle.Oracle(d)
    o.init_dynamics()
    o.run(int(fx["vv_steps"]))
    p, v, f = o.state()
    assert np.abs(p - fx["vv_pos"]).max() <= 1e-11
    assert np.abs(v - fx["vv_vel"]).max() <= 1e-10


def test_philox_known_answers():
    # Random123 known-answer vectors of philox4x32-10
    assert oracle.philox4x32([0, 0, 0, 0], [0, 0]) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert oracle.philox4x32([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert oracle.philox4x32([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0]) == \
        [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


def test_gaussian_stream_statistics():
    g = np.array([oracle.gaussian3(77, i, s) for i in range(2000) for s in range(5)]).ravel()
    assert abs(g.mean()) < 0.03
    assert abs(g.std() - 1.0) < 0.03
    # kurtosis of a normal is 3
    k = ((g - g.mean()) ** 4).mean() / g.var() ** 2
    assert abs(k - 3.0) < 0.2


def test_debye_length_constants():
    # lambda(300 K, 0.1 M) = 9.486 A, lambda(300 K, 0.15 M) = 7.697 A
    assert oracle.dh_params(300.0, 0.1, 5.5)[0] == pytest.approx(9.486, abs=2e-3)
    assert oracle.dh_params(300.0, 0.15, 5.5)[0] == pytest.approx(7.697, abs=2e-3)
    kB, NA, eps0, L2V = oracle.units()
    assert kB == pytest.approx(0.0019872036, rel=1e-7)
    assert L2V == 1e27


def test_exclusions_bond_within_three():
    from mjolnir_b200 import systems as S
    d = S.polymer_melt(nchains=2, nbeads=10, radius=30.0, seed=1)
    o = oracle.Oracle(d)
    r, idx = o.exclusions()
    # bead 5 of chain 0 ignores 2..8 (itself and three bonds either way)
    assert list(idx[r[5]:r[6]]) == [2, 3, 4, 5, 6, 7, 8]
    assert list(idx[r[0]:r[1]]) == [0, 1, 2, 3]
    mol = o.molecules()
    assert list(mol) == [0] * 10 + [1] * 10


# ------------------------------------------------------------- live reference
needs_ref = pytest.mark.skipif(not oracle.reference_available(),
                               reason="reference driver not built (no reference tree)")


@needs_ref
@pytest.mark.parametrize("seed", [21, 22])
def test_live_polymer_against_reference(seed):
    from mjolnir_b200 import systems as S
    d = S.polymer_melt(nchains=5, nbeads=40, radius=45.0, seed=seed)
    d.pos = d.pos + np.random.default_rng(seed).normal(0, 0.2, d.pos.shape)
    r = oracle.Reference(d)
    o = oracle.Oracle(d)
    for t in ("exv", "dh"):
        assert np.array_equal(r.neighbors(t), o.neighbors(t, d.pos))
    for t in ("bond", "angle", "dihedral", "exv", "dh"):
        fr, er = r.term_force(t)
        fo, eo = o.term_force(t, d.pos)
        assert np.array_equal(fr, fo), t
        assert er == eo, t


@needs_ref
def test_live_vv_trajectory_bit_exact():
    from mjolnir_b200 import systems as S
    d = S.polymer_melt(nchains=4, nbeads=40, radius=40.0, seed=3)
    d.integrator = "VelocityVerlet"
    d.dt = 0.005
    r = oracle.Reference(d)
    o = oracle.Oracle(d)
    r.initialize()
    o.init_dynamics()
    r.run(1000)
    o.run(1000)
    pr, vr, _ = r.state()
    po, vo, _ = o.state()
    assert np.array_equal(pr, po) and np.array_equal(vr, vo)


@needs_ref
def test_live_periodic_lj_against_reference():
    from mjolnir_b200 import systems as S
    d = S.lj_fluid(n=729, density=0.8, margin=0.3, seed=8)
    r = oracle.Reference(d)
    o = oracle.Oracle(d)
    assert np.array_equal(r.neighbors("lj"), o.neighbors("lj", d.pos))
    fr, er = r.term_force("lj")
    fo, eo = o.term_force("lj", d.pos)
    assert np.array_equal(fr, fo) and er == eo
