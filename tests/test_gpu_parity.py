"""Parity of the CUDA path (through the C ABI) with the reference and the oracle.

Tolerances (force error = relative RMS over all particles,
sqrt(sum|dF|^2 / sum|F|^2)):
  FP64 form    lists bit-exact; forces <= 1e-12; energies <= 1e-12 relative
  mixed form   lists bit-exact; forces <= 1e-5 relative RMS (the mixed form's bound);
               energies <= 1e-5 relative
"""
import numpy as np
import pytest

import oracle
from conftest import golden_cases, rel_rms
from mjolnir_b200 import systems as S
from mjolnir_b200.engine import Engine

pytestmark = pytest.mark.gpu

CASES = golden_cases()
FORCE_TOL = {"fp64": 1e-12, "mixed": 1e-5}
ENERGY_TOL = {"fp64": 1e-12, "mixed": 1e-7}


def engine_for(d, precision, **kw):
    e = Engine(precision, **kw)
    sid = e.add_system(d)
    e.commit()
    return e, sid


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", sorted(CASES))
def test_golden_lists_forces_energies(name, precision):
    d, fx = CASES[name]
    e, sid = engine_for(d, precision)
    for t in ("exv", "dh", "lj"):
        if f"pairs_{t}" in fx:
            got = e.neighbors(sid, t)
            assert np.array_equal(got, fx[f"pairs_{t}"].astype(np.int64)), (name, t)
    for t in ("bond", "angle", "dihedral", "exv", "dh", "lj"):
        if f"force_{t}" not in fx:
            continue
        f, en = e.term_force(sid, t)
        ref_f, ref_e = fx[f"force_{t}"], float(fx[f"energy_{t}"])
        assert rel_rms(f, ref_f) <= FORCE_TOL[precision], (name, t, rel_rms(f, ref_f))
        assert abs(en - ref_e) <= ENERGY_TOL[precision] * max(abs(ref_e), 1e-12), (name, t, en, ref_e)
    # ForceField::calc_energy per term equals the reference's calc_energy
    E = e.energies(sid)
    for t in ("bond", "angle", "dihedral", "exv", "dh", "lj"):
        if f"calc_energy_{t}" in fx:
            ref = float(fx[f"calc_energy_{t}"])
            assert abs(E[t] - ref) <= ENERGY_TOL[precision] * max(abs(ref), 1e-12), (name, t)
    e.close()


@pytest.mark.parametrize("name", [n for n in sorted(CASES) if "vv_pos" in CASES[n][1]])
def test_golden_velocity_verlet(name):
    """Frictionless, noise-free trajectory against the reference's own run."""
    d, fx = CASES[name]
    d = d.copy()
    d.integrator = "VelocityVerlet"
    d.dt = float(fx["vv_dt"])
    for precision, tol in (("fp64", 1e-8), ("mixed", 1e-4)):
        e, sid = engine_for(d, precision)
        e.step(int(fx["vv_steps"]))
        p, v, _ = e.state(sid)
        L = np.array(d.upper) - np.array(d.lower)
        dp = p - fx["vv_pos"]
        if d.periodic:
            dp -= L * np.round(dp / L)
        assert np.abs(dp).max() <= tol, (name, precision, np.abs(dp).max())
        e.close()


def test_baoab_matches_oracle_noise_stream():
    """BAOAB with the same Philox stream as the oracle: the trajectories agree."""
    d = S.polymer_melt(nchains=6, nbeads=60, radius=60.0, seed=5)
    o = oracle.Oracle(d)
    o.init_dynamics()
    o.run(100)
    po, vo, _ = o.state()
    for precision, tol in (("fp64", 1e-9), ("mixed", 1e-5)):
        e, sid = engine_for(d, precision)
        e.step(100)
        p, v, _ = e.state(sid)
        assert np.abs(p - po).max() <= tol, precision
        assert np.abs(v - vo).max() <= 10 * tol, precision
        e.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_lists_after_dynamics_bit_exact(precision):
    """After many rebuild cycles, the GPU lists equal the reference set on the
    GPU's own coordinates (checked by the oracle, pinned to the reference)."""
    d = S.polymer_melt(nchains=10, nbeads=50, radius=60.0, seed=12)
    e, sid = engine_for(d, precision)
    e.step(600)
    assert e.rebuild_count(sid, "exv") >= 1
    e.rebuild()
    p = e.positions(sid)
    o = oracle.Oracle(d)
    for t in ("exv", "dh"):
        assert np.array_equal(e.neighbors(sid, t), o.neighbors(t, p)), t
    e.close()


def test_periodic_fluid_lists_and_forces_after_dynamics():
    d = S.bead_fluid(n=4000, density=0.003, seed=13, dt=0.3)
    e, sid = engine_for(d, "mixed")
    e.step(200)
    e.rebuild()
    p = e.positions(sid)
    o = oracle.Oracle(d)
    for t in ("exv", "dh"):
        assert np.array_equal(e.neighbors(sid, t), o.neighbors(t, p)), t
        f, _ = e.term_force(sid, t)
        fo, _ = o.term_force(t, p)
        assert rel_rms(f, fo) <= 1e-5, t
    e.close()


def test_mixed_is_deterministic_and_graph_independent():
    d = S.polymer_melt(nchains=8, nbeads=50, radius=60.0, seed=4)
    runs = []
    for graphs in (True, True, False):
        e, sid = engine_for(d, "mixed", graphs=graphs)
        e.step(150)
        runs.append(e.state(sid))
        e.close()
    for r in runs[1:]:
        for a, b in zip(runs[0], r):
            assert np.array_equal(a, b)


def test_batch_equals_alone_bit_exact():
    """Systems packed into one arena evolve exactly as they do alone (mixed
    form: fixed-point sums do not depend on list order or neighbours)."""
    descs = [S.polymer_melt(nchains=4, nbeads=50, radius=50.0, seed=31, temperature=290.0),
             S.lj_fluid(n=512, seed=32),
             S.bead_fluid(n=2000, density=0.003, seed=33, dt=0.3),
             S.polymer_melt(nchains=3, nbeads=40, radius=40.0, seed=34, temperature=350.0,
                            ionic_strength=0.25)]
    alone = []
    for d in descs:
        e, sid = engine_for(d, "mixed")
        e.step(120)
        alone.append(e.state(sid))
        e.close()
    e = Engine("mixed")
    ids = [e.add_system(d) for d in descs]
    e.commit()
    e.step(120)
    for sid, ref in zip(ids, alone):
        got = e.state(sid)
        for a, b in zip(got, ref):
            assert np.array_equal(a, b)
    e.close()


def test_serving_style_admission_keeps_results():
    """Adding and removing systems between chunks (re-commit) changes nothing
    for the systems that stay."""
    a = S.polymer_melt(nchains=4, nbeads=50, radius=50.0, seed=41)
    b = S.polymer_melt(nchains=3, nbeads=60, radius=50.0, seed=42)
    c = S.bead_fluid(n=1500, density=0.003, seed=43, dt=0.3)
    e1, s1 = engine_for(a, "mixed")
    e1.step(100)
    ref = e1.state(s1)
    e1.close()
    e = Engine("mixed")
    ia = e.add_system(a)
    ib = e.add_system(b)
    e.commit()
    e.step(40)
    e.remove_system(ib)
    ic = e.add_system(c)
    e.commit()
    e.step(60)
    got = e.state(ia)
    for x, y in zip(got, ref):
        assert np.array_equal(x, y)
    assert e.step_count(ia) == 100 and e.step_count(ic) == 60
    e.close()


def test_list_overflow_rolls_back_and_recovers():
    """A list capacity that is too small for the next rebuild is detected on
    the device, the chunk is rolled back, the lists grow, and the result equals
    an undisturbed run (host-side fault injection; no device fault)."""
    d = S.lj_fluid(n=1000, density=0.8, margin=0.05, seed=44)
    e, sid = engine_for(d, "mixed")
    e.step(300)
    ref = e.state(sid)
    e.close()
    e, sid = engine_for(d, "mixed")
    e.debug_set_list_capacity("lj", 8)
    e.step(300)
    got = e.state(sid)
    for x, y in zip(got, ref):
        assert np.array_equal(x, y)
    e.close()


def test_langevin_temperature():
    """BAOAB holds the kinetic temperature: <KE> = 3/2 N kT within 3 %."""
    d = S.lj_fluid(n=1000, density=0.8, seed=45, gamma=1.0, dt=0.005)
    e, sid = engine_for(d, "mixed")
    e.step(2000)
    kes = []
    for _ in range(40):
        e.step(50)
        _, v, _ = e.state(sid)
        kes.append(0.5 * (v ** 2).sum())
    kT = 1.0
    assert np.mean(kes) == pytest.approx(1.5 * d.n * kT, rel=0.03)
    e.close()


def test_fixed_point_newton_third_law():
    """Pair forces cancel exactly in fixed point (sum of all pair forces is 0
    up to the per-pair rounding, which is antisymmetric)."""
    d = S.bead_fluid(n=3000, density=0.003, seed=46, dt=0.3)
    e, sid = engine_for(d, "mixed")
    for t in ("exv", "dh"):
        f, _ = e.term_force(sid, t)
        assert np.abs(f.sum(axis=0)).max() <= 1e-9
    e.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_launch_shapes_give_the_same_trajectory(precision):
    """Every threads-per-slot and partner-batch choice of the autotuner gives
    the same dynamics: bit for bit in the mixed form, within rounding of the
    summation order in FP64."""
    descs = [S.polymer_melt(nchains=4, nbeads=60, radius=45.0, seed=41),
             S.bead_fluid(n=3000, density=0.003, seed=42, dt=0.3),
             S.lj_fluid(n=512, seed=43)]
    ref = None
    shapes = [(0, tpp, unr) for tpp in (1, 2, 4, 8, 16, 32) for unr in (1, 2, 4)]
    shapes += [(sch, tpp, 1) for sch in (2, 3) for tpp in (2, 4, 8, 16)]
    shapes += [(4, tpp, unr) for tpp in (1, 4, 16, 32) for unr in (1, 2)]
    shapes += [(5, tpp, unr) for tpp in (1, 8, 16, 32) for unr in (1, 2, 4)]      # slot-major lists
    shapes += [(2, 32, 1), (3, 32, 1)]                                            # run as schedule 0
    if precision == "mixed":
        shapes += [(1, tpp, unr) for tpp in (1, 16, 32) for unr in (1, 2, 4)]
    for sch, tpp, unr in shapes:
        e = Engine(precision)
        ids = [e.add_system(d) for d in descs]
        e.commit()
        for term in ("exv", "dh", "lj"):
            e.set_pair_schedule(term, sch)
            e.set_threads_per_particle(term, tpp)
            e.set_pair_unroll(term, unr)
            assert (e.get_pair_schedule(term), e.get_pair_unroll(term)) == (sch, unr)
        e.step(30)
        got = [e.state(sid)[0] for sid in ids]
        e.close()
        if ref is None:
            ref = got
            continue
        for a, b in zip(got, ref):
            if precision == "mixed":
                assert np.array_equal(a, b), (sch, tpp, unr)
            else:
                assert np.abs(a - b).max() <= 1e-9 * np.abs(b).max(), (sch, tpp, unr)


def test_simulated_annealing_matches_oracle():
    """A linear annealing schedule (temperature updated every 25 steps) on the
    GPU follows the oracle driven by the same Philox stream and schedule."""
    from mjolnir_b200 import anneal
    d = S.polymer_melt(nchains=6, nbeads=60, radius=60.0, seed=6)
    first, last, total, each = 400.0, 250.0, 100, 25
    d.temperature = first
    o = oracle.Oracle(d)
    o.init_dynamics()
    done = 0
    while done < total:
        o.run(each)
        done += each
        o.set_temperature(anneal.current(first, last, done * (1.0 / total)))
    po, vo, _ = o.state()
    e, sid = engine_for(d, "fp64")
    anneal.run(e, {sid: (first, last)}, total, each)
    p, v, _ = e.state(sid)
    assert np.abs(p - po).max() <= 1e-9
    assert np.abs(v - vo).max() <= 1e-8
    e.close()


@pytest.mark.parametrize("lanes", [4, 8, 16, 32])
@pytest.mark.parametrize("case", ["melt", "fluid"])
def test_build_lanes_give_the_same_lists(case, lanes):
    """Every lanes-per-particle choice of the list build gives the reference's
    lists (a forced rebuild after dynamics) and, through the rebuilds during
    the dynamics, the same trajectory bit for bit (mixed form)."""
    if case == "melt":
        d = S.polymer_melt(nchains=10, nbeads=50, radius=60.0, seed=52)
    else:
        d = S.bead_fluid(n=4000, density=0.003, seed=53, dt=0.3)
    e, sid = engine_for(d, "mixed")
    for t in ("exv", "dh"):
        e.set_build_lanes(t, lanes)
        assert e.get_build_lanes(t) == lanes
    e.step(300)
    assert e.rebuild_count(sid, "exv") >= 1
    o = oracle.Oracle(d)
    traj = e.state(sid)
    e.rebuild()
    p = e.positions(sid)
    for t in ("exv", "dh"):
        assert np.array_equal(e.neighbors(sid, t), o.neighbors(t, p)), (t, lanes)
    e.close()
    e32, sid32 = engine_for(d, "mixed")
    e32.step(300)
    for a, b in zip(traj, e32.state(sid32)):
        assert np.array_equal(a, b), lanes
    e32.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_frozen_system_waits_and_resumes(precision):
    """A frozen system keeps its state (positions, velocities, forces, step
    counter) while the others advance; released, it continues as if it had
    never paused (mixed form: bit for bit)."""
    a = S.polymer_melt(nchains=3, nbeads=40, radius=40.0, seed=81)
    b = S.polymer_melt(nchains=3, nbeads=40, radius=40.0, seed=82)
    e = Engine(precision)
    sa, sb = e.add_system(a), e.add_system(b)
    e.commit()
    e.step(20)
    before = e.state(sa)
    e.freeze(sa)
    e.step(30)
    after = e.state(sa)
    for x, y in zip(before, after):
        assert np.array_equal(x, y)
    assert e.step_count(sa) == 20 and e.step_count(sb) == 50
    e.freeze(sa, False)
    e.step(25)
    got = e.state(sa)
    e.close()
    ref_e = Engine(precision)
    rid = ref_e.add_system(a)
    ref_e.commit()
    ref_e.step(45)
    want = ref_e.state(rid)
    ref_e.close()
    for x, y in zip(got, want):
        if precision == "mixed":
            assert np.array_equal(x, y)
        else:
            assert np.abs(x - y).max() <= 1e-9 * max(1.0, np.abs(y).max())


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_bulk_state_copies_match_per_system_state(precision):
    """mjg_get_state_all returns every system's state in arena order, and
    mjg_set_state_all followed by steps gives the trajectory of per-system
    mjg_set_state calls with the same arrays: bit for bit in the mixed form,
    to rounding in FP64 (whose bonded sums add in shared memory in the order
    the threads arrive)."""
    descs = [S.polymer_melt(nchains=3, nbeads=40, radius=35.0, seed=60),
             S.bead_fluid(n=2000, density=0.003, seed=61, dt=0.3),
             S.lj_fluid(n=343, seed=62)]

    def fresh():
        e = Engine(precision)
        ids = [e.add_system(d) for d in descs]
        e.commit()
        e.step(20)
        return e, ids

    e, ids = fresh()
    n = e.total_particles()
    pos, vel = np.empty((n, 3)), np.empty((n, 3))
    e.get_state_all(pos, vel)
    parts = [e.state(sid)[:2] for sid in ids]
    assert np.array_equal(pos, np.concatenate([p for p, _ in parts]))
    assert np.array_equal(vel, np.concatenate([v for _, v in parts]))
    vel2 = 0.5 * vel
    e.set_state_all(pos, vel2)
    e.step(30)
    bulk = [e.state(sid)[:2] for sid in ids]
    e.close()
    e, ids = fresh()
    off = 0
    for sid, d in zip(ids, descs):
        e.set_state(sid, pos[off:off + d.n], vel2[off:off + d.n])
        off += d.n
    e.step(30)
    each = [e.state(sid)[:2] for sid in ids]
    e.close()
    for (p0, v0), (p1, v1) in zip(bulk, each):
        if precision == "mixed":
            assert np.array_equal(p0, p1) and np.array_equal(v0, v1)
        else:
            assert np.abs(p0 - p1).max() <= 1e-9 * max(1.0, np.abs(p1).max())
            assert np.abs(v0 - v1).max() <= 1e-7 * max(1.0, np.abs(v1).max())
