"""The UnderdampedLangevin, G-JF and g-BAOAB integrators on the GPU against the oracle
(the same Philox noise stream, so the trajectories agree to the precision's
tolerance), across a checkpoint, a temperature change, and mixed with the
other integrators in one arena."""
import numpy as np
import pytest

import oracle
from mjolnir_b200 import systems as S
from mjolnir_b200.engine import Engine

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-9, "mixed": 1e-5}


INTEGRATORS = ["UnderdampedLangevin", "G-JFLangevin", "g-BAOABLangevin"]


def _with(d, integrator):
    d = d.copy()
    d.integrator = integrator
    if integrator == "G-JFLangevin":
        d.gamma = d.gamma * d.mass            # alpha = m gamma
    return d


def _wrap(dp, d):
    if d.periodic:
        L = np.array(d.upper) - np.array(d.lower)
        dp = dp - L * np.round(dp / L)
    return dp


def _oracle_run(d, steps, temperature_at=None):
    o = oracle.Oracle(d)
    o.init_dynamics()
    if temperature_at is None:
        o.run(steps)
    else:
        k, T = temperature_at
        o.run(k)
        o.set_temperature(T)
        o.run(steps - k)
    return o.state()


CASES = {
    "melt": lambda i: _with(S.polymer_melt(nchains=6, nbeads=60, radius=60.0, seed=41), i),
    "fluid": lambda i: _with(S.bead_fluid(n=3000, density=0.003, seed=42, dt=0.2, gamma=0.7), i),
    "lj": lambda i: _with(S.lj_fluid(n=729, density=0.8, margin=0.3, seed=43), i),
}


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("integrator", INTEGRATORS)
def test_matches_oracle_noise_stream(integrator, name, precision):
    d = CASES[name](integrator)
    po, vo, _ = _oracle_run(d, 120)
    e = Engine(precision)
    sid = e.add_system(d)
    e.commit()
    e.step(120)
    p, v, _ = e.state(sid)
    e.close()
    assert np.abs(_wrap(p - po, d)).max() <= TOL[precision], (name, precision)
    assert np.abs(v - vo).max() <= 10 * TOL[precision], (name, precision)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("integrator", INTEGRATORS)
def test_steps_in_chunks_equal_one_run(integrator, precision):
    """The closing half of a chunk's last step and the next chunk's first
    pass (the fused kick) give the same trajectory as one long chunk: bit for
    bit in the mixed form, within the rounding of the FP64 form's atomic
    force sums (their order varies from run to run)."""
    d = CASES["melt"](integrator)
    runs = []
    for chunks in ([90], [1, 30, 7, 52]):
        e = Engine(precision)
        sid = e.add_system(d)
        e.commit()
        for k in chunks:
            e.step(k)
        runs.append(e.state(sid))
        e.close()
    for a, b in zip(*runs):
        if precision == "mixed":
            assert np.array_equal(a, b)
        else:
            assert np.abs(a - b).max() <= 1e-9 * max(1.0, np.abs(b).max())


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("integrator", INTEGRATORS)
def test_temperature_change_matches_oracle(integrator, precision):
    d = CASES["melt"](integrator)
    po, vo, _ = _oracle_run(d, 100, temperature_at=(40, 450.0))
    e = Engine(precision)
    sid = e.add_system(d)
    e.commit()
    e.step(40)
    e.set_temperature(sid, 450.0)
    e.step(60)
    p, v, _ = e.state(sid)
    e.close()
    assert np.abs(p - po).max() <= TOL[precision]
    assert np.abs(v - vo).max() <= 10 * TOL[precision]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_mixed_integrators_in_one_arena(precision):
    """BAOAB, velocity Verlet, UnderdampedLangevin and G-JF systems side by
    side, each against its own oracle run."""
    descs = []
    for k, kind in enumerate(("BAOAB", "UnderdampedLangevin", "VelocityVerlet", "G-JFLangevin",
                              "UnderdampedLangevin", "G-JFLangevin")):
        d = S.polymer_melt(nchains=4, nbeads=50, radius=50.0, seed=44 + k)
        d = _with(d, kind)
        if kind == "VelocityVerlet":
            d.dt = 0.005
        descs.append(d)
    e = Engine(precision)
    sids = [e.add_system(d) for d in descs]
    e.commit()
    e.step(80)
    for d, sid in zip(descs, sids):
        po, vo, _ = _oracle_run(d, 80)
        p, v, _ = e.state(sid)
        assert np.abs(p - po).max() <= TOL[precision], d.integrator
        assert np.abs(v - vo).max() <= 10 * TOL[precision], d.integrator
    e.close()


@pytest.mark.parametrize("integrator", INTEGRATORS)
def test_checkpoint_restart_is_bit_exact(integrator, tmp_path):
    """Interrupted at step 70 and resumed in a new engine from the checkpoint
    files (UnderdampedLangevin: the acceleration is rebuilt from the forces
    and the noise of step 70), the run ends bit for bit where the
    uninterrupted run does (mixed form: its force sums do not depend on the
    list order)."""
    from mjolnir_b200 import checkpoint as K
    d = CASES["fluid"](integrator)
    e = Engine("mixed")
    sid = e.add_system(d)
    e.commit()
    e.step(70)
    K.save(e, sid, d, str(tmp_path / "ck"))
    e.step(90)
    ref = e.state(sid)
    e.close()
    r = K.restore(str(tmp_path / "ck"), d)
    e2 = Engine("mixed")
    sid2 = e2.add_system(r)
    e2.commit()
    assert e2.step_count(sid2) == 70
    e2.step(90)
    got = e2.state(sid2)
    e2.close()
    for a, b in zip(got, ref):
        assert np.array_equal(a, b)


def _stationary_kT(d):
    """kB T times the stationary m <v^2> / kB T of a free particle.
    UnderdampedLangevin, g = gamma dt / 2: v' = c v + (dt/2)(1 - g)(a + a'),
    c = (1 - g)((1 - g)^2 + g), variance kB T / m * 2 (1 - g)^2 / (2 - 2 g + g^2),
    a bias of about -g.  G-JF: v' = a v + (b/m) beta with a = (1 - x) / (1 + x),
    b = 1 / (1 + x), x = alpha dt / 2m: exactly kB T / m; g-BAOAB's O step
    likewise."""
    kT = S.KB_KCAL * d.temperature
    if d.integrator in ("G-JFLangevin", "g-BAOABLangevin"):
        return kT
    g = float(np.mean(d.gamma)) * d.dt / 2
    return kT * 2 * (1 - g) ** 2 / (2 - 2 * g + g * g)


@pytest.mark.parametrize("integrator", INTEGRATORS)
def test_equipartition(integrator):
    d = _with(S.bead_fluid(n=20000, density=0.002, seed=45, dt=0.1, gamma=0.5), integrator)
    d.vel = np.zeros_like(d.vel)
    e = Engine("mixed")
    sid = e.add_system(d)
    e.commit()
    e.step(600)
    kin = []
    for _ in range(20):
        e.step(25)
        v = e.state(sid)[1]
        kin.append(0.5 * float(np.sum(d.mass[:, None] * v * v)))
    e.close()
    assert np.mean(kin) == pytest.approx(1.5 * d.n * _stationary_kT(d), rel=0.01)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("integrator", ["BAOAB", "VelocityVerlet"] + INTEGRATORS)
def test_per_particle_masses_and_frictions(integrator, precision):
    """Masses and frictions that differ per particle (the per-particle
    coefficient array) beside a system with uniform ones (coefficients held
    in the system record), each against the oracle, across a temperature
    change."""
    rng = np.random.default_rng(46)
    mixed_d = S.polymer_melt(nchains=4, nbeads=40, radius=40.0, seed=46)
    mixed_d.mass = rng.uniform(0.5, 2.0, mixed_d.n)
    mixed_d.gamma = rng.uniform(0.2, 1.5, mixed_d.n)
    uniform_d = S.polymer_melt(nchains=3, nbeads=40, radius=40.0, seed=47)
    descs = []
    for d in (mixed_d, uniform_d):
        d = d.copy()
        d.integrator = integrator
        if integrator == "VelocityVerlet":
            d.dt = 0.005
        descs.append(d)
    e = Engine(precision)
    sids = [e.add_system(d) for d in descs]
    e.commit()
    e.step(30)
    if integrator != "VelocityVerlet":
        for sid in sids:
            e.set_temperature(sid, 380.0)
    e.step(30)
    for d, sid in zip(descs, sids):
        o = oracle.Oracle(d)
        o.init_dynamics()
        o.run(30)
        if integrator != "VelocityVerlet":
            o.set_temperature(380.0)
        o.run(30)
        po, vo, _ = o.state()
        p, v, _ = e.state(sid)
        assert np.abs(p - po).max() <= TOL[precision], (integrator, precision)
        assert np.abs(v - vo).max() <= 10 * TOL[precision], (integrator, precision)
    e.close()
