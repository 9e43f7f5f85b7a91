"""UnderdampedLangevin on the GPU against the oracle (the same Philox noise
stream, so the trajectories agree to the precision's tolerance), across a
checkpoint, a temperature change, and mixed with the other integrators in one
arena."""
import numpy as np
import pytest

import oracle
from mjolnir_b200 import systems as S
from mjolnir_b200.engine import Engine

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-9, "mixed": 1e-5}


def _underdamped(d, gamma=None):
    d = d.copy()
    d.integrator = "UnderdampedLangevin"
    if gamma is not None:
        d.gamma = gamma
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
    "melt": lambda: _underdamped(S.polymer_melt(nchains=6, nbeads=60, radius=60.0, seed=41)),
    "fluid": lambda: _underdamped(S.bead_fluid(n=3000, density=0.003, seed=42, dt=0.2, gamma=0.7)),
    "lj": lambda: _underdamped(S.lj_fluid(n=729, density=0.8, margin=0.3, seed=43)),
}


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", sorted(CASES))
def test_matches_oracle_noise_stream(name, precision):
    d = CASES[name]()
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
def test_steps_in_chunks_equal_one_run(precision):
    """The closing half of a chunk's last step and the next chunk's first
    pass (the fused kick) give the same trajectory as one long chunk."""
    d = CASES["melt"]()
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
        assert np.array_equal(a, b), precision


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_temperature_change_matches_oracle(precision):
    d = CASES["melt"]()
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
    """BAOAB, velocity Verlet and UnderdampedLangevin systems side by side,
    each against its own oracle run."""
    descs = []
    for k, kind in enumerate(("BAOAB", "UnderdampedLangevin", "VelocityVerlet", "UnderdampedLangevin")):
        d = S.polymer_melt(nchains=4, nbeads=50, radius=50.0, seed=44 + k)
        d.integrator = kind
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


def test_checkpoint_restart_is_bit_exact(tmp_path):
    """Interrupted at step 70 and resumed in a new engine from the checkpoint
    files: the acceleration is rebuilt from the saved forces and the noise of
    step 70, and the run ends bit for bit where the uninterrupted run does
    (mixed form: its force sums do not depend on the list order)."""
    from mjolnir_b200 import checkpoint as K
    d = CASES["fluid"]()
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
    """kB T times the stationary <m v^2> / kB T of the scheme for a free
    particle: with g = gamma dt / 2 the update is v' = c v + (dt/2)(1 - g)
    (a + a'), c = (1 - g)((1 - g)^2 + g), whose variance is
    kB T / m * 2 (1 - g)^2 / (2 - 2 g + g^2) (a discretisation bias of -g)."""
    g = float(np.mean(d.gamma)) * d.dt / 2
    return S.KB_KCAL * d.temperature * 2 * (1 - g) ** 2 / (2 - 2 * g + g * g)


def test_equipartition():
    d = _underdamped(S.bead_fluid(n=20000, density=0.002, seed=45, dt=0.1, gamma=0.5))
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
