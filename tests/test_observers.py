"""The trajectory and energy writers against the reference's own observers.

The reference (compiled from its sources) runs a velocity-Verlet trajectory
with its XYZ, DCD, TRR and energy observers through the call sequence of
MolecularDynamicsSimulator; the oracle, bit-exact with the reference on that
trajectory, feeds the same frames to :mod:`mjolnir_b200.observers`.  The files
must be equal byte for byte, except the 80-byte DCD title record, which names
this library."""
import os
import struct

import numpy as np
import pytest

import oracle
from mjolnir_b200 import observers as O
from mjolnir_b200 import systems as S
from mjolnir_b200.__main__ import present_terms

needs_ref = pytest.mark.skipif(not oracle.reference_available(),
                               reason="reference driver not built (no reference tree)")

FORMATS = ["xyz", "dcd", "trr"]
DCD_TITLE = slice(100, 180)       # 4 + 84 + 4 bytes of the first record, 4 + 4 into the second


def _files(prefix):
    return [prefix + s for s in (".ene", "_position.xyz", "_velocity.xyz", "_position.dcd",
                                 "_velocity.dcd", ".trr")]


def _frame(o, d, terms, molecules):
    p, v, f = o.state()
    return O.Frame(pos=p, vel=v, force=f, mass=d.mass,
                   energies=[(title, o.term_energy(key, p)) for key, title in terms],
                   attributes={"temperature": d.temperature, "ionic_strength": d.ionic_strength},
                   periodic=d.periodic, width=tuple(u - lo for u, lo in zip(d.upper, d.lower)),
                   molecules=molecules)


def _ours(d, prefix, total, save):
    o = oracle.Oracle(d)
    o.init_dynamics()
    terms = present_terms(d)
    molecules = int(o.molecules().max()) + 1
    obs = O.make(FORMATS, prefix)
    fr = _frame(o, d, terms, molecules)
    for ob in obs:
        ob.initialize(total, save, d.dt, fr)
    for st in range(total):
        if st % save == 0:
            fr = _frame(o, d, terms, molecules)
            for ob in obs:
                ob.output(st, d.dt, fr)
        o.run(1)
    fr = _frame(o, d, terms, molecules)
    for ob in obs:
        ob.output(total, d.dt, fr)
    for ob in obs:
        ob.finalize(total, d.dt, fr)


CASES = {
    "melt": lambda: S.polymer_melt(nchains=3, nbeads=12, radius=25.0, seed=61),
    "fluid": lambda: S.bead_fluid(n=300, density=0.003, seed=62, dt=0.05),
    "lj": lambda: S.lj_fluid(n=216, density=0.7, margin=0.3, seed=63),
}


@needs_ref
@pytest.mark.parametrize("name", sorted(CASES))
def test_files_identical_to_reference_observers(name, tmp_path):
    d = CASES[name]()
    d.integrator = "VelocityVerlet"
    d.dt = min(d.dt, 0.005)
    total, save = 23, 5
    prefix = str(tmp_path / "out")
    r = oracle.Reference(d)
    r.initialize()
    r.observe(prefix, FORMATS, total, save, d.dt)
    ref = {p: open(p, "rb").read() for p in _files(prefix)}
    _ours(d, prefix, total, save)
    for p in _files(prefix):
        got = open(p, "rb").read()
        want = ref[p]
        assert len(got) == len(want), os.path.basename(p)
        if p.endswith(".dcd"):
            got = got[:DCD_TITLE.start] + got[DCD_TITLE.stop:]
            want = want[:DCD_TITLE.start] + want[DCD_TITLE.stop:]
        assert got == want, os.path.basename(p)


def test_dcd_layout(tmp_path):
    """The DCD records parse back to the frames written: CORD header with the
    frame count patched at finalize, the unit cell in the position file only."""
    d = S.bead_fluid(n=50, density=0.003, seed=64)
    rng = np.random.default_rng(0)
    frames = [O.Frame(pos=rng.normal(size=(50, 3)), vel=rng.normal(size=(50, 3)), force=np.zeros((50, 3)),
                      mass=d.mass, periodic=True, width=(11.0, 12.0, 13.0), molecules=7) for _ in range(3)]
    ob = O.DCDObserver(str(tmp_path / "t"))
    ob.initialize(30, 10, 0.25, frames[0])
    for k, fr in enumerate(frames):
        ob.output(10 * k, 0.25, fr)
    ob.finalize(30, 0.25, frames[-1])
    raw = open(str(tmp_path / "t_position.dcd"), "rb").read()
    assert raw[4:8] == b"CORD"
    nframes, first, interval, total, chains = struct.unpack("<5i", raw[8:28])
    assert (nframes, first, interval, total, chains) == (3, 0, 10, 30, 7)
    assert struct.unpack("<f", raw[44:48])[0] == 0.25 and struct.unpack("<i", raw[48:52])[0] == 1
    off = 92 + 92 + 12
    for fr in frames:
        assert struct.unpack("<i6di", raw[off:off + 56])[1:7] == (11.0, 90.0, 12.0, 90.0, 90.0, 13.0)
        off += 56
        for k in range(3):
            n = struct.unpack("<i", raw[off:off + 4])[0]
            xs = np.frombuffer(raw[off + 4:off + 4 + n], dtype="<f4")
            assert np.array_equal(xs, fr.pos[:, k].astype(np.float32))
            off += n + 8
    assert off == len(raw)
    vel = open(str(tmp_path / "t_velocity.dcd"), "rb").read()
    assert len(vel) == 92 + 92 + 12 + 3 * 3 * (200 + 8)


def test_trr_float_real_type(tmp_path):
    fr = O.Frame(pos=np.ones((4, 3)), vel=np.zeros((4, 3)), force=np.full((4, 3), 2.0), mass=np.ones(4))
    ob = O.TRRObserver(str(tmp_path / "t"), real="f4")
    ob.output(12, 0.5, fr)
    raw = open(str(tmp_path / "t.trr"), "rb").read()
    title = str(tmp_path / "t").encode()
    assert struct.unpack("<3i", raw[:12]) == (1993, 13, len(title))
    head = struct.unpack("<13i", raw[12 + len(title):12 + len(title) + 52])
    assert head[2] == 0 and head[7:12] == (48, 48, 48, 4, 12)
    assert len(raw) == 12 + len(title) + 52 + 8 + 3 * 48


def test_energy_kinetic_sum_is_sequential():
    v = np.array([[1e8, 0, 0], [1.0, 0, 0], [-1e8, 0, 0]])
    m = np.ones(3)
    # ((1e16 + 1) + 1e16) * 0.5 in particle order
    assert O.kinetic_energy(v, m) == ((1e16 + 1.0) + 1e16) * 0.5
