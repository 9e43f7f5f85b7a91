"""A system read from a Mjolnir input file runs exactly like the same system
handed to the engine directly, and the runner writes the energy file."""
import numpy as np
import pytest

from mjolnir_b200 import input as I
from mjolnir_b200 import systems as S
from mjolnir_b200.__main__ import run
from mjolnir_b200.engine import Engine

pytestmark = pytest.mark.gpu


def test_toml_run_matches_direct(tmp_path):
    d = S.polymer_melt(nchains=4, nbeads=50, radius=45.0, seed=21)
    path = str(tmp_path / "melt.toml")
    I.dump(d, path, total_step=40, save_step=20, prefix="melt")
    text = open(path).read().replace('output.path = "./"', f'output.path = "{tmp_path}/"')
    open(path, "w").write(text)
    res = run(path, precision="mixed")
    unit_line, head = open(res["energy_file"]).readlines()[:2]
    assert unit_line == "# unit of length : angstrom, unit of energy : kcal/mol\n"
    assert head.split() == ["#", "timestep", "BondLength:Harmonic", "BondAngle:Harmonic",
                            "DihedralAngle:Cosine", "GlobalPairExcludedVolume", "Pair:DebyeHuckel",
                            "kinetic_energy", "attribute:ionic_strength", "attribute:temperature"]
    ene = np.loadtxt(res["energy_file"])
    assert ene.shape == (3, 9)                       # steps 0, 20, 40; 5 terms, kinetic, 2 attributes
    assert list(ene[:, 0]) == [0, 20, 40]
    assert ene[0, 8] == d.temperature and ene[0, 7] > 0
    e = Engine("mixed")
    sid = e.add_system(d)
    e.commit()
    e.step(40)
    en = e.energies(sid)
    row = ene[-1]
    for k, t in enumerate(("bond", "angle", "dihedral", "exv", "dh")):
        assert row[1 + k] == pytest.approx(en[t], rel=1e-6, abs=1e-6)    # six decimals
    p, v, _ = e.state(sid)
    kin = 0.5 * float(np.sum(d.mass[:, None] * v * v))
    assert row[6] == pytest.approx(kin, rel=1e-6, abs=1e-6)
    xyz = open(res["trajectory"]).read().split("\n")
    assert xyz[0] == str(d.n) and xyz[1] == "step = 0" and xyz[2].startswith("X ")
    from mjolnir_b200 import checkpoint as K
    ck = K.read_system(str(tmp_path / "melt_system.msg"))           # the last checkpoint: step 40
    assert np.array_equal(ck["pos"], p) and K.read_rng(str(tmp_path / "melt_rng.msg"))[1] == 40
    e.close()


@pytest.mark.parametrize("desc", [S.polymer_melt(nchains=3, nbeads=60, radius=45.0, seed=23),
                                  S.bead_fluid(n=2000, density=0.003, seed=24, dt=0.3)])
def test_checkpoint_restart_is_bit_exact(desc, tmp_path):
    """A run interrupted by a checkpoint and resumed in a new engine ends in
    the same state, bit for bit (mixed form), as the uninterrupted run."""
    from mjolnir_b200 import checkpoint as K
    e = Engine("mixed")
    sid = e.add_system(desc)
    e.commit()
    e.step(70)
    K.save(e, sid, desc, str(tmp_path / "ck"))
    e.step(90)
    ref = e.state(sid)
    e.close()
    r = K.restore(str(tmp_path / "ck"), desc)
    e2 = Engine("mixed")
    sid2 = e2.add_system(r)
    e2.commit()
    assert e2.step_count(sid2) == 70
    e2.step(90)
    got = e2.state(sid2)
    e2.close()
    for a, b in zip(got, ref):
        assert np.array_equal(a, b)


def test_runner_writes_dcd_and_trr(tmp_path):
    """format = ["xyz", "dcd", "trr"]: every file is written, the DCD frames
    are the engine's states in single precision and the last TRR frame is
    the engine's final state (mixed form: the chunking of the run does not
    change a bit)."""
    import struct
    d = S.bead_fluid(n=1500, density=0.003, seed=25, dt=0.2)
    path = str(tmp_path / "f.toml")
    I.dump(d, path, total_step=30, save_step=10, prefix="f")
    text = open(path).read().replace('output.path = "./"', f'output.path = "{tmp_path}/"')
    text = text.replace('output.format = "xyz"', 'output.format = ["xyz", "dcd", "trr"]')
    open(path, "w").write(text)
    res = run(path, precision="mixed")
    assert res["formats"] == ["xyz", "dcd", "trr"]
    e = Engine("mixed")
    sid = e.add_system(d)
    e.commit()
    e.step(30)
    p, v, f = e.state(sid)
    nmol = e.molecule_count(sid)
    e.close()
    raw = open(res["trr"], "rb").read()
    title = str(tmp_path / "f").encode()
    frame = 12 + len(title) + 52 + 16 + 72 + 3 * 24 * d.n
    assert len(raw) == 4 * frame                       # steps 0, 10, 20, 30
    last = raw[3 * frame:]
    assert struct.unpack("<i", last[12 + len(title) + 44:12 + len(title) + 48])[0] == 30
    data = np.frombuffer(last[12 + len(title) + 52 + 16 + 72:], dtype="<f8").reshape(3, d.n, 3)
    assert np.array_equal(data[0], p) and np.array_equal(data[1], v) and np.array_equal(data[2], f)
    dcd = open(res["dcd"], "rb").read()
    assert nmol == 1                                 # the fluid's single-molecule trick
    assert struct.unpack("<5i", dcd[8:28]) == (4, 0, 10, 30, d.n)   # the input file has no bonds
    tail = dcd[-3 * (4 * d.n + 8):]
    for k in range(3):
        xs = np.frombuffer(tail[k * (4 * d.n + 8) + 4:(k + 1) * (4 * d.n + 8) - 4], dtype="<f4")
        assert np.array_equal(xs, p[:, k].astype(np.float32))
