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
    head = open(res["energy_file"]).readline()
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
