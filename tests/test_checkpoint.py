"""Checkpoints in the reference's MsgPack layout: files written here are the
bytes the reference's MsgPackSaver writes for the same state, the reference's
MsgPackLoader reads them, files the reference writes are read here, and a
checkpoint restarts a TOML input."""
import os

import numpy as np
import pytest

import oracle
from conftest import golden_cases
from mjolnir_b200 import checkpoint as K
from mjolnir_b200 import input as I
from mjolnir_b200 import systems as S

CASES = golden_cases()
needs_ref = pytest.mark.skipif(not oracle.reference_available(), reason="reference driver not built")


def _state(d):
    r = oracle.Reference(d)
    r.initialize()                      # wraps positions, computes forces
    p, v, f = r.state()
    return r, p, v, f


@needs_ref
@pytest.mark.parametrize("name", sorted(CASES))
def test_bytes_identical_to_reference_saver(name, tmp_path):
    d, _ = CASES[name]
    r, p, v, f = _state(d)
    r.save_msgpack(str(tmp_path / "ref"))
    ours = K.system_bytes(p, v, f, d.mass, d.periodic, d.lower, d.upper,
                          {"temperature": d.temperature, "ionic_strength": d.ionic_strength})
    theirs = open(tmp_path / "ref_system.msg", "rb").read()
    assert ours == theirs
    r.close()


@needs_ref
def test_reference_loader_reads_our_file(tmp_path):
    d, _ = CASES["polymer_small"]
    rng = np.random.default_rng(5)
    f = rng.normal(size=d.pos.shape)
    path = str(tmp_path / "x_system.msg")
    K.write_system(path, d.pos, d.vel, f, d.mass, d.periodic, d.lower, d.upper,
                   {"temperature": 310.0, "ionic_strength": 0.2})
    got = oracle.Reference.load_msgpack(path, d.periodic)
    assert np.array_equal(got["pos"], d.pos) and np.array_equal(got["vel"], d.vel)
    assert np.array_equal(got["force"], f) and np.array_equal(got["mass"], d.mass)
    assert (got["temperature"], got["ionic_strength"]) == (310.0, 0.2)


@needs_ref
def test_we_read_reference_file(tmp_path):
    d, _ = CASES["fluid_small"]
    r, p, v, f = _state(d)
    r.save_msgpack(str(tmp_path / "ref"))
    got = K.read_system(str(tmp_path / "ref_system.msg"))
    assert got["periodic"] and got["lower"] == tuple(d.lower) and got["upper"] == tuple(d.upper)
    assert np.array_equal(got["pos"], p) and np.array_equal(got["vel"], v) and np.array_equal(got["force"], f)
    assert got["names"][0] == "X" and got["groups"][0] == "NONE"
    assert got["attributes"] == {"ionic_strength": d.ionic_strength, "temperature": d.temperature}
    r.close()


def test_round_trip_and_rng(tmp_path):
    d = S.polymer_melt(nchains=2, nbeads=20, radius=30.0, seed=9)
    path = str(tmp_path / "a_system.msg")
    K.write_system(path, d.pos, d.vel, np.zeros_like(d.pos), d.mass, False, attributes={"temperature": 300.0})
    got = K.read_system(path)
    assert not got["periodic"] and np.array_equal(got["pos"], d.pos)
    K.write_rng(str(tmp_path / "a_rng.msg"), 9, 12345)
    assert K.read_rng(str(tmp_path / "a_rng.msg")) == (9, 12345)
    out = K.restore(str(tmp_path / "a"), d)
    assert out.start_step == 12345 and np.array_equal(out.pos, d.pos)
    with pytest.raises(K.CheckpointError):
        K.restore(str(tmp_path / "a"), S.polymer_melt(nchains=3, nbeads=20, radius=30.0, seed=9))
    (tmp_path / "bad.msg").write_bytes(b"\x81\xa1x\x01")
    with pytest.raises(K.CheckpointError):
        K.read_system(str(tmp_path / "bad.msg"))


def test_toml_restarts_from_checkpoint(tmp_path):
    d = S.polymer_melt(nchains=2, nbeads=20, radius=30.0, seed=9)
    I.dump(d, str(tmp_path / "in.toml"))
    moved = d.pos + 0.25
    K.write_system(str(tmp_path / "ck_system.msg"), moved, -d.vel, np.zeros_like(d.pos), d.mass, False,
                   attributes={"temperature": 320.0, "ionic_strength": 0.05})
    text = open(tmp_path / "in.toml").read()
    start = text.index("[[systems]]")
    end = text.index("[[forcefields]]")
    text = (text[:start] + '[[systems]]\nfile_name = "ck_system.msg"\n\n' + text[end:]).replace(
        "[files]", f'[files]\ninput.path = "{tmp_path}/"')
    open(tmp_path / "restart.toml", "w").write(text)
    g = I.load(str(tmp_path / "restart.toml")).desc
    assert np.array_equal(g.pos, moved) and np.array_equal(g.vel, -d.vel)
    assert g.temperature == 320.0 and g.ionic_strength == 0.05
    np.testing.assert_array_equal(g.bonds[0], d.bonds[0])
