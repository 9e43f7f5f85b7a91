"""The C ABI from a C++ host (tests/abi_host.cpp): it builds against
include/mjolnir_b200.h and the library alone, and on a GPU it reproduces what
the Python front end computes for the same system."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from mjolnir_b200 import systems as S

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIBDIR = os.path.join(ROOT, "mjolnir_b200")


def build_host(tmp_path) -> str:
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    exe = str(tmp_path / "abi_host")
    cuda_lib = "/usr/local/cuda/lib64"
    cmd = [gxx, "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), os.path.join(HERE, "abi_host.cpp"),
           "-o", exe, os.path.join(LIBDIR, "libmjolnir_b200.so"), f"-Wl,-rpath,{LIBDIR}",
           f"-Wl,-rpath-link,{cuda_lib}", f"-L{cuda_lib}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def write_input(d, path):
    def w(f, a, dt):
        f.write(np.ascontiguousarray(np.asarray(a, dtype=dt)).tobytes())
    with open(path, "wb") as f:
        w(f, [d.n], np.int64)
        w(f, d.pos, np.float64); w(f, d.vel, np.float64); w(f, d.mass, np.float64)
        w(f, [d.temperature, d.ionic_strength, d.dt], np.float64)
        w(f, [d.seed], np.uint64)
        w(f, d.gamma, np.float64)
        for terms, ncol in ((d.bonds, 2), (d.angles, 3)):
            idx, k, v0 = terms
            w(f, [len(k)], np.int64); w(f, idx, np.int64); w(f, k, np.float64); w(f, v0, np.float64)
        idx, k, nn, v0 = d.dihedrals
        w(f, [len(k)], np.int64); w(f, idx, np.int64); w(f, k, np.float64); w(f, nn, np.int32); w(f, v0, np.float64)
        x = d.exv
        w(f, [len(x.idx)], np.int64); w(f, x.idx, np.int64); w(f, x.param0, np.float64)
        w(f, [x.epsilon, x.cutoff, x.margin], np.float64)
        q = d.dh
        w(f, [len(q.idx)], np.int64); w(f, q.idx, np.int64); w(f, q.param0, np.float64)
        w(f, [q.cutoff, q.margin], np.float64)
        w(f, [d.ignore_bond_within], np.int32)


def test_host_builds_against_the_header_and_library(tmp_path):
    exe = build_host(tmp_path)
    assert os.path.exists(exe)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_host_matches_python_front_end(precision, tmp_path):
    from mjolnir_b200.engine import Engine
    d = S.polymer_melt(nchains=5, nbeads=40, radius=45.0, seed=71)
    exe = build_host(tmp_path)
    write_input(d, str(tmp_path / "in.bin"))
    subprocess.run([exe, str(tmp_path / "in.bin"), str(tmp_path / "out.bin"),
                    "1" if precision == "mixed" else "0", "60"], check=True, timeout=300)
    out = np.fromfile(str(tmp_path / "out.bin"), dtype=np.float64)
    n = d.n
    p, v, f, e = out[:3 * n].reshape(n, 3), out[3 * n:6 * n].reshape(n, 3), out[6 * n:9 * n].reshape(n, 3), out[9 * n:]
    eng = Engine(precision)
    sid = eng.add_system(d)
    eng.commit()
    eng.step(60)
    pp, vv, ff = eng.state(sid)
    ee = eng.energies(sid)
    eng.close()
    if precision == "mixed":            # fixed-point sums: the same bits whoever calls
        assert np.array_equal(p, pp) and np.array_equal(v, vv) and np.array_equal(f, ff)
    else:                               # FP64 atomics: the same within rounding
        assert np.abs(p - pp).max() <= 1e-9 and np.abs(v - vv).max() <= 1e-8
    for k, t in enumerate(("bond", "angle", "dihedral", "exv", "dh")):
        assert e[k] == pytest.approx(ee[t], rel=1e-9, abs=1e-9), t
