"""The C-ABI library: it loads without a GPU, exports every symbol the headers
declare, refuses bad input, and its host-only builders work."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT, gpu_available
from mjolnir_b200 import _capi as A
from mjolnir_b200 import systems as S


def declared(header):
    src = open(os.path.join(ROOT, "include", header)).read()
    return set(re.findall(r"MJG(?:_SYNTH)?_API\s+[\w\s\*]+?\b(mjg_\w+)\s*\(", src))


def test_library_exports_every_declared_symbol():
    lib = A.lib()
    names = declared("mjolnir_b200.h") | declared("mjolnir_b200_synthetic.h")
    assert len(names) >= 35
    for n in sorted(names):
        assert hasattr(lib, n), n
    # and the binding covers all of them
    assert names == set(A.SIGNATURES) | set(A.SYNTH_SIGNATURES)


def test_library_is_built_for_sm100a():
    # the fatbin of the library carries sm_100a code: cuobjdump is not used;
    # the build flags are the evidence
    from mjolnir_b200 import build
    assert "arch=compute_100a,code=sm_100a" in " ".join(build.ARCH)


@pytest.mark.skipif(gpu_available(), reason="checks the no-GPU error path")
def test_context_create_fails_cleanly_without_gpu():
    h = C.c_void_p()
    code = A.lib().mjg_context_create(0, A.PRECISION_MIXED, C.byref(h))
    assert code == A.ECUDA and not h.value


def test_null_arguments_are_rejected():
    lib = A.lib()
    assert lib.mjg_context_create(0, 7, None) == A.EINVAL
    assert lib.mjg_commit(None) == A.EINVAL
    assert lib.mjg_step(None, 1) == A.EINVAL


def test_synthetic_polymer_chains():
    d = S.polymer_melt(nchains=20, nbeads=100, radius=150.0, seed=2)
    bonds = np.linalg.norm(d.pos[1:100] - d.pos[:99], axis=1)
    assert np.allclose(bonds, 3.8, atol=1e-9)
    assert (np.linalg.norm(d.pos, axis=1) <= 150.0 + 1e-9).all()
    # non-bonded beads at least 4 A apart
    from scipy.spatial import cKDTree
    pairs = cKDTree(d.pos).query_pairs(4.0 - 1e-9, output_type="ndarray")
    bonded = set(map(tuple, d.bonds[0].tolist()))
    assert all(tuple(p) in bonded for p in pairs.tolist())
    # net charge zero, 20 % charged
    assert d.dh.param0.sum() == 0 and len(d.dh.idx) == 400


def test_synthetic_fluid_min_distance():
    d = S.bead_fluid(n=5000, density=0.003, seed=3)
    L = d.upper[0]
    from scipy.spatial import cKDTree
    t = cKDTree(d.pos, boxsize=L)
    assert len(t.query_pairs(4.0 - 1e-9)) == 0
    assert d.dh.param0.sum() == 0


def test_polymer_batch_shapes():
    b = S.polymer_batch(nsys=8, seed=5)
    ns = [x.n for x in b]
    assert all(400 <= n <= 21000 for n in ns)
    assert len({x.temperature for x in b}) == 8
    assert all(280 <= x.temperature <= 360 and 0.05 <= x.ionic_strength <= 0.3 for x in b)
