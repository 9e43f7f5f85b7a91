"""The CUDA path on the edge systems of tests/edge_systems.py against the
oracle (which tests/test_oracle_edges.py pins to the reference): lists bit
for bit, forces and energies within the form's tolerance, and 200 steps of
dynamics that stay finite and keep the lists exact."""
import numpy as np
import pytest

import oracle
from conftest import rel_rms
from edge_systems import CASES
from mjolnir_b200.engine import Engine

pytestmark = pytest.mark.gpu

FORCE_TOL = {"fp64": 1e-12, "mixed": 1e-5}


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", sorted(CASES))
def test_edges_against_oracle(name, precision):
    d = CASES[name]()
    o = oracle.Oracle(d)
    e = Engine(precision)
    sid = e.add_system(d)
    e.commit()
    p = e.positions(sid)                         # wrapped into the box like the reference
    for t in ("exv", "dh", "lj"):
        term = getattr(d, t)
        if term is None or len(term.idx) == 0:
            continue
        assert np.array_equal(e.neighbors(sid, t), o.neighbors(t, p)), (name, t)
        f, en = e.term_force(sid, t)
        fo, eo = o.term_force(t, p)
        if np.abs(fo).max() > 0:
            assert rel_rms(f, fo) <= FORCE_TOL[precision], (name, t, rel_rms(f, fo))
        else:
            assert np.abs(f).max() == 0
        assert abs(en - eo) <= FORCE_TOL[precision] * max(abs(eo), 1e-12), (name, t, en, eo)
    e.step(200)
    e.rebuild()                                  # lists at the current coordinates
    p, v, f = e.state(sid)
    assert np.all(np.isfinite(p)) and np.all(np.isfinite(v))
    for t in ("exv", "dh", "lj"):
        term = getattr(d, t)
        if term is not None and len(term.idx) > 0:
            assert np.array_equal(e.neighbors(sid, t), o.neighbors(t, p)), (name, t, "after dynamics")
    e.close()
