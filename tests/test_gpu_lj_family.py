"""The Lennard-Jones family on the GPU against the oracle (pinned to the
reference by tests/test_oracle_lj_family.py): lists bit for bit, forces and
both energy paths within the form's tolerance, and dynamics that keep the
lists exact."""
import numpy as np
import pytest

import oracle
from conftest import rel_rms
from lj_family import KINDS, fluid
from mjolnir_b200.engine import Engine

pytestmark = pytest.mark.gpu
TOL = {"fp64": 1e-12, "mixed": 1e-5}


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("kind", KINDS)
def test_family_against_oracle(kind, precision):
    d = fluid(kind)
    o = oracle.Oracle(d)
    e = Engine(precision)
    sid = e.add_system(d)
    e.commit()
    p = e.positions(sid)
    assert np.array_equal(e.neighbors(sid, "lj"), o.neighbors("lj", p))
    f, en = e.term_force(sid, "lj")
    fo, eo = o.term_force("lj", p)
    assert rel_rms(f, fo) <= TOL[precision], (kind, rel_rms(f, fo))
    assert abs(en - eo) <= TOL[precision] * max(abs(eo), 1e-12), (kind, en, eo)
    ec = e.energies(sid)["lj"]
    eco = o.term_energy("lj", p)
    assert abs(ec - eco) <= TOL[precision] * max(abs(eco), 1e-12), (kind, ec, eco)
    e.step(300)
    e.rebuild()
    p = e.positions(sid)
    assert np.all(np.isfinite(p))
    assert np.array_equal(e.neighbors(sid, "lj"), o.neighbors("lj", p))
    e.close()
