"""The ExcludedVolume family (InversePower, HardCoreExcludedVolume) on the
GPU against the oracle (pinned to the reference by
tests/test_oracle_exv_family.py)."""
import numpy as np
import pytest

import oracle
from conftest import rel_rms
from exv_family import CASES, system
from mjolnir_b200.engine import Engine

pytestmark = pytest.mark.gpu
TOL = {"fp64": 1e-12, "mixed": 1e-5}


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("periodic", [True, False])
@pytest.mark.parametrize("case", CASES)
def test_family_against_oracle(case, periodic, precision):
    d = system(case, periodic)
    o = oracle.Oracle(d)
    e = Engine(precision)
    sid = e.add_system(d)
    e.commit()
    p = e.positions(sid)
    assert np.array_equal(e.neighbors(sid, "exv"), o.neighbors("exv", p))
    f, en = e.term_force(sid, "exv")
    fo, eo = o.term_force("exv", p)
    assert rel_rms(f, fo) <= TOL[precision], (case, rel_rms(f, fo))
    assert abs(en - eo) <= TOL[precision] * max(abs(eo), 1e-12), (case, en, eo)
    ec = e.energies(sid)["exv"]
    eco = o.term_energy("exv", p)
    assert abs(ec - eco) <= TOL[precision] * max(abs(eco), 1e-12), (case, ec, eco)
    e.step(200)
    e.rebuild()
    p = e.positions(sid)
    assert np.all(np.isfinite(p))
    assert np.array_equal(e.neighbors(sid, "exv"), o.neighbors("exv", p))
    e.close()
