"""The oracle's ExcludedVolume family (InversePower, HardCoreExcludedVolume
through the generic pair loop) against the reference's own potentials."""
import numpy as np
import pytest

import oracle
from exv_family import CASES, system

needs_ref = pytest.mark.skipif(not oracle.reference_available(), reason="reference driver not built")


@needs_ref
@pytest.mark.parametrize("periodic", [True, False])
@pytest.mark.parametrize("case", CASES)
def test_family_matches_reference(case, periodic):
    d = system(case, periodic)
    o = oracle.Oracle(d)
    r = oracle.Reference(d)
    r.initialize()
    p, _, _ = r.state()
    assert np.array_equal(o.neighbors("exv", p), r.neighbors("exv"))
    fo, eo = o.term_force("exv", p)
    fr, er = r.term_force("exv")
    assert np.abs(fr).max() > 0
    assert np.abs(fo - fr).max() <= 1e-14 * np.abs(fr).max(), case
    assert eo == pytest.approx(er, rel=1e-14, abs=1e-300)
    assert o.term_energy("exv", p) == pytest.approx(r.term_energy("exv"), rel=1e-14, abs=1e-300)
    r.close()
