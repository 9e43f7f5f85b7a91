"""The oracle's Lennard-Jones family (WCA, LennardJonesAttractive,
UniformLennardJones through the generic pair loop) against the reference's
own potentials: lists, forces and both energy paths (calc_force_and_energy,
where pairs with zero force add nothing, and calc_energy over every listed
pair)."""
import numpy as np
import pytest

import oracle
from lj_family import KINDS, fluid

needs_ref = pytest.mark.skipif(not oracle.reference_available(), reason="reference driver not built")


@needs_ref
@pytest.mark.parametrize("kind", KINDS)
def test_family_matches_reference(kind):
    d = fluid(kind)
    o = oracle.Oracle(d)
    r = oracle.Reference(d)
    r.initialize()
    p, _, _ = r.state()
    assert np.array_equal(o.neighbors("lj", p), r.neighbors("lj"))
    fo, eo = o.term_force("lj", p)
    fr, er = r.term_force("lj")
    assert np.abs(fr).max() > 0
    assert np.abs(fo - fr).max() <= 1e-14 * np.abs(fr).max(), kind
    assert eo == pytest.approx(er, rel=1e-14, abs=1e-300)
    assert o.term_energy("lj", p) == pytest.approx(r.term_energy("lj"), rel=1e-14, abs=1e-300)
    r.close()


def test_attractive_energy_paths_differ():
    # pairs closer than 2^(1/6) sigma have zero force: the force pass skips
    # them, calc_energy adds -epsilon for each
    d = fluid("LennardJonesAttractive", density=0.9)
    o = oracle.Oracle(d)
    _, e_force_pass = o.term_force("lj", d.pos)
    e_calc = o.term_energy("lj", d.pos)
    assert e_calc < e_force_pass
