"""Half Verlet lists of the mixed form (`mjg_set_half_lists`): each pair is
stored in the list of its lower slot, and the force launch adds the negated
fixed-point pair force to the partner.  The integer sums are the full lists'
sums, so every result is the full lists' result bit for bit: forces,
trajectories through list rebuilds and rollbacks, the exported pairs
(SpatialPartition::neighbors' half list, core/NeighborList.hpp:151-266) and
the energies (to FP64 summation order, 1e-10), over every force-launch schedule,
every potential of the three global terms and the cell-list edge cases."""
import numpy as np
import pytest

import edge_systems as E
from exv_family import CASES as EXV_CASES, system as exv_system
from lj_family import KINDS as LJ_KINDS, fluid as lj_fluid_kind
from mjolnir_b200 import _capi as A
from mjolnir_b200 import systems as S
from mjolnir_b200.engine import Engine

pytestmark = pytest.mark.gpu

GLOBAL = ("exv", "dh", "lj")


def terms_of(d):
    return [t for t in GLOBAL if getattr(d, t) is not None and len(getattr(d, t).idx) > 0]


def run(descs, half, schedule=0, tpp=1, steps=30, capacity=None):
    e = Engine("mixed")
    ids = [e.add_system(d) for d in descs]
    e.commit()
    present = sorted({t for d in descs for t in terms_of(d)})
    for t in GLOBAL:
        e.set_pair_schedule(t, schedule)
        if t in present:
            e.set_threads_per_particle(t, tpp)
        e.set_half_lists(t, half)
        assert e.get_half_lists(t) == half
    out = {"nbr": [], "force": [], "energy": []}
    for sid, d in zip(ids, descs):
        for t in terms_of(d):
            out["nbr"].append(e.neighbors(sid, t))
            out["force"].append(e.term_force(sid, t)[0])
        out["energy"].append(e.energies(sid))
    if capacity is not None:            # the next rebuild overflows, rolls back and grows the lists
        for t in present:
            e.debug_set_list_capacity(t, capacity)
    e.step(steps)
    out["state"] = [e.state(sid)[:2] for sid in ids]
    out["after"] = [e.neighbors(sid, t) for sid, d in zip(ids, descs) for t in terms_of(d)]
    e.close()
    return out


def same(a, b, what):
    for x, y in zip(a["nbr"], b["nbr"]):
        assert np.array_equal(x, y), what
    for x, y in zip(a["after"], b["after"]):
        assert np.array_equal(x, y), what
    for x, y in zip(a["force"], b["force"]):
        assert np.array_equal(x, y), what
    for x, y in zip(a["state"], b["state"]):
        assert np.array_equal(x[0], y[0]) and np.array_equal(x[1], y[1]), what
    # energies: FP64 sums added with atomics in arrival order (a DebyeHuckel
    # energy of cancelling charges keeps ~1e-13 of that order)
    for x, y in zip(a["energy"], b["energy"]):
        for k in x:
            assert abs(x[k] - y[k]) <= 1e-10 * max(abs(y[k]), 1e-12), (what, k, x[k], y[k])


MIXED = [S.polymer_melt(nchains=4, nbeads=60, radius=45.0, seed=41),
         S.bead_fluid(n=3000, density=0.003, seed=42, dt=0.3),
         S.lj_fluid(n=512, seed=43)]


@pytest.mark.parametrize("schedule,tpp", [(0, 1), (0, 4), (0, 32), (1, 1), (1, 16), (2, 2), (3, 4),
                                          (4, 2), (4, 16), (4, 32), (5, 8), (5, 32)])
def test_half_lists_equal_full_lists_every_schedule(schedule, tpp):
    ref = run(MIXED, False, 0, 1)
    got = run(MIXED, True, schedule, tpp)
    same(got, ref, (schedule, tpp))


@pytest.mark.parametrize("kind", LJ_KINDS)
def test_half_lists_lj_family(kind):
    d = lj_fluid_kind(kind)
    same(run([d], True, 2, 2, steps=100), run([d], False, steps=100), kind)


@pytest.mark.parametrize("periodic", [True, False])
@pytest.mark.parametrize("case", EXV_CASES)
def test_half_lists_exv_family(case, periodic):
    d = exv_system(case, periodic)
    same(run([d], True, 4, 2, steps=100), run([d], False, steps=100), (case, periodic))


@pytest.mark.parametrize("name", sorted(E.CASES))
def test_half_lists_edge_systems(name):
    d = E.CASES[name]()
    same(run([d], True, 3, 2, steps=50), run([d], False, steps=50), name)


def test_half_lists_through_overflow_rollback():
    """Lists that overflow a capacity of 8 words roll the chunk back and grow;
    the half lists' run is the full lists' run."""
    d = S.lj_fluid(n=1000, density=0.8, seed=44)
    same(run([d], True, 0, 1, steps=300, capacity=8), run([d], False, steps=300), "rollback")


def test_half_lists_in_a_batch_with_frozen_and_retired_systems():
    """Systems added, frozen and retired between chunks: the half lists
    follow the arena's changes like the full ones."""
    descs = [S.polymer_melt(nchains=2, nbeads=50, radius=30.0, seed=50 + k) for k in range(4)]
    states = {}
    for half in (False, True):
        e = Engine("mixed")
        ids = [e.add_system(d) for d in descs[:3]]
        e.commit()
        for t in ("exv", "dh"):
            e.set_half_lists(t, half)
        e.step(40)
        e.freeze(ids[1])
        e.step(40)
        e.remove_system(ids[0])
        ids.append(e.add_system(descs[3]))
        e.commit()
        e.freeze(ids[1], False)
        e.step(40)
        states[half] = [e.state(sid)[:2] for sid in ids[1:]]
        e.close()
    for x, y in zip(states[True], states[False]):
        assert np.array_equal(x[0], y[0]) and np.array_equal(x[1], y[1])


def test_half_lists_need_the_mixed_form():
    e = Engine("fp64")
    e.add_system(MIXED[0])
    e.commit()
    with pytest.raises(A.MjgError):
        e.set_half_lists("exv", True)
    assert not e.get_half_lists("exv")
    e.close()
