"""The allocation-free ExcludedVolume entry point against the context path.

mjg_exv_force_noalloc exists for callers that may not allocate device memory
(a host that owns every allocation through its own pool, an embedding that
forbids cudaMalloc after start-up): they hand over device buffers they already
own and get forces and energy back without the library allocating anything.
This test plays such a caller -- it owns the device buffers (torch allocates
them, standing in for the host's pool) -- and compares two calls in a row,
on two different systems so that the shared scratch array is reused, with
mjg_term_force(MJG_TERM_EXV) of an FP64 context holding the same system.
Tolerances are the FP64 ones of the parity tests: forces 1e-12 relative RMS,
energy 1e-12 relative.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import rel_rms
from mjolnir_b200 import _capi as A
from mjolnir_b200 import systems as S
from mjolnir_b200.engine import Engine

pytestmark = pytest.mark.gpu


def context_exv(d):
    e = Engine("fp64")
    sid = e.add_system(d)
    e.commit()
    f, en = e.term_force(sid, "exv")
    e.close()
    return f, en


def noalloc_exv(d):
    import torch
    dev = torch.device("cuda", 0)
    pos = torch.tensor(np.ascontiguousarray(d.pos), dtype=torch.float64, device=dev)
    radius = torch.zeros(d.n, dtype=torch.float64, device=dev)
    radius[torch.as_tensor(d.exv.idx, device=dev)] = torch.tensor(d.exv.param0, dtype=torch.float64, device=dev)
    force = torch.full((d.n, 3), float("nan"), dtype=torch.float64, device=dev)
    energy = torch.full((1,), float("nan"), dtype=torch.float64, device=dev)
    lower = (C.c_double * 3)(*d.lower)
    upper = (C.c_double * 3)(*d.upper)
    stream = torch.cuda.current_stream(dev).cuda_stream
    code = A.lib().mjg_exv_force_noalloc(
        d.n, A.PERIODIC_CUBOID if d.periodic else A.UNLIMITED, lower, upper,
        pos.data_ptr(), radius.data_ptr(), float(d.exv.epsilon), float(d.exv.cutoff),
        force.data_ptr(), energy.data_ptr(), stream)
    assert code == A.OK
    torch.cuda.synchronize(dev)
    return force.cpu().numpy(), float(energy.cpu()[0])


def test_noalloc_matches_context_two_calls():
    # a periodic EXV fluid, then an unbounded one of another size: the second
    # call must not see anything the first left in the scratch array
    fluid = S.bead_fluid(n=3000, density=0.003, seed=61, dt=0.3)
    fluid.dh = None
    blob = S.bead_fluid(n=1200, density=0.004, seed=62, dt=0.3)
    blob.dh = None
    blob.boundary = "Unlimited"
    blob.pos = blob.pos - blob.pos.mean(axis=0)
    for d in (fluid, blob):
        f_ref, e_ref = context_exv(d)
        f, e = noalloc_exv(d)
        assert np.isfinite(f).all()
        assert rel_rms(f, f_ref) <= 1e-12
        assert abs(e - e_ref) <= 1e-12 * max(abs(e_ref), 1e-12)


def test_noalloc_rejects_oversize():
    lower = (C.c_double * 3)(0, 0, 0)
    upper = (C.c_double * 3)(1, 1, 1)
    code = A.lib().mjg_exv_force_noalloc(65537, A.PERIODIC_CUBOID, lower, upper, 1, 1, 0.2, 2.0, 1, 1, None)
    assert code == A.EINVAL


def test_noalloc_small_box_large_grid_and_outside_positions():
    # a periodic box narrower than three cutoffs (the grid is held at 3 cells
    # per axis), a box whose cutoff would ask for more cells than the scratch
    # array holds (the grid is shrunk to fit), and particles pushed outside
    # the box by up to a fifth of its width (their cells wrap): each against
    # the context path on the same system with the positions wrapped back
    small = S.bead_fluid(n=64, density=0.006, seed=63, dt=0.3)
    small.dh = None
    assert small.upper[0] - small.lower[0] < 3 * (2 * 2.0 * small.exv.cutoff)
    big = S.bead_fluid(n=20000, density=0.0005, seed=64, dt=0.3)
    big.dh = None
    big.exv.cutoff = 1.2                  # rc = 4.8 A: 70 cells per axis asked, 64^3 > the limit
    outside = S.bead_fluid(n=3000, density=0.003, seed=65, dt=0.3)
    outside.dh = None
    W = np.array(outside.upper) - np.array(outside.lower)
    rng = np.random.default_rng(65)
    shift = rng.integers(-1, 2, size=outside.pos.shape) * W
    near_edge = (outside.pos < outside.lower[0] + 0.2 * W) | (outside.pos > outside.upper[0] - 0.2 * W)
    moved = outside.pos + np.where(near_edge, shift, 0.0)
    moved = np.where(np.abs(moved - outside.pos.mean()) < 0.7 * W, moved, outside.pos)
    for d, tol in ((small, 1e-12), (big, 1e-12)):
        f_ref, e_ref = context_exv(d)
        f, e = noalloc_exv(d)
        assert rel_rms(f, f_ref) <= tol
        assert abs(e - e_ref) <= tol * max(abs(e_ref), 1e-12)
    f_ref, e_ref = context_exv(outside)
    out = outside.copy()
    out.pos = moved
    assert (moved < outside.lower[0]).any() or (moved >= outside.upper[0]).any()
    f, e = noalloc_exv(out)
    assert rel_rms(f, f_ref) <= 1e-10       # displacements taken across a shift round differently
    assert abs(e - e_ref) <= 1e-10 * abs(e_ref)


def test_noalloc_allocates_nothing_per_call():
    import torch
    d = S.bead_fluid(n=2000, density=0.003, seed=66, dt=0.3)
    d.dh = None
    noalloc_exv(d)                        # the first call may load the module holding the array
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    for _ in range(3):
        noalloc_exv(d)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0
