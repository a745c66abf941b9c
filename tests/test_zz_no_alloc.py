"""ffs_lbm_step_noalloc against ffs_lbm_step, through the C ABI.

The no-allocation variant keeps its link table and force accumulators in a
fixed device array of the library.  Two grids start from the same state; one
is advanced with ffs_lbm_step, the other with ffs_lbm_step_noalloc, on two
calls in a row, and after each call the moments and surface forces must agree
within the parity tolerances of the step itself:
  * moments ......... max |diff| <= 2e-6
  * surface forces .. max |diff| <= 1e-4 x max |F|

Further cases: a surface large enough that the force conversion runs as its
own kernel on sums held in the fixed array; a surface whose links fill the
fixed table (status bit 2, no fault); and the entry point's main claim, that
stepping a fresh grid through it leaves the device's free memory unchanged.

This file is collected last: it must pass alone in a fresh process (the first
call on the device performs the scratch look-up) and after every other test.
"""
import ctypes as C

import numpy as np
import pytest

from freeflow_b200 import _capi as A
from freeflow_b200 import workloads as W

from helpers import make_gpu, max_abs

pytestmark = pytest.mark.gpu


def _step_noalloc(grid, surf):
    L = A.load()
    s = surf.c_struct()
    return L.ffs_lbm_step_noalloc(grid.handle, C.byref(s), None)


def _compare_two_calls(wl):
    import torch

    ga, sa = make_gpu(wl)
    gb, sb = make_gpu(wl)
    try:
        for call in range(2):
            v, u = wl.surface_at(call)
            sa.update(v, u)
            sb.update(v, u)
            ga.step(sa)
            rc = _step_noalloc(gb, sb)
            assert rc == A.FFS_OK, A.load().ffs_last_error()
            torch.cuda.synchronize()
            ma, mb = ga.get_moments(), gb.get_moments()
            fa = sa.forces64.cpu().numpy()
            fb = sb.forces64.cpu().numpy()
            assert max_abs(ma, mb) <= 2e-6, f"call {call}: moments differ by {max_abs(ma, mb)}"
            assert np.abs(fa).max() > 0
            assert max_abs(fa, fb) <= 1e-4 * np.abs(fa).max(), f"call {call}: forces differ"
            assert ga.status() == 0
            assert gb.status() == 0
    finally:
        ga.close()
        gb.close()


def test_noalloc_step_matches_step_d3q27(cuda):
    _compare_two_calls(W.swimmer_3d(nx=64, ny=32, nz=32, body_frac=0.3, nlat=12, nlon=16, seed=5))


def test_noalloc_large_surface_separate_force_kernel(cuda):
    """More than 2048 force components (a 770-vertex surface): the sums are
    converted by the separate force kernel, reading them from the fixed array."""
    wl = W.swimmer_3d(nx=64, ny=32, nz=32, body_frac=0.4, nlat=25, nlon=32, seed=6)
    assert wl.rest.shape[0] * 3 > 2048
    _compare_two_calls(wl)


def test_noalloc_step_matches_step_d2q9(cuda):
    _compare_two_calls(W.swimmer_2d(nx=160, ny=64, body_frac=0.5, n_boundary=60, seed=4))


def test_noalloc_rejects_surface_beyond_scratch(cuda):
    """More vertices than the fixed scratch holds: FFS_ERR_CAPACITY, a message
    naming the limit, and no work (the grid's state is unchanged)."""
    from freeflow_b200 import DeviceSurface

    wl = W.swimmer_3d(nx=32, ny=16, nz=16, body_frac=0.3, nlat=8, nlon=12, seed=1)
    g, _ = make_gpu(wl)
    try:
        nv = A.NOALLOC_MAX_VERTICES + 1
        v = np.zeros((nv, 3), np.float32)
        e = np.zeros((1, 3), np.uint32)
        big = DeviceSurface(v, v, e)
        before = g.get_moments()
        rc = _step_noalloc(g, big)
        assert rc == 4  # FFS_ERR_CAPACITY
        assert str(A.NOALLOC_MAX_VERTICES).encode() in A.load().ffs_last_error()
        assert np.array_equal(before, g.get_moments())
    finally:
        g.close()


def test_noalloc_allocates_nothing(cuda):
    """A fresh grid (whose first ffs_lbm_step would allocate its link table and
    force sums) stepped twice through the entry point: the device's free
    memory is the same before and after.  A first grid of the same kind is
    stepped beforehand, so that loading the kernels' code is not counted."""
    import torch

    wl = W.swimmer_3d(nx=48, ny=32, nz=32, body_frac=0.3, nlat=12, nlon=16, seed=8)
    warm, ws = make_gpu(wl)
    try:
        assert _step_noalloc(warm, ws) == A.FFS_OK
        torch.cuda.synchronize()
    finally:
        warm.close()
    g, s = make_gpu(wl)
    try:
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info()
        for _ in range(2):
            assert _step_noalloc(g, s) == A.FFS_OK, A.load().ffs_last_error()
        torch.cuda.synchronize()
        free1, _ = torch.cuda.mem_get_info()
        assert free1 == free0, f"free device memory changed by {free0 - free1} bytes"
        assert g.status() == 0
    finally:
        g.close()


def test_noalloc_full_link_table_sets_status(cuda):
    """A flat plate of 140 x 140 cells between two cell layers gives every cell
    of both layers links: about 39,000 link cells, more than the fixed table's
    32,768 slots.  The step returns normally, latches status bit 2 (link
    table overflow) and faults nothing; the grid steps on afterwards."""
    import torch

    from freeflow_b200 import DeviceSurface, FluidGrid

    n, nz, m = 160, 16, 140
    g = FluidGrid(dim=3, nx=n, ny=n, nz=nz, fluid_viscosity=0.01, fluid_density=1.0, fluid_dx=1.0, dt=1.0,
                  boundary_velocities=[0] * 6, storage="f32", periodic=7)
    try:
        g.set_flags(np.full(n * n * nz, W.FLUID, np.uint8))
        g.set_moments(W.equilibrium_moments(np.ones(n * n * nz), np.zeros((n * n * nz, 3))))
        # plate vertices on a (m+1) x (m+1) lattice at z = 8.5 (between cell centres 8 and 9)
        ii, jj = np.meshgrid(np.arange(m + 1), np.arange(m + 1), indexing="ij")
        v = np.stack([7.0 + ii, 7.0 + jj, np.full(ii.shape, 8.5)], axis=-1).reshape(-1, 3).astype(np.float32)
        v += np.random.default_rng(3).uniform(-1e-3, 1e-3, v.shape).astype(np.float32)
        idx = lambda a, b: a * (m + 1) + b
        tris = []
        for a in range(m):
            for b in range(m):
                tris.append([idx(a, b), idx(a + 1, b), idx(a + 1, b + 1)])
                tris.append([idx(a, b), idx(a + 1, b + 1), idx(a, b + 1)])
        e = np.asarray(tris, np.uint32)
        assert v.shape[0] <= A.NOALLOC_MAX_VERTICES
        s = DeviceSurface(v, np.zeros_like(v), e)
        rc = _step_noalloc(g, s)
        assert rc == A.FFS_OK, A.load().ffs_last_error()
        torch.cuda.synchronize()
        st = g.status(clear=True)
        assert st & 2, f"status {st:#x}: link table overflow not latched"
        g.step()  # the device still works
        torch.cuda.synchronize()
        assert g.status() == 0
    finally:
        g.close()
