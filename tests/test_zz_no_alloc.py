"""ffs_lbm_step_noalloc against ffs_lbm_step, through the C ABI.

The no-allocation variant keeps its link table and force accumulators in a
fixed device array of the library.  Two grids start from the same state; one
is advanced with ffs_lbm_step, the other with ffs_lbm_step_noalloc, on two
calls in a row, and after each call the moments and surface forces must agree
within the parity tolerances of the step itself:
  * moments ......... max |diff| <= 2e-6
  * surface forces .. max |diff| <= 1e-4 x max |F|

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
