"""fill_solid (fillSolidFlags2D) on the GPU against the oracle's per-cell
crossing test: the masks must be identical, for a convex body, a concave
swimmer outline, and a comb with more crossings per row than the kernel keeps
in shared memory (its per-cell fallback).  On D3Q27 grids, against the
oracle's restatement of the row-parity fill (oracle.fill_solid3, itself pinned
to the reference's 3D inside test in test_fill_solid3_oracle.py)."""
import numpy as np
import pytest

from freeflow_b200 import workloads as W

from helpers import make_gpu, make_oracle

pytestmark = pytest.mark.gpu


def _check(wl, vertices, elements):
    from freeflow_b200 import DeviceSurface, FluidGrid

    g = FluidGrid(**wl.grid_kwargs())
    g.set_flags(wl.flags)
    surf = DeviceSurface(vertices, np.zeros_like(vertices), elements)
    g.fill_solid(surf)
    o = make_oracle(wl)
    o.fill_solid(vertices, elements)
    gf, of = g.get_flags(), o.get_flags()
    assert np.array_equal(gf, of)
    n = int((gf == W.SOLID_DYNAMIC).sum())
    g.close()
    o.close()
    return n


def test_fill_solid_swimmer_outline(cuda):
    wl = W.swimmer_2d(nx=300, ny=120, body_frac=0.5, n_boundary=120, seed=2)
    v, _ = wl.surface_at(17)
    assert _check(wl, v, wl.elements) > 100


def test_fill_solid_comb_beyond_shared_memory(cuda):
    """A comb of 200 teeth: rows through the teeth cross 400 edges, more than
    the 256 crossings a row keeps in shared memory."""
    nx, ny = 640, 40
    wl = W.cylinder_channel_2d(nx=nx, ny=ny, radius=4.0, center=(20.0, 20.0), nseg=16)
    wl.flags[:] = W.FLUID
    dx = wl.fluid_dx
    teeth = 200
    pts = [(0.5, 2.5)]
    for t in range(teeth):
        x0 = 1.0 + 3.0 * t
        pts += [(x0, 30.5), (x0 + 1.5, 30.5), (x0 + 1.5, 10.5), (x0 + 3.0, 10.5)]
    pts += [(1.0 + 3.0 * teeth, 2.5)]
    v = (np.array(pts) * dx).astype(np.float32)
    e = np.stack([np.arange(len(v)), (np.arange(len(v)) + 1) % len(v)], 1).astype(np.uint32)
    assert _check(wl, v, e) > 1000


# ------------------------------------------------------------------ D3Q27
def _check3(wl, flags, vertices, elements, fills=1, shift=None):
    """fill_solid on a D3Q27 grid against the oracle's restatement
    (oracle.fill_solid3), `fills` times with the body moved by `shift`
    between fills; the flags must be identical after every fill."""
    from freeflow_b200 import DeviceSurface, FluidGrid
    from oracle import oracle as O

    g = FluidGrid(**wl.grid_kwargs())
    g.set_flags(flags)
    g.initialize()
    want = np.asarray(flags, np.uint8).reshape(-1)
    v = np.asarray(vertices, np.float32)
    n = 0
    for _ in range(fills):
        g.fill_solid(DeviceSurface(v, np.zeros_like(v), elements))
        want = O.fill_solid3(want, wl.nx, wl.ny, wl.nz, wl.fluid_dx, v, elements)
        got = g.get_flags()
        assert np.array_equal(got, want)
        n = int((got == W.SOLID_DYNAMIC).sum())
        if shift is not None:
            v = v + np.float32(shift)
    g.step()
    assert g.status() == 0
    g.close()
    return n


def test_fill_solid3_undulating_ellipsoid(cuda):
    wl = W.swimmer_3d(nx=96, ny=48, nz=48, body_frac=0.4, nlat=24, nlon=32, seed=4)
    v, _ = wl.surface_at(3)
    assert _check3(wl, wl.flags, v, wl.elements) > 300          # about 4/3 pi 19.2 x 2.4 x 2.4 cells


def test_fill_solid3_box_on_cell_centre_rows_ragged_width(cuda):
    """Box faces on rows of cell centres (rays through shared edges and
    corners); 70 cells per row, so the row masks end inside a word."""
    import sys, os
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from test_fill_solid3_oracle import box_mesh

    wl = W.taylor_green_3d(n=8, u0=0.0, viscosity=0.01)
    wl.nx, wl.ny, wl.nz, wl.fluid_dx = 70, 12, 13, 1.0
    flags = np.full(70 * 12 * 13, W.FLUID, np.uint8)
    wl.flags = flags
    v, e = box_mesh((3.2, 2.5, 3.5), (66.7, 8.5, 9.5))
    assert _check3(wl, flags, v, e) == 64 * 6 * 6


def test_fill_solid3_refill_after_moving(cuda):
    wl = W.swimmer_3d(nx=80, ny=40, nz=40, body_frac=0.4, nlat=16, nlon=24, seed=8)
    v, _ = wl.surface_at(0)
    assert _check3(wl, wl.flags, v, wl.elements, fills=3, shift=(0.05, 0.02, -0.01)) > 150
