"""fill_solid (fillSolidFlags2D) on the GPU against the oracle's per-cell
crossing test: the masks must be identical, for a convex body, a concave
swimmer outline, and a comb with more crossings per row than the kernel keeps
in shared memory (its per-cell fallback)."""
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
