"""Edge cases of the fluid step on the GPU, each against the oracle where the
result is defined: grids that are not a multiple of the tile, a surface
outside the grid (no links), duplicated elements (equal keys, the smaller
element wins), a bad element index and a full link table (reported through
the status word, never a fault)."""
import numpy as np
import pytest

from freeflow_b200 import _capi as A
from freeflow_b200 import workloads as W

from helpers import make_gpu, make_oracle, max_abs, run_pair

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nx,ny", [(37, 19), (33, 9), (65, 31)])
def test_2d_ragged_grids(cuda, nx, ny):
    wl = W.swimmer_2d(nx=nx * 2, ny=ny * 2, body_frac=0.4, n_boundary=40, seed=nx)
    gm, om, gf, of, st = run_pair(wl, 6)
    assert st == 0
    assert max_abs(gm, om) <= 2e-6
    assert max_abs(gf, of) <= 1e-4 * max(np.abs(of).max(), 1e-30)


@pytest.mark.parametrize("shape", [(37, 19, 11), (33, 9, 5), (31, 40, 3)])
def test_3d_ragged_grids(cuda, shape):
    nx, ny, nz = shape
    wl = W.taylor_green_3d(n=8, u0=0.03, viscosity=0.01)
    # a ragged periodic box: Taylor-Green flow sampled on nx x ny x nz cells
    z, y, x = np.meshgrid(*(2 * np.pi * (np.arange(n) + 0.5) / n for n in (nz, ny, nx)), indexing="ij")
    u = np.stack([0.03 * np.sin(x) * np.cos(y), -0.03 * np.cos(x) * np.sin(y), 0.01 * np.cos(z)], -1).reshape(-1, 3)
    wl.nx, wl.ny, wl.nz = nx, ny, nz
    wl.flags = np.full(nx * ny * nz, W.FLUID, np.uint8)
    wl.moments = W.equilibrium_moments(np.ones(nx * ny * nz), u, dtype=np.float64)
    for periodic in (7, 0):
        gm, om, _, _, st = run_pair(wl, 5, periodic=periodic)
        assert st == 0
        assert max_abs(gm, om) <= 2e-6


def test_surface_outside_the_grid_makes_no_links(cuda):
    wl = W.swimmer_2d(nx=120, ny=48, body_frac=0.5, n_boundary=40, seed=3)
    g, surf = make_gpu(wl)
    v, u = wl.surface_at(0)
    surf.update(v + np.float32(10.0), u)            # 10 m away: far outside the grid
    cq, _ = g.debug_links(surf)
    assert cq.size == 0
    g.step(surf)
    assert g.status() == 0
    assert not surf.forces64.cpu().numpy().any()
    g.close()


def test_duplicated_elements_match_the_oracle(cuda):
    """Every triangle twice: equal depths, the lower element index wins in
    both (the key orders by depth, then element)."""
    wl = W.swimmer_3d(nx=40, ny=24, nz=24, body_frac=0.3, nlat=8, nlon=12, seed=4)
    wl.elements = np.concatenate([wl.elements, wl.elements]).astype(np.uint32)
    gm, om, gf, of, st = run_pair(wl, 3)
    assert st == 0
    assert max_abs(gm, om) <= 4e-6
    assert max_abs(gf, of) <= 1e-4 * np.abs(of).max()


def test_bad_element_index_is_reported_not_faulted(cuda):
    from freeflow_b200 import DeviceSurface

    for wl in (W.swimmer_2d(nx=96, ny=48, body_frac=0.5, n_boundary=40, seed=1),
               W.swimmer_3d(nx=40, ny=24, nz=24, body_frac=0.3, nlat=8, nlon=12, seed=2)):
        g, _ = make_gpu(wl)
        v, u = wl.surface_at(0)
        e = wl.elements.copy()
        e[3, 1] = v.shape[0] + 5                      # past the vertex array
        g.step(DeviceSurface(v, u, e))
        assert g.status() & A.STATUS_BAD_ELEMENT
        g.initialize()
        g.step()
        assert g.status() == 0                        # the grid keeps working
        g.close()


def test_full_link_table_is_reported_not_faulted(cuda):
    # about 6800 cells own links; the smallest table holds 2048
    wl = W.swimmer_3d(nx=256, ny=128, nz=128, nlat=16, nlon=24, seed=6)
    g, surf = make_gpu(wl)
    g.reserve_surface(surf.num_vertices, 8)
    g.step(surf)
    assert g.status() & A.STATUS_LINK_OVERFLOW
    g.close()
