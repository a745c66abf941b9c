"""The D3Q27 solid fill restated in the oracle (ffo_fill_solid3: parity of
the triangles a ray along +x crosses, row by row) pinned on the CPU:

  * against the reference's own inside test, SolidGeometryProxy_Device<3>::
    isInside (segment to the origin, restated as ffo_inside3_ref), cell by
    cell on a seeded ellipsoid in lattice units, where the reference's
    absolute 1e-6 tolerances are far below the geometry;
  * against the analytic answer for a box whose faces and edges lie exactly
    on rows of cell centres (rays through shared edges and vertices);
  * flags other than Fluid/SolidDynamic are kept, and a second fill with the
    body moved returns the cells it left to Fluid.
"""
import numpy as np

from freeflow_b200 import workloads as W
from oracle import oracle as O


def box_mesh(lo, hi):
    """Closed box, two triangles per face, outward winding."""
    x0, y0, z0 = lo
    x1, y1, z1 = hi
    v = np.array([[x0, y0, z0], [x1, y0, z0], [x1, y1, z0], [x0, y1, z0],
                  [x0, y0, z1], [x1, y0, z1], [x1, y1, z1], [x0, y1, z1]], dtype=np.float32)
    quads = [(0, 3, 2, 1), (4, 5, 6, 7), (0, 1, 5, 4), (3, 7, 6, 2), (0, 4, 7, 3), (1, 2, 6, 5)]
    e = []
    for a, b, c, d in quads:
        e += [(a, b, c), (a, c, d)]
    return v, np.asarray(e, dtype=np.uint32)


def seeded_ellipsoid(center, axes, nlat=16, nlon=24, seed=3, jitter=0.05):
    v, e = W.ellipsoid_mesh(*axes, nlat, nlon)
    rng = np.random.default_rng(seed)
    return (v + rng.uniform(-jitter, jitter, v.shape) + np.asarray(center)).astype(np.float32), e


def test_fill_matches_the_reference_inside_test_cell_by_cell():
    nx, ny, nz = 40, 32, 28
    v, e = seeded_ellipsoid((19.7, 15.9, 13.8), (14.3, 7.1, 6.2))
    f = O.fill_solid3(np.full(nx * ny * nz, W.FLUID, np.uint8), nx, ny, nz, 1.0, v, e)
    got = (f == W.SOLID_DYNAMIC).reshape(nz, ny, nx)
    ref = np.zeros_like(got)
    for z in range(nz):
        for y in range(ny):
            for x in range(nx):
                ref[z, y, x] = O.inside3_ref(v, e, (x + 0.5, y + 0.5, z + 0.5))
    assert ref.sum() > 2000
    assert np.array_equal(got, ref)


def test_box_with_faces_on_cell_centre_rows():
    """Faces y = 2.5, 8.5 and z = 3.5, 9.5 hold whole rows of cell centres,
    so rows run through the triangles' shared edges and corners. The edge tie
    rule is half-open, like a rasterizer's: a centre on the faces y = 8.5 or
    z = 3.5 belongs to the box, one on y = 2.5 or z = 9.5 does not, and every
    other cell gets the analytic answer."""
    nx, ny, nz = 16, 12, 13
    v, e = box_mesh((3.2, 2.5, 3.5), (10.7, 8.5, 9.5))
    f = O.fill_solid3(np.full(nx * ny * nz, W.FLUID, np.uint8), nx, ny, nz, 1.0, v, e)
    got = (f == W.SOLID_DYNAMIC).reshape(nz, ny, nx)
    z, y, x = np.meshgrid(np.arange(nz) + 0.5, np.arange(ny) + 0.5, np.arange(nx) + 0.5, indexing="ij")
    inside = (x > 3.2) & (x < 10.7) & (y > 2.5) & (y <= 8.5) & (z >= 3.5) & (z < 9.5)
    assert inside.sum() == 8 * 6 * 6
    assert np.array_equal(got, inside)


def test_other_flags_kept_and_refill_clears():
    nx, ny, nz = 30, 20, 20
    flags = np.full((nz, ny, nx), W.FLUID, np.uint8)
    flags[:, :, 0] = W.INLET_LEFT
    flags[0], flags[-1] = W.WALL, W.WALL
    flags[5, 10, 10] = W.SOLID                       # a static solid cell inside the body
    v, e = seeded_ellipsoid((12.0, 10.0, 10.0), (8.0, 5.0, 5.0), seed=7)
    f1 = O.fill_solid3(flags.reshape(-1), nx, ny, nz, 1.0, v, e).reshape(nz, ny, nx)
    assert f1[5, 10, 10] == W.SOLID
    assert (f1[0] == W.WALL).all() and (f1[1:-1, :, 0] == W.INLET_LEFT).all()
    assert (f1 == W.SOLID_DYNAMIC).sum() > 500
    f2 = O.fill_solid3(f1.reshape(-1), nx, ny, nz, 1.0, v + np.float32([6.0, 0.0, 0.0]), e).reshape(nz, ny, nx)
    moved = O.fill_solid3(flags.reshape(-1), nx, ny, nz, 1.0, v + np.float32([6.0, 0.0, 0.0]), e)
    assert np.array_equal(f2.reshape(-1), moved)
