"""GPU parity of the CUDA fluid step against the CPU oracle, through the C ABI.

Tolerances (FP32 moments of a stable flow; the oracle and the kernels
evaluate the same expressions in different FP32 operation orders, and the
kernels contract into FMAs):
  * moments, FP32 tile, vs the ref32 oracle ...... max |diff| <= 2e-6 after the steps run
  * moments, FP32 kernels vs the FP64 oracle ....... max |diff| <= 5e-6 (FP32 rounding drift)
  * moments, binary16 D2Q9 tile (reference mode) .. rms <= 1e-4, max <= 1e-3 (a population
    that lands on the other side of a binary16 rounding boundary moves by one half-ulp)
  * link sets ...................................... identical (cell, direction, depth, element)
  * surface forces (FP64 sums) ..................... max |diff| <= 1e-4 x max |F|
"""
import numpy as np
import pytest

from freeflow_b200 import workloads as W

from helpers import make_gpu, make_oracle, max_abs, rms, run_pair

pytestmark = pytest.mark.gpu


def small_cylinder():
    return W.cylinder_channel_2d(nx=64, ny=32, radius=6.0, center=(16.0, 16.0), nseg=48, seed=3)


def small_swimmer_2d():
    return W.swimmer_2d(nx=160, ny=64, body_frac=0.5, n_boundary=60, seed=4)


def small_swimmer_3d():
    return W.swimmer_3d(nx=64, ny=32, nz=32, body_frac=0.3, nlat=12, nlon=16, seed=5)


# ------------------------------------------------------------------- D2Q9
def test_2d_cylinder_fp32_matches_oracle(cuda):
    gm, om, gf, of, st = run_pair(small_cylinder(), 12)
    assert st == 0
    assert max_abs(gm, om) <= 2e-6
    assert max_abs(gf, of) <= 1e-4 * max(np.abs(of).max(), 1e-30)


def test_2d_cylinder_half_tile_matches_reference_mode(cuda):
    gm, om, _, _, st = run_pair(small_cylinder(), 12, ref_half=True)
    assert st == 0
    assert rms(gm, om) <= 1e-4
    assert max_abs(gm, om) <= 1e-3


def test_2d_swimmer_moving_wall_and_forces(cuda):
    gm, om, gf, of, st = run_pair(small_swimmer_2d(), 10)
    assert st == 0
    assert max_abs(gm, om) <= 2e-6
    assert np.abs(of).max() > 0
    assert max_abs(gf, of) <= 1e-4 * np.abs(of).max()


def test_2d_links_identical(cuda):
    wl = small_swimmer_2d()
    g, surf = make_gpu(wl)
    o = make_oracle(wl)
    v, u = wl.surface_at(7)
    surf.update(v, u)
    gcq, gkey = g.debug_links(surf)
    o.step(v, u, wl.elements, None)
    ocq, okey = o.links()
    assert len(ocq) > 0
    assert np.array_equal(gcq, ocq)
    assert np.array_equal(gkey, okey)


def test_2d_periodic_with_cylinder(cuda):
    wl = W.cylinder_channel_2d(nx=48, ny=40, radius=5.0, center=(20.0, 20.0), nseg=40)
    wl.flags[:] = W.FLUID
    gm, om, gf, of, st = run_pair(wl, 20, periodic=3)
    assert st == 0
    assert max_abs(gm, om) <= 2e-6
    assert max_abs(gf, of) <= 1e-4 * np.abs(of).max()


def test_2d_periodic_fp32_vs_fp64(cuda):
    wl = W.cylinder_channel_2d(nx=48, ny=40, radius=5.0, center=(20.0, 20.0), nseg=40)
    wl.flags[:] = W.FLUID
    gm, om, gf, of, st = run_pair(wl, 20, precision="phys64", periodic=3)
    assert st == 0
    assert max_abs(gm, om) <= 5e-6
    assert max_abs(gf, of) <= 1e-4 * np.abs(of).max()


def test_2d_fill_solid_matches_oracle(cuda):
    from freeflow_b200 import DeviceSurface

    wl = small_cylinder()
    g, surf = make_gpu(wl)
    o = make_oracle(wl)
    g.fill_solid(surf)
    o.fill_solid(wl.rest, wl.elements)
    gf, of = g.get_flags(), o.get_flags()
    assert np.array_equal(gf, of)
    assert (gf == W.SOLID_DYNAMIC).sum() > 0


# ------------------------------------------------------------------ D3Q27
def test_3d_swimmer_matches_oracle(cuda):
    gm, om, gf, of, st = run_pair(small_swimmer_3d(), 6)
    assert st == 0
    assert max_abs(gm, om) <= 2e-6
    assert np.abs(of).max() > 0
    assert max_abs(gf, of) <= 1e-4 * np.abs(of).max()


def test_3d_links_identical(cuda):
    wl = small_swimmer_3d()
    g, surf = make_gpu(wl)
    o = make_oracle(wl)
    v, u = wl.surface_at(3)
    surf.update(v, u)
    gcq, gkey = g.debug_links(surf)
    o.step(v, u, wl.elements, None)
    ocq, okey = o.links()
    assert len(ocq) > 0
    assert np.array_equal(gcq, ocq)
    assert np.array_equal(gkey, okey)


def test_3d_taylor_green_periodic_vs_fp64(cuda):
    wl = W.taylor_green_3d(n=32, u0=0.04, viscosity=0.005)
    gm, om, _, _, st = run_pair(wl, 20, precision="phys64")
    assert st == 0
    assert max_abs(gm, om) <= 5e-6


def test_3d_reference_halo_without_periodicity(cuda):
    """Reference semantics without periodicity: the halo wraps at the low face
    and clamps at the high face of each axis (FsiCoupling3D.cu:106-108)."""
    wl = W.taylor_green_3d(n=20, u0=0.04, viscosity=0.01)
    gm, om, _, _, st = run_pair(wl, 8, periodic=0)
    assert st == 0
    assert max_abs(gm, om) <= 2e-6


def test_3d_walls_inlet_outlet_channel(cuda):
    wl = W.swimmer_3d(nx=40, ny=24, nz=24, nlat=8, nlon=12)
    wl.elements = None
    gm, om, _, _, st = run_pair(wl, 8)
    assert st == 0
    # near-wall cells add the bounce-back populations as a correction of the
    # pulled ones (subtract, then add): a few FP32 ulps more than elsewhere
    assert max_abs(gm, om) <= 4e-6


def test_3d_open_face_with_wall_across_the_wrap(cuda):
    """Fluid cells on a non-periodic face whose wrapped neighbour is a wall:
    the reference bounces back (wall test on the wrapped index).  At a low
    face the halo wraps too, at a high face it is clamped to the face, so
    there the pulled value must be replaced (FsiCoupling3D.cu:106-108 vs
    :203-216)."""
    wl = W.taylor_green_3d(n=20, u0=0.03, viscosity=0.01)
    f = wl.flags.reshape(20, 20, 20)
    f[:, :, 19] = W.WALL   # x = nx-1: x = 0 cells see it across the wrap
    f[0, :, :] = W.WALL    # z = 0: z = nz-1 cells see it across the wrap
    wl.flags = f.reshape(-1)
    gm, om, _, _, st = run_pair(wl, 6, periodic=0)
    assert st == 0
    assert max_abs(gm, om) <= 4e-6


# ------------------------------------------------------- storage precision
@pytest.mark.parametrize("storage,l2_tol,max_tol", [("f16", 1e-3, 2e-3), ("bf16", 2e-2, 5e-2)])
def test_reduced_storage_error_vs_fp64(cuda, storage, l2_tol, max_tol):
    """Velocity error of FP16/BF16 scaled-moment storage against FP64 after 50
    Taylor-Green steps: relative L2 (||u - u64|| / ||u64|| over the field) and
    max-norm relative to max |u64|.  FP16 holds the target (1e-3).  BF16 has
    no target: its 8-bit significand rounds each stored velocity by up to
    2^-9 relative, and the bound only checks that it stays in that range
    (about 1e-2 here)."""
    wl = W.taylor_green_3d(n=32, u0=0.04, viscosity=0.005)
    gm, om, _, _, st = run_pair(wl, 50, storage=storage, precision="phys64")
    assert st == 0
    du = gm[:, 1:4] - om[:, 1:4]
    l2 = np.linalg.norm(du) / np.linalg.norm(om[:, 1:4])
    mx = np.abs(du).max() / np.abs(om[:, 1:4]).max()
    assert l2 <= l2_tol
    assert mx <= max_tol


# ----------------------------------------------------------- status / faults
def test_poisoned_state_sets_status_without_fault(cuda):
    """Failure detection without a GPU fault: a block of cells with negative
    density (poisoned on the host) drives the cell at its centre to zero
    density; the kernel latches the status bit and the context stays usable."""
    from freeflow_b200 import FluidGrid

    wl = small_cylinder()
    g = FluidGrid(**wl.grid_kwargs())
    g.set_flags(wl.flags)
    m = wl.moments.copy().reshape(wl.ny, wl.nx, 6)
    m[8:13, 36:41, :] = 0.0
    m[8:13, 36:41, 0] = -1.0
    g.set_moments(m.reshape(-1, 6))
    g.step()
    assert g.status() & 1
    assert g.status() == 0  # cleared by the previous read
    g.initialize()          # the grid keeps working after the report
    g.step()
    assert g.status() == 0


def test_deterministic_repeat(cuda):
    wl = small_swimmer_3d()
    a = run_pair(wl, 4)
    b = run_pair(wl, 4)
    assert np.array_equal(a[0], b[0])
    assert np.array_equal(a[2], b[2])


def test_surface_in_the_solids_full_vertex_arrays(cuda):
    """The step reads the solid's own vertex arrays: boundary elements that
    index a full mesh (interior vertices included) give the same flow and the
    same boundary forces as a gathered surface, and zero force on interior
    vertices, so no gather or scatter pass is needed around the step."""
    from freeflow_b200 import DeviceSurface

    wl = small_swimmer_2d()
    v, u = wl.surface_at(5)
    nb = v.shape[0]
    rng = np.random.default_rng(0)
    interior = rng.uniform(v.min(0), v.max(0), size=(57, 2)).astype(np.float32)
    # full mesh: interior vertices first, then the boundary ones
    V = np.concatenate([interior, v])
    U = np.concatenate([np.zeros_like(interior), u])
    E = wl.elements.astype(np.uint32) + 57
    g1, s1 = make_gpu(wl)
    g2, _ = make_gpu(wl)
    s1.update(v, u)
    s2 = DeviceSurface(V, U, E, with_forces64=True)
    for _ in range(4):
        g1.step(s1)
        g2.step(s2)
    assert np.array_equal(g1.get_moments(), g2.get_moments())
    f1 = s1.forces64.cpu().numpy()
    f2 = s2.forces64.cpu().numpy()
    assert np.array_equal(f2[57:], f1) and np.abs(f1).max() > 0
    assert not f2[:57].any()
    assert nb == f1.shape[0]
