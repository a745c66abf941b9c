"""Dense passes under random node types: grids of odd sizes (no dimension a
multiple of the tile) with walls, static solids and moving-solid cells
scattered through the interior and over the faces, an inlet and an outlet,
with and without periodic axes, and random equilibrium states.  Every
D3Q27 variant and the D2Q9 pass must match the oracle within the wall
tolerance of test_gpu_parity.py (4e-6: near-wall cells add the bounce-back
populations as a correction of the pulled ones)."""
import numpy as np
import pytest

from freeflow_b200 import workloads as W

from helpers import run_pair

pytestmark = pytest.mark.gpu


def _random_state(shape, dim, rng):
    n = int(np.prod(shape))
    rho = 1.0 + rng.uniform(-0.01, 0.01, n)
    u = rng.uniform(-0.05, 0.05, (n, dim))
    return W.equilibrium_moments(rho, u).astype(np.float32)


def _flags(shape, rng, periodic):
    f = np.full(shape, W.FLUID, dtype=np.uint8)
    r = rng.random(shape)
    f[r < 0.06] = W.WALL
    f[(r >= 0.06) & (r < 0.09)] = W.SOLID
    f[(r >= 0.09) & (r < 0.12)] = W.SOLID_DYNAMIC
    if not periodic:
        # faces: x = 0 inlet, x = n-1 outlet, the others half walls
        f[..., 0] = W.INLET_LEFT
        f[..., -1] = W.OUTLET_RIGHT
        for ax in range(f.ndim - 1):
            for side in (0, -1):
                sl = [slice(None)] * f.ndim
                sl[ax] = side
                face = f[tuple(sl)]
                face[rng.random(face.shape) < 0.5] = W.WALL
    return f.reshape(-1)


def _workload_3d(nx, ny, nz, periodic, seed):
    rng = np.random.default_rng(seed)
    wl = W.taylor_green_3d(n=8)
    wl.nx, wl.ny, wl.nz = nx, ny, nz
    wl.flags = _flags((nz, ny, nx), rng, periodic)
    wl.moments = _random_state((nz, ny, nx), 3, rng)
    wl.periodic = 7 if periodic else 0
    wl.boundary_velocities = [0.04, 0, 0, 0, 0, 0]
    wl.fluid_viscosity = 0.02
    return wl


@pytest.fixture(params=[0, 1, 2, 3], ids=lambda v: f"v{v}")
def variant(request, monkeypatch):
    monkeypatch.setenv("FFS_DENSE3D_VARIANT", str(request.param))
    return request.param


@pytest.mark.parametrize("periodic", [False, True], ids=["open", "periodic"])
def test_d3q27_random_node_types(cuda, variant, periodic):
    wl = _workload_3d(37, 21, 19, periodic, seed=3 + periodic)
    gm, om, _, _, st = run_pair(wl, 6)
    assert st == 0
    assert np.abs(gm - om).max() <= 4e-6


def test_d3q27_random_node_types_multiple_of_16_width(cuda, variant):
    """nx a multiple of 4 and 8, so that variant 3 stages by TMA (other widths fall back)."""
    wl = _workload_3d(48, 21, 19, False, seed=7)
    gm, om, _, _, st = run_pair(wl, 6)
    assert st == 0
    assert np.abs(gm - om).max() <= 4e-6


@pytest.mark.parametrize("periodic", [False, True], ids=["open", "periodic"])
def test_d2q9_random_node_types(cuda, periodic):
    rng = np.random.default_rng(11 + periodic)
    wl = W.cylinder_channel_2d(nx=83, ny=45, nseg=16)
    wl.elements = None
    wl.flags = _flags((45, 83), rng, periodic)
    wl.moments = _random_state((45, 83), 2, rng)
    wl.periodic = 3 if periodic else 0
    wl.fluid_viscosity = 0.02
    gm, om, _, _, st = run_pair(wl, 8)
    assert st == 0
    assert np.abs(gm - om).max() <= 4e-6
