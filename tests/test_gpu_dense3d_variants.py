"""Every D3Q27 dense-kernel variant against the oracle (the tuner picks one
per grid by speed, so each must pass the parity cases on its own).

Variants: 0 and 1 are the single-plane z-march built for two and three CTAs
per SM; 2 is the two-CTA march with the paired shared-memory layout and
packed c_z = -1 / +1 arithmetic; 3 is variant 2 with each halo plane's
moments staged in shared memory by TMA copies (32-bit indices only; grids
whose rows are not a multiple of 16 bytes run variant 2).
Tolerances are those of test_gpu_parity.py: 2e-6 against the ref32 oracle,
4e-6 next to walls (bounce-back added as a correction), 5e-6 against FP64.
"""
import numpy as np
import pytest

from freeflow_b200 import workloads as W

from helpers import max_abs, run_pair

pytestmark = pytest.mark.gpu

# (variant, index width): the single-plane variants run with 32-bit indices on
# grids of up to 429 M cells and 64-bit ones beyond; FFS_DENSE3D_INDEX64 forces
# the 64-bit path here
VARIANTS = [(0, 32), (1, 32), (2, 32), (3, 32), (0, 64), (1, 64), (2, 64)]


@pytest.fixture(params=VARIANTS, ids=lambda v: f"v{v[0]}-i{v[1]}")
def variant(request, monkeypatch):
    v, width = request.param
    monkeypatch.setenv("FFS_DENSE3D_VARIANT", str(v))
    if width == 64:
        monkeypatch.setenv("FFS_DENSE3D_INDEX64", "1")
    return v


def test_swimmer(cuda, variant):
    wl = W.swimmer_3d(nx=64, ny=32, nz=32, body_frac=0.3, nlat=12, nlon=16, seed=5)
    gm, om, gf, of, st = run_pair(wl, 6)
    assert st == 0
    assert max_abs(gm, om) <= 2e-6
    assert max_abs(gf, of) <= 1e-4 * np.abs(of).max()


def test_taylor_green_periodic_vs_fp64(cuda, variant):
    wl = W.taylor_green_3d(n=32, u0=0.04, viscosity=0.005)
    gm, om, _, _, st = run_pair(wl, 20, precision="phys64")
    assert st == 0
    assert max_abs(gm, om) <= 5e-6


def test_reference_halo(cuda, variant):
    """Non-periodic faces: the halo wraps at the low and clamps at the high face."""
    wl = W.taylor_green_3d(n=20, u0=0.04, viscosity=0.01)
    gm, om, _, _, st = run_pair(wl, 8, periodic=0)
    assert st == 0
    assert max_abs(gm, om) <= 2e-6


def test_walls_inlet_outlet(cuda, variant):
    wl = W.swimmer_3d(nx=40, ny=24, nz=24, nlat=8, nlon=12)
    wl.elements = None
    gm, om, _, _, st = run_pair(wl, 8)
    assert st == 0
    assert max_abs(gm, om) <= 4e-6


def test_open_face_with_wall_across_the_wrap(cuda, variant):
    wl = W.taylor_green_3d(n=20, u0=0.03, viscosity=0.01)
    f = wl.flags.reshape(20, 20, 20)
    f[:, :, 19] = W.WALL
    f[0, :, :] = W.WALL
    wl.flags = f.reshape(-1)
    gm, om, _, _, st = run_pair(wl, 6, periodic=0)
    assert st == 0
    assert max_abs(gm, om) <= 4e-6


@pytest.mark.parametrize("nz", [17, 40])
def test_odd_and_chunked_depths(cuda, variant, nz):
    """Plane counts that leave a single plane in the last pair, and depths
    split into several z chunks."""
    wl = W.swimmer_3d(nx=48, ny=24, nz=nz, body_frac=0.3, nlat=8, nlon=12, seed=9)
    gm, om, _, _, st = run_pair(wl, 4)
    assert st == 0
    assert max_abs(gm, om) <= 4e-6


def test_periodic_width_not_a_tile_multiple(cuda, variant):
    """nx = 48 with x periodic: the last tile's halo wraps onto the first
    columns, and its cells beyond nx only serve as halo."""
    wl = W.taylor_green_3d(n=48, u0=0.04, viscosity=0.01)
    nm = wl.moments.shape[1]
    wl.moments = np.ascontiguousarray(wl.moments.reshape(48, 48, 48, nm)[:12, :20, :].reshape(-1, nm))
    wl.flags = np.ascontiguousarray(wl.flags.reshape(48, 48, 48)[:12, :20, :].reshape(-1))
    wl.ny, wl.nz = 20, 12
    gm, om, _, _, st = run_pair(wl, 6)
    assert st == 0
    assert max_abs(gm, om) <= 2e-6


def test_odd_width(cuda, variant):
    """nx odd: rows whose cells do not pair up on 8-byte boundaries."""
    wl = W.swimmer_3d(nx=41, ny=24, nz=20, body_frac=0.3, nlat=8, nlon=12, seed=11)
    gm, om, _, _, st = run_pair(wl, 4)
    assert st == 0
    assert max_abs(gm, om) <= 4e-6


@pytest.mark.parametrize("storage", ["f32", "f16"])
def test_tuned_variants_round_identically(cuda, monkeypatch, storage):
    """The first step's timing chooses among the variants, so all must give
    the same bits (moments and surface forces, with walls, an inlet, an
    outlet and a moving surface): the choice cannot change a result."""
    import torch

    from helpers import make_gpu

    wl = W.swimmer_3d(nx=64, ny=32, nz=32, body_frac=0.4, nlat=16, nlon=24, seed=4)
    out = []
    for v in ("0", "1", "2", "3"):
        monkeypatch.setenv("FFS_DENSE3D_VARIANT", v)
        g, s = make_gpu(wl, storage)
        for k in range(6):
            s.update(*wl.surface_at(k))
            g.step(s)
        torch.cuda.synchronize()
        assert g.status() == 0
        out.append((g.get_moments(), s.forces64.cpu().numpy()))
        g.close()
    for o in out[1:]:
        assert np.array_equal(out[0][0], o[0])
        assert np.array_equal(out[0][1], o[1])
