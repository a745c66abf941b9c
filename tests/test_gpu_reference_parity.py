"""The product and the CPU oracle against the reference's own fluid step.

``oracle/_ref/libffs_ref.so`` is the reference's unmodified FsiCoupling2D/3D.cu,
LbmUtilsFunc.cu, LbmConstants.cu and LbmFlowField2D/3D.cpp compiled for this
GPU (``make -C oracle ref``, stand-in headers for glm, spdlog, nlohmann-json
and VTK in oracle/ref_shim); ``oracle/ref.py`` drives it.  Each case runs the
same seeded input through the reference, the product (through the C ABI) and
the oracle's FP32 restatement, and compares moments (max |diff|) and the
accumulated surface forces (max |diff| relative to max |F|).

The reference is FP32 compiled with nvcc's default multiply-add contraction
and sums surface forces with FP32 atomics in arbitrary order, so nothing is
bit-identical; the tolerances are a few times what was measured:
  D3Q27 moments ............ 4e-6   (1.3e-6 .. 1.6e-6)
  D3Q27 forces ............. 2e-4   (2.9e-5 .. 3.4e-5)
  D2Q9, binary16 tile ...... see each case (one binary16 half-ulp of a
                             population moves a moment by up to ~1e-3)

Two behaviours of the reference are reproduced on purpose:
  * its halo index (unsigned arithmetic in min(n-1, max(0, i-1+blockDim*
    blockIdx))) wraps at the low face of every axis and clamps at the high
    face, while the bounce-back test always looks at the wrapped neighbour;
  * its 2D kernel overwrites the bounce-back value with the ordinary pull
    (is_blocked is set only on the moving-wall path), so 2D walls stream
    their stored moments; ``ref_2d_wall_stream`` reproduces that, and
    without it the product bounces back as in 3D (checked below).
"""
import os

import numpy as np
import pytest

from freeflow_b200 import workloads as W

from helpers import make_gpu, make_oracle, max_abs

pytestmark = pytest.mark.gpu


def _ref():
    from oracle import ref as R

    if not R.available():
        pytest.skip("oracle/_ref/libffs_ref.so is not built (the reference's sources were not present)")
    return R


def run_three(wl, steps, half=False, wall_stream=False, periodic=0, oracle=True):
    import torch

    R = _ref()
    g, surf = make_gpu(wl, "f32", half, periodic, wall_stream=wall_stream)
    r = R.RefStep(wl.dim, wl.nx, wl.ny, wl.nz, wl.fluid_viscosity, wl.fluid_density, wl.fluid_dx, wl.dt)
    r.set_flags(wl.flags)
    r.set_moments(wl.moments)
    o = make_oracle(wl, "ref32", half, periodic, wall_stream=wall_stream) if oracle else None
    nf = wl.rest.size if wl.elements is not None else 0
    Fr, Fo = np.zeros(nf), np.zeros(nf)
    for s in range(steps):
        if wl.elements is not None:
            v, u = wl.surface_at(s)
            surf.update(v, u)
            g.step(surf)
            r.step(v, u, wl.elements, Fr)
            if o is not None:
                o.step(v, u, wl.elements, Fo)
        else:
            g.step()
            r.step()
            if o is not None:
                o.step()
    torch.cuda.synchronize()
    out = {"gpu": g.get_moments().astype(np.float64), "ref": r.get_moments(), "status": g.status()}
    if o is not None:
        out["oracle"] = o.get_moments()
        o.close()
    if nf:
        out["F_gpu"] = surf.forces64.cpu().numpy().reshape(-1)
        out["F_ref"] = Fr
        out["F_oracle"] = Fo
    g.close()
    r.close()
    return out


def frel(a, b):
    return max_abs(a, b) / float(np.abs(b).max())


def check3(out, mom=4e-6, force=2e-4):
    assert out["status"] == 0
    assert max_abs(out["gpu"], out["ref"]) <= mom
    if "oracle" in out:
        assert max_abs(out["oracle"], out["ref"]) <= mom
    if "F_ref" in out:
        assert np.abs(out["F_ref"]).max() > 0
        assert frel(out["F_gpu"], out["F_ref"]) <= force
        if "oracle" in out:
            assert frel(out["F_oracle"], out["F_ref"]) <= force


def test_d3q27_swimmer(cuda):
    check3(run_three(W.swimmer_3d(nx=64, ny=32, nz=32, body_frac=0.3, nlat=12, nlon=16, seed=5), 10))


def test_d3q27_walls_inlet_outlet(cuda):
    wl = W.swimmer_3d(nx=40, ny=24, nz=24, nlat=8, nlon=12)
    wl.elements = None
    check3(run_three(wl, 10))


def test_d3q27_open_faces(cuda):
    """Fluid on every face of a non-periodic box: the low faces pull through
    the wrapped halo, the high faces through the clamped one."""
    check3(run_three(W.taylor_green_3d(n=32, u0=0.04, viscosity=0.01), 10))


def test_d3q27_walls_on_both_sides_of_the_wrap(cuda):
    """Walls on open faces, placed so that high-face cells meet both cases of
    the clamped-halo / wrapped-test mismatch: a wall only at the wrapped
    neighbour (its pulled value must go) and a wall only in the clamped halo
    (its own population must come in)."""
    n = 16
    wl = W.taylor_green_3d(n=n, u0=0.03, viscosity=0.01)
    f = wl.flags.reshape(n, n, n)     # [z][y][x]
    f[:, n - 1, 5] = W.WALL           # in the high-y face: the clamped halo of (6, n-1) along (+x, -y)
    f[:, 0, 9] = W.WALL               # in the low-y face: the wrapped neighbour of (10, n-1) along (+x, -y)
    f[n - 1, 3:6, 3:6] = W.WALL       # a patch in the high-z face
    f[0, 10:13, 10:13] = W.WALL       # and in the low-z face
    f[4:7, 4:7, n - 1] = W.SOLID      # the high-x face
    wl.flags = f.reshape(-1)
    check3(run_three(wl, 8))


def test_d3q27_random_node_types(cuda):
    """Walls, static solids and moving-solid cells scattered through an odd-
    sized box and over its faces, an inlet and an outlet, random equilibrium
    states: the product and the oracle against the reference's own step."""
    from test_gpu_random_flags import _workload_3d

    check3(run_three(_workload_3d(37, 21, 19, False, seed=5), 8))


def test_d3q27_full_size_swimmer(cuda):
    """Config D at its full size (384 x 192 x 192, 4034-vertex undulating
    ellipsoid), 20 steps, product against the reference (the oracle is
    compared at this size in test_gpu_full_configs.py)."""
    check3(run_three(W.swimmer_3d(), 20, oracle=False))


def _tie_distance(wl, cell, d):
    """Distance (lattice units) from the link segment of (cell, direction d)
    to the nearest vertex of the surface polygon."""
    # D2Q9 velocities in the reference's numbering (LbmConstants.hpp:48-51)
    ex = (0, 1, 0, -1, 0, 1, -1, -1, 1)
    ey = (0, 0, 1, 0, -1, 1, 1, -1, -1)
    x, y = cell % wl.nx, cell // wl.nx
    cx, cy = ex[d], ey[d]
    p1 = np.array([x, y], np.float64)
    p2 = np.array([x - cx, y - cy], np.float64)
    V = wl.rest.astype(np.float64) / wl.fluid_dx
    t = np.clip(((V - p1) @ (p2 - p1)) / ((p2 - p1) @ (p2 - p1)), 0.0, 1.0)
    return float(np.min(np.linalg.norm(p1 + t[:, None] * (p2 - p1) - V, axis=1)))


def test_d2q9_cylinder_link_ties(cuda):
    """Config A's cylinder (a 128-gon centred on a lattice point): the link
    sets of the product and the reference agree except where a link segment
    passes exactly through a vertex of the polygon.  Such ties are decided by
    the last bit of the intersection arithmetic, which the reference forms
    with fused multiply-adds (nvcc's default contraction) and the product
    with singly rounded operations, bit for bit as the oracle does.  Every
    differing link must be such a tie; shared links name the same element."""
    R = _ref()
    wl = W.cylinder_channel_2d()
    g, surf = make_gpu(wl, "f32", True, 0, wall_stream=True)
    r = R.RefStep(2, wl.nx, wl.ny, 1, wl.fluid_viscosity, wl.fluid_density, wl.fluid_dx, wl.dt)
    r.set_flags(wl.flags)
    r.set_moments(wl.moments)
    v, u = wl.surface_at(0)
    surf.update(v, u)
    g.step(surf)
    r.step(v, u, wl.elements, None)
    cq, key = g.debug_links(surf)
    mine = {int(c): int(k) & 0xFFFFFFFF for c, k in zip(cq, key)}
    H = r.hits().reshape(-1)
    theirs = {int(i): int(H[i]) & 0xFFFF for i in np.nonzero(H != 0xFFFFFFFF)[0]}
    g.close()
    r.close()
    diff = set(mine) ^ set(theirs)
    assert len(diff) <= 8, sorted(diff)
    for c in diff:
        assert _tie_distance(wl, c // 9, c % 9) < 1e-3, (c // 9, c % 9)
    for c in set(mine) & set(theirs):
        assert mine[c] == theirs[c]


def test_d2q9_cylinder_reference_walls(cuda):
    """A cylinder channel like config A, with the cylinder's centre moved off
    the lattice by a hundredth of a cell so that no link segment meets a
    polygon vertex exactly, 200 steps with the reference's 2D kernel
    semantics (binary16 population tile, walls streaming their moments):
    moments max |diff| <= 4e-3 (one binary16 half-ulp of a population moves
    a moment by up to ~1e-3) and accumulated forces <= 1e-2 x max |F|."""
    wl = W.cylinder_channel_2d(center=(64.013, 63.991))
    out = run_three(wl, 200, half=True, wall_stream=True)
    assert out["status"] == 0
    assert max_abs(out["gpu"], out["ref"]) <= 4e-3
    assert max_abs(out["oracle"], out["ref"]) <= 4e-3
    assert frel(out["F_gpu"], out["F_ref"]) <= 1e-2
    assert frel(out["F_oracle"], out["F_ref"]) <= 1e-2


def test_d2q9_moving_swimmer(cuda):
    wl = W.swimmer_2d(nx=300, ny=120, body_frac=0.4, n_boundary=60, seed=3)
    out = run_three(wl, 100, half=True, wall_stream=True)
    assert out["status"] == 0
    assert max_abs(out["gpu"], out["ref"]) <= 4e-3
    assert max_abs(out["oracle"], out["ref"]) <= 4e-3
    assert frel(out["F_gpu"], out["F_ref"]) <= 2e-3
    assert frel(out["F_oracle"], out["F_ref"]) <= 2e-3


def _channel2(nx=64, ny=32):
    f = np.full((ny, nx), W.FLUID, np.uint8)
    f[0, :] = W.WALL
    rng = np.random.default_rng(0)
    u = np.zeros((ny, nx, 2))
    u[..., 0] = 0.05 + rng.uniform(-1e-3, 1e-3, (ny, nx))
    u[..., 1] = rng.uniform(-1e-3, 1e-3, (ny, nx))
    m = W.equilibrium_moments(np.ones(ny * nx), u.reshape(-1, 2))
    return W.Workload("wall channel", 2, nx, ny, 1, 0.016, 1.0, 1.0, 1.0, [0] * 4, f.reshape(-1), m, 0)


def test_d2q9_reference_walls_stream(cuda):
    """The reference's 2D walls do not bounce back: next to a wall row, one
    step of a uniform stream equals the same step without the wall (the
    reference against itself), and the product matches it with
    ref_2d_wall_stream; without it the product bounces back, as in 3D, and
    slows the wall row's flow."""
    wl = _channel2()
    plain = _channel2()
    plain.flags = np.full_like(plain.flags, W.FLUID)
    walls_ref = run_three(wl, 1, oracle=False)["ref"]
    nowall_ref = run_three(plain, 1, oracle=False)["ref"]
    nx = wl.nx
    assert np.array_equal(walls_ref[nx:2 * nx], nowall_ref[nx:2 * nx])
    # the reference rounds its population tile to binary16: so does the
    # product here (one half-ulp flip moves a moment by up to ~1e-3)
    stream = run_three(wl, 1, half=True, wall_stream=True)
    assert max_abs(stream["gpu"], stream["ref"]) <= 2e-3
    assert max_abs(stream["oracle"], stream["ref"]) <= 2e-3
    assert float(np.sqrt(np.mean((stream["gpu"] - stream["ref"]) ** 2))) <= 1e-4
    bounce = run_three(wl, 1)
    ux_row1 = bounce["gpu"][nx:2 * nx, 1]
    assert np.all(ux_row1 < 0.04)                     # the wall takes momentum out
    assert max_abs(bounce["gpu"], bounce["oracle"]) <= 2e-6
