"""Link detection under stress: random segments (D2Q9) and triangles (D3Q27)
of every orientation and size, a share of them with vertices on or within
1e-6 of lattice points, so that many links pass through or near cell
centres and element edges.  The CUDA detection (its conservative
prefilters, and the queue that batches the exact tests) must produce the
same link set as the oracle's exhaustive exact test: identical (cell,
direction, depth, element) entries."""
import math

import numpy as np
import pytest

from freeflow_b200 import workloads as W

from helpers import make_gpu, make_oracle

pytestmark = pytest.mark.gpu


def _snap(p, rng, cl):
    """Half of the points move onto a lattice point, some of those off it by 1e-6 cells."""
    out = p.copy()
    on = rng.random(len(p)) < 0.5
    out[on] = np.round(p[on] / cl) * cl
    jit = on & (rng.random(len(p)) < 0.5)
    out[jit] += rng.choice([-1e-6, 1e-6], size=(int(jit.sum()), p.shape[1])) * cl
    return out


def _links(wl):
    g, surf = make_gpu(wl)
    o = make_oracle(wl)
    v, u = wl.surface_at(0)
    surf.update(v, u)
    gcq, gkey = g.debug_links(surf)
    o.step(v, u, wl.elements, None)
    ocq, okey = o.links()
    g.close()
    o.close()
    return gcq, gkey, ocq, okey


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_random_segments_links_identical(cuda, seed):
    rng = np.random.default_rng(seed)
    wl = W.cylinder_channel_2d(nx=96, ny=64, radius=6.0, center=(30.0, 30.0), nseg=32, seed=seed)
    cl = wl.fluid_dx
    n = 400
    c = rng.uniform([4, 4], [wl.nx - 5, wl.ny - 5], size=(n, 2)) * cl
    ang = rng.uniform(0, 2 * math.pi, n)
    special = rng.random(n) < 0.3     # axis-aligned and diagonal segments
    ang[special] = rng.choice([0.0, 0.5 * math.pi, 0.25 * math.pi, 0.75 * math.pi], size=int(special.sum()))
    length = rng.uniform(0.2, 6.0, n) * cl
    d = np.stack([np.cos(ang), np.sin(ang)], 1) * (0.5 * length)[:, None]
    a, b = _snap(c - d, rng, cl), _snap(c + d, rng, cl)
    wl.rest = np.concatenate([a, b]).astype(np.float32)
    wl.elements = np.stack([np.arange(n), np.arange(n) + n], 1).astype(np.uint32)
    gcq, gkey, ocq, okey = _links(wl)
    assert len(ocq) > 1000
    assert np.array_equal(gcq, ocq)
    assert np.array_equal(gkey, okey)


@pytest.mark.parametrize("seed", [0, 1])
def test_random_triangles_links_identical(cuda, seed):
    rng = np.random.default_rng(100 + seed)
    wl = W.swimmer_3d(nx=48, ny=32, nz=32, body_frac=0.3, nlat=8, nlon=12, seed=seed)
    cl = wl.fluid_dx
    n = 300
    c = rng.uniform([4, 4, 4], [wl.nx - 5, wl.ny - 5, wl.nz - 5], size=(n, 3)) * cl
    size = rng.uniform(0.5, 4.0, n) * cl
    off = rng.normal(size=(n, 3, 3))
    axis = rng.random(n) < 0.25      # triangles in a coordinate plane
    k = rng.integers(0, 3, n)
    off[axis, :, k[axis]] = 0.0
    off /= np.linalg.norm(off, axis=2, keepdims=True)
    tri = c[:, None, :] + off * size[:, None, None]
    tri = _snap(tri.reshape(-1, 3), rng, cl).reshape(n, 3, 3)
    wl.rest = tri.reshape(-1, 3).astype(np.float32)
    wl.elements = np.arange(3 * n, dtype=np.uint32).reshape(n, 3)
    wl.kinematics = None
    gcq, gkey, ocq, okey = _links(wl)
    assert len(ocq) > 1000
    assert np.array_equal(gcq, ocq)
    assert np.array_equal(gkey, okey)
