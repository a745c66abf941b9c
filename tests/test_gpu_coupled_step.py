"""ffs_lbm_step_coupled: the reference's coupled sequence (surface gather from
the volume mesh, fluid step, force scatter back to the volume mesh) in one
call on one stream.

The volume mesh here is the workload's surface with interior vertices mixed
in, the surface vertices placed at a seeded permutation of the volume
indices.  Each coupled step must equal, bit for bit, a plain ffs_lbm_step on
the gathered surface followed by the scatter: the same moments, the
gathered surface in the caller's arrays, this step's forces at the mapped
volume vertices and zeros elsewhere.  Positions and velocities of the
interior vertices never reach the fluid.
"""
import numpy as np
import pytest

from freeflow_b200 import workloads as W

from helpers import make_gpu

pytestmark = pytest.mark.gpu


def volume_layout(nv, n_interior, seed):
    rng = np.random.default_rng(seed)
    nvol = nv + n_interior
    perm = rng.permutation(nvol)[:nv].astype(np.uint32)   # volume index of surface vertex i
    return nvol, perm


def volume_arrays(v, u, nvol, perm, rng):
    vp = rng.uniform(-1.0, 1.0, (nvol, v.shape[1])).astype(np.float32)   # interior: arbitrary
    vv = rng.uniform(-1.0, 1.0, (nvol, v.shape[1])).astype(np.float32)
    vp[perm] = v
    vv[perm] = u
    return vp, vv


def small_workload(dim):
    if dim == 2:
        return W.swimmer_2d(nx=300, ny=120, body_frac=0.5, n_boundary=120, seed=2)
    return W.swimmer_3d(nx=64, ny=32, nz=32, body_frac=0.4, nlat=16, nlon=24, seed=4)


@pytest.mark.parametrize("dim", [2, 3])
def test_coupled_step_equals_gather_step_scatter(cuda, dim):
    import torch

    from freeflow_b200 import VolumeSurface

    wl = small_workload(dim)
    nv = wl.rest.shape[0]
    nvol, perm = volume_layout(nv, 3 * nv // 2, seed=7)
    rng = np.random.default_rng(11)
    gp, sp = make_gpu(wl)            # plain step on the gathered surface
    gc, _ = make_gpu(wl)             # coupled step
    v0, u0 = wl.surface_at(0)
    vol = VolumeSurface(*volume_arrays(v0, u0, nvol, perm, rng), perm, wl.elements)
    interior = np.setdiff1d(np.arange(nvol), perm)
    for s in range(8):
        v, u = wl.surface_at(s)
        vol.update(*volume_arrays(v, u, nvol, perm, rng))
        sp.update(v, u)
        sp.forces.zero_()
        gp.step(sp)
        gc.step_coupled(vol)
        torch.cuda.synchronize()
        assert np.array_equal(vol.surface_positions.cpu().numpy(), v.astype(np.float32))
        assert np.array_equal(vol.surface_velocities.cpu().numpy(), u.astype(np.float32))
        vf = vol.volume_forces.cpu().numpy()
        fp = sp.forces.cpu().numpy()
        assert np.array_equal(vf[perm], fp)
        assert not vf[interior].any()
    assert np.abs(fp).max() > 0
    assert gp.status() == 0 and gc.status() == 0
    assert np.array_equal(gp.get_moments(), gc.get_moments())
    gp.close()
    gc.close()


def test_coupled_steps_in_a_cuda_graph(cuda):
    """Two coupled steps captured in one graph replay like eager steps (the
    volume arrays are read when the graph runs)."""
    import torch

    from freeflow_b200 import VolumeSurface

    wl = small_workload(3)
    nv = wl.rest.shape[0]
    nvol, perm = volume_layout(nv, nv, seed=3)
    rng = np.random.default_rng(5)
    ge, _ = make_gpu(wl)
    gg, _ = make_gpu(wl)
    v0, u0 = wl.surface_at(0)
    arrays = volume_arrays(v0, u0, nvol, perm, rng)
    ve = VolumeSurface(*arrays, perm, wl.elements)
    va = VolumeSurface(*arrays, perm, wl.elements)
    vb = VolumeSurface(*arrays, perm, wl.elements)
    ge.step_coupled(ve)
    gg.step_coupled(va)
    torch.cuda.synchronize()
    stream = torch.cuda.Stream()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=stream):
        gg.step_coupled(va, stream=stream)
        gg.step_coupled(vb, stream=stream)
    for k in range(1, 7, 2):
        fe = np.zeros((nvol, 3), np.float32)
        for j in (k, k + 1):
            ve.update(*volume_arrays(*wl.surface_at(j), nvol, perm, np.random.default_rng(j)))
            ge.step_coupled(ve)
            fe += ve.volume_forces.cpu().numpy()
        va.update(*volume_arrays(*wl.surface_at(k), nvol, perm, np.random.default_rng(k)))
        vb.update(*volume_arrays(*wl.surface_at(k + 1), nvol, perm, np.random.default_rng(k + 1)))
        graph.replay()
        torch.cuda.synchronize()
        fg = va.volume_forces.cpu().numpy() + vb.volume_forces.cpu().numpy()
        assert np.array_equal(fg, fe)
    assert ge.status() == 0 and gg.status() == 0
    assert np.array_equal(ge.get_moments(), gg.get_moments())
    del graph
    ge.close()
    gg.close()


def test_map_entry_out_of_range_latches_status(cuda):
    import torch

    from freeflow_b200 import VolumeSurface, _capi

    wl = small_workload(2)
    nv = wl.rest.shape[0]
    nvol, perm = volume_layout(nv, 10, seed=1)
    g, _ = make_gpu(wl)
    v0, u0 = wl.surface_at(0)
    vol = VolumeSurface(*volume_arrays(v0, u0, nvol, perm, np.random.default_rng(0)), perm, wl.elements)
    bad = perm.copy()
    bad[5] = nvol + 3
    vol.surface_to_volume.copy_(torch.as_tensor(bad.view(np.int32)))
    g.step_coupled(vol)
    torch.cuda.synchronize()
    assert g.status() & _capi.STATUS_BAD_ELEMENT
    assert np.isfinite(vol.volume_forces.cpu().numpy()).all()
    g.close()


def test_argument_checks(cuda):
    import ctypes

    from freeflow_b200 import FfsError, VolumeSurface, _capi

    wl = small_workload(2)
    nv = wl.rest.shape[0]
    nvol, perm = volume_layout(nv, 4, seed=2)
    g, _ = make_gpu(wl)
    v0, u0 = wl.surface_at(0)
    vol = VolumeSurface(*volume_arrays(v0, u0, nvol, perm, np.random.default_rng(0)), perm, wl.elements)
    L = _capi.load()
    s = vol.c_struct()
    s.dim = 3
    assert L.ffs_lbm_step_coupled(g._h, ctypes.byref(s), None) == 1
    s = vol.c_struct()
    s.volume_forces = None
    assert L.ffs_lbm_step_coupled(g._h, ctypes.byref(s), None) == 1
    s = vol.c_struct()
    s.surface_to_volume = None
    assert L.ffs_lbm_step_coupled(g._h, ctypes.byref(s), None) == 1
    assert L.ffs_lbm_step_coupled(g._h, None, None) == 1
    flat = VolumeSurface(np.zeros((nvol, 3), np.float32), np.zeros((nvol, 3), np.float32), perm[:3],
                         np.arange(3, dtype=np.uint32))
    with pytest.raises(FfsError):
        g.step_coupled(flat)      # a 3D surface on a D2Q9 grid
    assert g.status() == 0
    g.close()
