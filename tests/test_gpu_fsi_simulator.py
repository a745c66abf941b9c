"""The fsi_simulator mirror on the GPU: a JSON configuration and a Medit mesh
in the reference's formats drive Simulator2D / Simulator3D, and the steps
match the oracle fed the same surfaces (tolerances of test_gpu_parity.py:
moments 2e-6, forces 1e-4 x max |F|).  The accessors return the volume mesh
as the reference's do: the surface is getBoundaryVertices / getBoundaryElements
with the map getBoundaryPointIdx, and getForce holds the last step's force on
the surface's volume vertices."""
import json
import math

import numpy as np
import pytest

from freeflow_b200 import fsi_simulator as F
from freeflow_b200 import meshio

from helpers import max_abs

pytestmark = pytest.mark.gpu


def _disk_mesh(path, r, n):
    """A triangle fan: centre vertex plus n rim vertices."""
    th = 2 * math.pi * np.arange(n) / n
    v = np.concatenate([[[0.0, 0.0]], np.stack([r * np.cos(th), r * np.sin(th)], 1)])
    t = np.array([[0, 1 + i, 1 + (i + 1) % n] for i in range(n)])
    meshio.write_medit(path, v, triangles=t)


def _config_2d(tmp_path, nx=96, ny=48):
    bcs = [{"pos": [x, 0], "type": "Wall"} for x in range(nx)] + \
          [{"pos": [x, ny - 1], "type": "Wall"} for x in range(nx)] + \
          [{"pos": [0, y], "type": "InletLeft"} for y in range(1, ny - 1)] + \
          [{"pos": [nx - 1, y], "type": "OutletRight"} for y in range(1, ny - 1)]
    mesh = str(tmp_path / "disk.mesh")
    _disk_mesh(mesh, 1.0, 40)
    cfg = {"fluid_nx": nx, "fluid_ny": ny, "fluid_viscosity": 0.02, "fluid_density": 10.0, "fluid_dx": 0.01,
           "dt": 0.004, "boundary_velocities": [0.04, 0, 0, 0], "boundaries": bcs,
           "solids": [{"mesh_path": mesh, "translate": [0.3, 0.24], "scale": [0.06, 0.06], "rotate": 15}]}
    path = tmp_path / "cfg.json"
    path.write_text(json.dumps(cfg))
    c = F.Config2D()
    assert c.load(str(path))
    return c.get_params()


def _oracle_for(sim, p, dim):
    from oracle.oracle import Oracle

    bc = list(p.boundary_velocities) or [0.0] * (2 * dim)
    o = Oracle(dim, p.fluid_nx, p.fluid_ny, getattr(p, "fluid_nz", 1), viscosity=p.fluid_viscosity,
               density=p.fluid_density, dx=p.fluid_dx, dt=p.dt, boundary_velocities=bc, periodic=0,
               precision="ref32")
    o.set_flags(F.flags_from_params(p))
    o.set_moments(sim.get_fluid_moments().reshape(-1, 6 if dim == 2 else 10).astype(np.float64))
    return o


def test_simulator2d_config_mesh_and_kinematic_body_match_oracle(cuda, tmp_path):
    p = _config_2d(tmp_path)
    sim = F.Simulator2D(p)
    sim.initialize()
    sim.apply_kinematic_control(0, [[0.5, 0.3], [0.6, 0.2]], 0.02)
    o = _oracle_for(sim, p, 2)
    elements = sim.getBoundaryElements().reshape(-1, 2)
    assert elements.shape == (40, 2)
    # the volume mesh is the disk fan: its centre vertex is interior
    smap = sim.getBoundaryPointIdx()
    assert sim.getVertices().shape == (41, 2) and sim.getTriangles().size == 40 * 3
    assert smap.size == 40 and 0 not in smap
    assert np.array_equal(sim.getBoundaryVertices(), sim.getVertices()[smap])
    for _ in range(6):
        V, U = sim.getBoundaryVertices(), sim.getVelocity()[smap]
        Fo = np.zeros(V.size)
        o.step(V, U, elements, Fo)
        sim.step()
    assert max_abs(sim.get_fluid_moments().reshape(-1, 6), o.get_moments()) <= 2e-6
    F_all = sim.getForce()
    Fg = F_all[smap].reshape(-1).astype(np.float64)
    assert np.abs(Fo).max() > 0
    assert max_abs(Fg, Fo) <= 1e-4 * np.abs(Fo).max() + 1e-6 * np.abs(Fg).max()
    assert not F_all[0].any()       # no fluid force on the interior vertex
    # the body moved towards its first target at 0.02 per unit time
    assert np.allclose(sim.getVelocity()[0], 0.02 * np.array([0.2, 0.06]) / np.hypot(0.2, 0.06), rtol=1e-5)
    assert sim.status() == 0
    o.close()
    sim.close()


def test_simulator2d_accessors_fill_solid_and_profiler(cuda, tmp_path):
    p = _config_2d(tmp_path)
    sim = F.Simulator2D(p)
    sim.initialize()
    cells = sim.fill_solid()
    assert len(cells) > 0 and all(0 < x < p.fluid_nx and 0 < y < p.fluid_ny for x, y in cells)
    sim.begin_profiler("steps")
    for _ in range(3):
        sim.step()
    rep = sim.end_profiler()
    assert rep["dense"][1] == 3 and rep["detect_links"][1] == 3
    m_cur, m_a = sim.get_fluid_moments(), sim.get_fluid_moments(buffer="A")
    assert m_cur.shape == (p.fluid_ny, p.fluid_nx, 6)
    assert not np.array_equal(m_cur, m_a)   # after an odd number of steps buffer A is the older one
    sim.save_frame_data(3)
    sim.reset()
    assert np.allclose(sim.get_fluid_moments()[..., 0], 1.0)
    sim.close()


def test_simulator3d_config_and_tet_mesh_match_oracle(cuda, tmp_path):
    nx, ny, nz = 40, 24, 24
    v = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], float)
    tets = np.array([[0, 1, 2, 6], [0, 2, 3, 6], [0, 3, 7, 6], [0, 7, 4, 6], [0, 4, 5, 6], [0, 5, 1, 6]])
    mesh = str(tmp_path / "cube.mesh")
    meshio.write_medit(mesh, v, tetrahedra=tets)
    bcs = [{"pos": [0, y, z], "type": "InletLeft"} for y in range(ny) for z in range(nz)] + \
          [{"pos": [nx - 1, y, z], "type": "OutletRight"} for y in range(ny) for z in range(nz)]
    cfg = {"fluid_nx": nx, "fluid_ny": ny, "fluid_nz": nz, "fluid_viscosity": 0.02, "fluid_density": 10.0,
           "fluid_dx": 0.01, "dt": 0.004, "boundary_velocities": [0.03, 0, 0, 0, 0, 0], "boundaries": bcs,
           "solids": [{"mesh_path": mesh, "translate": [0.12, 0.1, 0.1], "scale": [0.05, 0.04, 0.04],
                       "rotate": [10, 20, 30]}]}
    path = tmp_path / "c3.json"
    path.write_text(json.dumps(cfg))
    c = F.Config3D()
    assert c.load(str(path))
    p = c.get_params()
    sim = F.Simulator3D(p)
    sim.initialize()
    sim.apply_kinematic_control(0, [[0.2, 0.12, 0.1], [0.1, 0.1, 0.1]], 0.01)
    o = _oracle_for(sim, p, 3)
    elements = sim.getBoundaryElements().reshape(-1, 3)
    assert elements.shape == (12, 3)
    smap = sim.getBoundaryPointIdx()
    assert sim.getVertices().shape == (8, 3) and sim.getTetrahedra().size == 6 * 4
    for _ in range(4):
        V, U = sim.getBoundaryVertices(), sim.getVelocity()[smap]
        Fo = np.zeros(V.size)
        o.step(V, U, elements, Fo)
        sim.step()
    assert max_abs(sim.get_fluid_moments().reshape(-1, 10), o.get_moments()) <= 4e-6
    Fg = sim.getForce()[smap].reshape(-1).astype(np.float64)
    assert np.abs(Fo).max() > 0
    assert max_abs(Fg, Fo) <= 1e-4 * np.abs(Fo).max() + 1e-6 * np.abs(Fg).max()
    o.close()
    sim.close()
