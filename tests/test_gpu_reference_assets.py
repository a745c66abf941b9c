"""FreeFlow's own shipped configurations and meshes (tests/golden/reference_assets/)
driven through Simulator2D on the GPU and checked against the oracle fed the
same surfaces (tolerances of test_gpu_parity.py: moments 2e-6, forces
1e-4 x max |F|).

* vortexstreet2d.json: 801 x 201 channel, inlet on the left, outlet on the
  right, walls top and bottom, the static sphere2d.mesh disk;
* fish2d_lbs_control.json: 1200 x 400 tank with outlets on all four sides and
  the fish2d.mesh body of a "vbd" solid; the solid solver is outside this
  package, so the test moves the body itself through set_surface, as the
  owner of a deformable model does.
"""
import math

import numpy as np
import pytest

from freeflow_b200 import fsi_simulator as F

from helpers import max_abs
from test_reference_assets import asset_file

pytestmark = pytest.mark.gpu


def _load(tmp_path, config, mesh):
    c = F.Config2D()
    assert c.load(asset_file(tmp_path, config))
    p = c.get_params()
    p.solids[0].mesh_path = asset_file(tmp_path, mesh)
    return p


def _oracle_for(sim, p):
    from oracle.oracle import Oracle

    o = Oracle(2, p.fluid_nx, p.fluid_ny, 1, viscosity=p.fluid_viscosity, density=p.fluid_density,
               dx=p.fluid_dx, dt=p.dt, boundary_velocities=list(p.boundary_velocities), periodic=0,
               precision="ref32")
    o.set_flags(F.flags_from_params(p))
    o.set_moments(sim.get_fluid_moments().reshape(-1, 6).astype(np.float64))
    return o


def _run(sim, o, steps, move=None):
    smap = sim.getBoundaryPointIdx()
    elements = sim.getBoundaryElements().reshape(-1, 2)
    for s in range(steps):
        if move is not None:
            move(s)
        V, U = sim.getBoundaryVertices(), sim.getVelocity()[smap]
        Fo = np.zeros(V.size)
        o.step(V, U, elements, Fo)
        sim.step()
    Fg = sim.getForce()[smap].reshape(-1).astype(np.float64)
    return Fg, Fo


def test_vortex_street_config_matches_oracle(cuda, tmp_path):
    p = _load(tmp_path, "vortexstreet2d.json", "sphere2d.mesh")
    sim = F.Simulator2D(p)
    sim.initialize()
    # a moving cylinder, so that the moving-wall links carry momentum
    sim.apply_kinematic_control(0, [[0.6, 0.5], [0.4, 0.5]], 0.05)
    o = _oracle_for(sim, p)
    Fg, Fo = _run(sim, o, 6)
    assert max_abs(sim.get_fluid_moments().reshape(-1, 6), o.get_moments()) <= 2e-6
    assert np.abs(Fo).max() > 0
    assert max_abs(Fg, Fo) <= 1e-4 * np.abs(Fo).max() + 1e-6 * np.abs(Fg).max()
    assert sim.status() == 0
    o.close()
    sim.close()


def test_fish_config_with_a_body_moved_by_its_owner_matches_oracle(cuda, tmp_path):
    p = _load(tmp_path, "fish2d_lbs_control.json", "fish2d.mesh")
    sim = F.Simulator2D(p)
    with pytest.warns(UserWarning, match="deformable"):
        sim.initialize()
    rest = sim.getVertices().copy()
    c = rest.mean(axis=0)

    def move(s):
        # a travelling body wave along x, as a solid model would report it
        t = (s + 1) * p.dt
        k, w, a = 2 * math.pi / 0.2, 2 * math.pi * 2.0, 0.01
        x = rest[:, 0] - c[0]
        y = rest[:, 1] + a * np.sin(k * x - w * t)
        vy = -a * w * np.cos(k * x - w * t)
        sim.set_surface(np.stack([rest[:, 0], y], 1), np.stack([np.zeros_like(vy), vy], 1))

    o = _oracle_for(sim, p)
    Fg, Fo = _run(sim, o, 5, move)
    assert max_abs(sim.get_fluid_moments().reshape(-1, 6), o.get_moments()) <= 2e-6
    assert np.abs(Fo).max() > 0
    assert max_abs(Fg, Fo) <= 1e-4 * np.abs(Fo).max() + 1e-6 * np.abs(Fg).max()
    assert sim.status() == 0
    o.close()
    sim.close()
