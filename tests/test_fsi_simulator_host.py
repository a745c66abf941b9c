"""The fsi_simulator mirror on the host (no GPU): JSON configuration with the
reference's fields and defaults, node flags from the boundary list, Medit mesh
reading, surface extraction and solid placement."""
import json
import math

import numpy as np
import pytest

from freeflow_b200 import fsi_simulator as F
from freeflow_b200 import meshio


def _write(tmp_path, name, obj):
    p = tmp_path / name
    p.write_text(json.dumps(obj))
    return str(p)


def test_config2d_fields_defaults_and_boundaries(tmp_path):
    path = _write(tmp_path, "c.json", {
        "fluid_nx": 16, "fluid_ny": 8, "fluid_viscosity": 0.02, "dt": 0.0025, "fluid_dx": 0.005,
        "boundary_velocities": [0.05, 0, 0, 0],
        "boundaries": [{"pos": [0, 3], "type": "InletLeft"}, {"pos": [15, 3], "type": "OutletRight"},
                       {"pos": [4, 0], "type": "Wall"}, {"pos": [4, 0], "type": "Bogus"}],
        "solids": [{"mesh_path": "fish.mesh", "translate": [1, 2], "rotate": 30, "density": 50}],
        "global_fem_options": {"iterations": 4},
    })
    c = F.Config2D()
    with pytest.warns(UserWarning, match="unrecognized"):
        assert c.load(path)
    p = c.get_params()
    assert (p.fluid_nx, p.fluid_ny, p.fluid_viscosity, p.dt, p.fluid_dx) == (16, 8, 0.02, 0.0025, 0.005)
    assert p.fluid_density == 1000.0 and p.solid_solver_type == "static" and p.output_frequency == 100
    assert p.boundary_velocities == [float(np.float32(0.05)), 0.0, 0.0, 0.0]  # std::vector<float>
    assert [b.flag for b in p.boundaries] == [13, 20, 5, 0]
    s = p.solids[0]
    assert s.mesh_path == "fish.mesh" and s.translate == [1.0, 2.0] and s.rotate == 30.0 and s.density == 50.0
    assert s.scale == [1.0, 1.0] and s.lbs_control_config.cnum == 2
    assert p.global_fem_options.iterations == 4 and p.global_fem_options.omega == 0.8
    # getCf in float: rho dx^2 dx / dt^2
    assert p.get_cf() == float(np.float32(float(np.float32(1000.0 * 0.005 * 0.005)) * 0.005 / 0.0025 ** 2))


def test_config_defaults_when_fields_are_absent(tmp_path):
    c2, c3 = F.Config2D(), F.Config3D()
    assert c2.load(_write(tmp_path, "a.json", {}))
    assert c3.load(_write(tmp_path, "b.json", {"fluid_nz": 12}))
    p2, p3 = c2.get_params(), c3.get_params()
    assert (p2.fluid_nx, p2.fluid_ny, p2.boundary_velocities) == (400, 400, [0.0] * 4)
    assert (p3.fluid_nx, p3.fluid_ny, p3.fluid_nz, p3.boundary_velocities) == (128, 128, 12, [])


def test_config_load_failures(tmp_path, capsys):
    c = F.Config2D()
    assert not c.load(str(tmp_path / "missing.json"))
    bad = tmp_path / "bad.json"
    bad.write_text("{ not json")
    assert not c.load(str(bad))
    assert not c.load(_write(tmp_path, "t.json", {"boundaries": [{"type": "Wall"}]}))  # no "pos"
    assert "FATAL" in capsys.readouterr().err


def test_flags_from_boundaries_later_entry_wins_and_outside_is_ignored():
    p = F.SimulationParameters2D(fluid_nx=5, fluid_ny=4)
    p.boundaries = [F.BoundaryCondition([0, 0], 5), F.BoundaryCondition([0, 0], 13),
                    F.BoundaryCondition([4, 3], 20), F.BoundaryCondition([5, 0], 5)]
    with pytest.warns(UserWarning, match="outside"):
        f = F.flags_from_params(p)
    assert f.shape == (20,) and f[0] == 13 and f[19] == 20 and (f[1:19] == F.FLUID).all()
    p3 = F.SimulationParameters3D(fluid_nx=3, fluid_ny=2, fluid_nz=2)
    p3.boundaries = [F.BoundaryCondition([2, 1, 1], 24)]
    f3 = F.flags_from_params(p3)
    assert f3[(1 * 2 + 1) * 3 + 2] == 24 and (f3 == F.FLUID).sum() == 11


def test_boundary_boxes_equal_their_cells(tmp_path):
    """A "boundaries" entry with "to" covers its inclusive box: the channel walls,
    inlet and outlet of a 40x12 grid as four entries give the same flags as the
    reference's one entry per cell (and later entries still win)."""
    nx, ny = 40, 12
    cells = ([{"type": "Wall", "pos": [x, y]} for y in (0, ny - 1) for x in range(nx)]
             + [{"type": "InletLeft", "pos": [0, y]} for y in range(1, ny - 1)]
             + [{"type": "OutletRight", "pos": [nx - 1, y]} for y in range(1, ny - 1)])
    boxes = [{"type": "Wall", "pos": [0, 0], "to": [nx - 1, 0]}, {"type": "Wall", "pos": [nx - 1, ny - 1], "to": [0, ny - 1]},
             {"type": "InletLeft", "pos": [0, 1], "to": [0, ny - 2]}, {"type": "OutletRight", "pos": [nx - 1, 1], "to": [nx - 1, ny - 2]}]
    flags = []
    for entries in (cells, boxes):
        c = F.Config2D()
        assert c.load(_write(tmp_path, "b.json", {"fluid_nx": nx, "fluid_ny": ny, "boundaries": entries}))
        flags.append(F.flags_from_params(c.get_params()))
    assert np.array_equal(flags[0], flags[1])
    assert (flags[1] != F.FLUID).sum() == 2 * nx + 2 * (ny - 2)
    p3 = F.SimulationParameters3D(fluid_nx=6, fluid_ny=5, fluid_nz=4)
    p3.boundaries = [F.BoundaryCondition([0, 0, 0], 5, [5, 4, 0]), F.BoundaryCondition([2, 2, 0], 13),
                     F.BoundaryCondition([-3, 1, 1], 24, [1, 1, 9])]
    f3 = F.flags_from_params(p3).reshape(4, 5, 6)
    assert (f3[0] == 5).sum() == 29 and f3[0, 2, 2] == 13
    assert (f3[1:, 1, :2] == 24).all() and (f3 == 24).sum() == 6


def _square_mesh(n):
    xs = np.linspace(0.0, 1.0, n + 1)
    v = np.array([[x, y] for y in xs for x in xs])
    t = []
    for j in range(n):
        for i in range(n):
            a = j * (n + 1) + i
            t += [[a, a + 1, a + n + 2], [a, a + n + 2, a + n + 1]]
    return v, np.array(t)


def test_medit_round_trip_and_2d_surface(tmp_path):
    v, t = _square_mesh(4)
    path = str(tmp_path / "sq.mesh")
    meshio.write_medit(path, v, triangles=t)
    m = meshio.load_medit(path, dimension=2)
    assert np.allclose(m.vertices, v) and np.array_equal(m.triangles, t)
    sv, se, ids = meshio.surface_of(m)
    assert se.shape == (16, 2) and len(sv) == 16          # 4 x 4 boundary edges, 16 boundary vertices
    # every boundary vertex lies on the unit square's boundary
    on = np.isclose(sv[:, 0], 0) | np.isclose(sv[:, 0], 1) | np.isclose(sv[:, 1], 0) | np.isclose(sv[:, 1], 1)
    assert on.all()
    # oriented edges form closed loops: every vertex starts exactly one edge and ends exactly one
    assert np.array_equal(np.sort(se[:, 0]), np.arange(16)) and np.array_equal(np.sort(se[:, 1]), np.arange(16))


def test_tet_boundary_faces():
    # a cube split into 6 tetrahedra around the diagonal 0-6: 12 boundary triangles
    v = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], float)
    tets = np.array([[0, 1, 2, 6], [0, 2, 3, 6], [0, 3, 7, 6], [0, 7, 4, 6], [0, 4, 5, 6], [0, 5, 1, 6]])
    faces = meshio.boundary_faces(tets)
    assert faces.shape == (12, 3)
    sv, se, _ = meshio.surface_of(meshio.MeditMesh(3, v, np.zeros((0, 3), int), tets))
    assert len(sv) == 8 and se.shape == (12, 3)


def test_medit_rejects_wrong_dimension_and_short_entries(tmp_path):
    v, t = _square_mesh(1)
    path = str(tmp_path / "s.mesh")
    meshio.write_medit(path, v, triangles=t)
    with pytest.raises(ValueError, match="3D mesh was expected"):
        meshio.load_medit(path, dimension=3)
    bad = tmp_path / "b.mesh"
    bad.write_text("MeshVersionFormatted 1\nDimension 2\nVertices\n2\n0 0\n1\n")
    with pytest.raises(ValueError, match="short"):
        meshio.load_medit(str(bad))


def test_place_follows_the_reference_conventions():
    # 2D: scale, then the reference's rotation (points turn by -rotate), then translate
    p = meshio.place(np.array([[1.0, 0.0]]), [10.0, 20.0], 90.0, [2.0, 1.0])
    assert np.allclose(p, [[10.0, 18.0]])
    # 3D: R = Ry(rot[1]) Rx(rot[0]) Rz(rot[2]); a quarter turn about z maps x to y
    q = meshio.place(np.array([[1.0, 0.0, 0.0]]), [0, 0, 0], [0.0, 0.0, 90.0], [1, 1, 1])
    assert np.allclose(q, [[0.0, 1.0, 0.0]], atol=1e-12)
    r = meshio.place(np.array([[0.0, 0.0, 1.0]]), [0, 0, 0], [0.0, 90.0, 0.0], [1, 1, 1])
    assert np.allclose(r, [[1.0, 0.0, 0.0]], atol=1e-12)
    assert math.isclose(np.linalg.norm(meshio.place(np.array([[3.0, 4.0, 0.0]]), [0, 0, 0], [10, 20, 30],
                                                    [1, 1, 1])), 5.0)


def test_solid_scene_volume_surface_and_map(tmp_path):
    """Two solids become one scene as FemScene builds it: volume vertices placed and
    concatenated in mesh order, volume triangles in volume numbering, surface edges
    in compact surface numbering, and a map from surface to volume vertices whose
    positions are the surface's."""
    v, t = _square_mesh(3)                      # 16 vertices, 4 interior, 18 triangles
    a, b = str(tmp_path / "a.mesh"), str(tmp_path / "b.mesh")
    meshio.write_medit(a, v, triangles=t)
    meshio.write_medit(b, v, triangles=t)
    p = F.SimulationParameters2D(fluid_nx=32, fluid_ny=16)
    p.solids = [F.SolidBodyConfig2D(mesh_path=a, translate=[0.1, 0.2], scale=[0.5, 0.5], rotate=0.0),
                F.SolidBodyConfig2D(mesh_path=b, translate=[0.6, 0.2], scale=[0.25, 0.25], rotate=30.0)]
    sc = F.build_solid_scene(p, 2)
    assert sc.positions.shape == (32, 2) and sc.elements.shape == (36, 3)
    assert np.array_equal(sc.elements[18:], t + 16)
    assert np.allclose(sc.positions[:16], meshio.place(v, [0.1, 0.2], 0.0, [0.5, 0.5]))
    assert np.allclose(sc.positions[16:], meshio.place(v, [0.6, 0.2], 30.0, [0.25, 0.25]))
    assert sc.surface_to_volume.size == 24 and sc.surface_elements.shape == (24, 2)
    interior = {5, 6, 9, 10}
    assert not (set(sc.surface_to_volume[:12].tolist()) & interior)
    assert not (set((sc.surface_to_volume[12:] - 16).tolist()) & interior)
    # surface elements of the second solid use surface indices 12..23 and map into its vertices
    assert sc.surface_elements[:12].max() < 12 and sc.surface_elements[12:].min() >= 12
    assert (sc.surface_to_volume[sc.surface_elements[12:]] >= 16).all()
    # each surface edge is an edge of a volume triangle
    tri_edges = {tuple(sorted(e)) for tr in sc.elements for e in ((tr[0], tr[1]), (tr[1], tr[2]), (tr[2], tr[0]))}
    for e in sc.surface_to_volume[sc.surface_elements]:
        assert tuple(sorted(e.tolist())) in tri_edges
    assert np.array_equal(sc.mesh_of_vertex, np.repeat([0, 1], 16))


def test_deformable_solid_controls_raise_clearly():
    p = F.SimulationParameters2D(fluid_nx=8, fluid_ny=8)
    sim = F.Simulator2D(p)
    for call in (lambda: sim.apply_lbs_control(0, [], []), lambda: sim.apply_active_strain(0, []),
                 lambda: sim.getLBSVertices()):
        try:
            call()
        except NotImplementedError:
            pass
        else:
            raise AssertionError("expected NotImplementedError")
    assert sim.getControlPointIdx() == []
