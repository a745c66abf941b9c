"""Drop-in check against FreeFlow's own shipped files (copied unmodified into
tests/golden/reference_assets/ by tests/golden/make_reference_assets.py):
the configurations vortexstreet2d.json and fish2d_lbs_control.json and the
Medit meshes fish2d.mesh and sphere2d.mesh.

Each expectation is restated here from the reference's source, independently
of the package code under test:

* parameters and defaults: ``from_json`` of SimulationParameters2D
  (include/FSI_Simulator/utils/Config.hpp:103-123), FemSolverOptions
  (include/FSI_Simulator/fem/FemConfig.hpp:48-65), LBSControlConfig (:79-86)
  and SolidBodyConfig2D (:105-116), with the member defaults of the structs;
* node flags: initializeState2D (src/lbm/LbmInitializer2D.cu:103-124), with
  the flag numbers of LbmNodeFlag (include/FSI_Simulator/lbm/LbmDataTypes.cuh:17-56);
* the mesh: MeshLoader2D::load (src/io/MeshLoader.cpp:147-271);
* the placement: Mesh2D::applyInitialTransform (src/fem/DeformableMesh.cpp:403-423).
"""
import gzip
import hashlib
import json
import math
import os
import warnings

import numpy as np
import pytest

from freeflow_b200 import fsi_simulator as F
from freeflow_b200 import meshio

ASSETS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_assets")
MANIFEST = json.load(open(os.path.join(ASSETS, "MANIFEST.json")))
CONFIGS = ["vortexstreet2d.json", "fish2d_lbs_control.json"]
MESHES = ["fish2d.mesh", "sphere2d.mesh"]


def asset_bytes(name):
    with open(os.path.join(ASSETS, name + ".gz"), "rb") as f:
        return gzip.decompress(f.read())


def asset_file(tmp_path, name):
    path = tmp_path / name
    path.write_bytes(asset_bytes(name))
    return str(path)


# ---------------------------------------------------------------- restatements
# LbmNodeFlag, in declaration order (LbmDataTypes.cuh:17-56)
_ENUM = ["Invalid", "Fluid", "FluidRest", "Solid", "SolidDynamic", "Wall", "WallLeft", "WallRight",
         "WallFront", "WallBack", "WallDown", "WallUp", "WallCorner", "InletLeft", "InletRight", "InletUp",
         "InletDown", "InletFront", "InletBack", "OutletLeft", "OutletRight", "OutletUp", "OutletDown",
         "OutletFront", "OutletBack", "Receptor", "Deactivated", "Smoke"]
# the "type" strings that from_json(BoundaryCondition) maps (Config.hpp:29-62); others are Invalid
_BC_TYPES = {"Wall", "InletLeft", "InletRight", "InletUp", "InletDown", "InletFront", "InletBack",
             "OutletLeft", "OutletRight", "OutletUp", "OutletDown", "OutletFront", "OutletBack"}

_PARAM_DEFAULTS = {  # SimulationParameters2D members (Config.hpp:64-95)
    "dimension": 2, "fluid_viscosity": 0.001, "fluid_density": 1000.0, "fluid_nx": 400, "fluid_ny": 400,
    "fluid_dx": 1.0, "solid_solver_type": "static", "total_time": 10.0, "dt": 0.001, "output_frequency": 100,
    "output_path": "./output", "log_level": "info", "log_file": "simulation.log", "use_newton": True,
}
_FEM_DEFAULTS = {  # FemSolverOptions members (FemConfig.hpp:14-46)
    "optimizer_type": "newton", "iterations": 10, "line_search_method": "backtracking", "ls_max_iter": 10,
    "ls_beta": 0.5, "ls_alpha": 1e-4, "linear_solver_type": "eigen_ldlt", "force_density_abs_tol": 1e-3,
    "grad_check": False, "thread_ct": 8, "substeps": 3, "omega": 0.8, "vbd_iterations": 30,
}
_LBS_DEFAULTS = {"cnum": 2, "lbs_distance_type": "geodesic", "random_first": False, "omega": 0.5,
                 "stiffness": 10.0}
_SOLID_DEFAULTS = {"mesh_path": "", "density": 1000.0, "youngs_modulus": 1.0e6, "poisson_ratio": 0.45,
                   "translate": [0.0, 0.0], "rotate": 0.0, "scale": [1.0, 1.0], "initial_velocity": [0.0, 0.0]}


def value(j, key, default):
    """nlohmann::json::value(key, default): the member if present, else the default."""
    return j[key] if key in j else default


def ref_flags(j):
    """initializeState2D (LbmInitializer2D.cu:103-124): Fluid everywhere, then every boundary
    entry in file order; entries outside the grid are skipped."""
    nx, ny = value(j, "fluid_nx", 400), value(j, "fluid_ny", 400)
    flags = [_ENUM.index("Fluid")] * (nx * ny)
    for bc in value(j, "boundaries", []):
        x, y = bc["pos"][0], bc["pos"][1]
        flag = _ENUM.index(bc["type"]) if bc["type"] in _BC_TYPES else 0
        if 0 <= x < nx and 0 <= y < ny:
            flags[y * nx + x] = flag
    return np.array(flags, dtype=np.uint8)


def ref_load_mesh2d(text):
    """MeshLoader2D::load (MeshLoader.cpp:147-271), line by line: two header lines, then blocks
    whose keyword is the whole line; vertices read as two doubles, indices made 0-based."""
    lines = text.split("\n")
    pos = 0

    def getline():
        nonlocal pos
        line = lines[pos] if pos < len(lines) else None
        pos += 1
        return line

    kw, version = getline().split()[:2]
    assert kw == "MeshVersionFormatted"
    kw, dim = getline().split()[:2]
    assert kw == "Dimension" and int(dim) == 2
    verts, edges, tris = [], [], []
    while True:
        line = getline()
        if line is None:
            break
        if not line.strip():
            continue
        if line in ("Vertices", "Edges", "Triangles"):
            count = int(getline())
            for _ in range(count):
                t = getline().split()
                if line == "Vertices":
                    verts.append((float(t[0]), float(t[1])))
                elif line == "Edges":
                    edges.append((int(t[0]) - 1, int(t[1]) - 1))
                else:
                    tris.append((int(t[0]) - 1, int(t[1]) - 1, int(t[2]) - 1))
    return np.array(verts), np.array(edges, dtype=np.int64).reshape(-1, 2), np.array(tris, dtype=np.int64)


def ref_place2d(v, translate, rotate, scale):
    """Mesh2D::applyInitialTransform (DeformableMesh.cpp:403-423) in double: scale and translate
    through float, the angle as glm::radians(float(rotate)) in float, and glm's column-major
    mat2(cos, -sin, sin, cos) applied to (scale * v)."""
    f32 = np.float32
    sx, sy = float(f32(scale[0])), float(f32(scale[1]))
    a = float(f32(f32(rotate) * f32(0.01745329251994329576923690768489)))
    c, s = math.cos(a), math.sin(a)
    tx, ty = float(f32(translate[0])), float(f32(translate[1]))
    out = np.empty_like(v)
    for i, (x, y) in enumerate(v):
        x, y = sx * x, sy * y
        out[i] = (c * x + s * y + tx, -s * x + c * y + ty)
    return out


# ------------------------------------------------------------------------ tests
@pytest.mark.parametrize("name", CONFIGS + MESHES)
def test_assets_are_the_reference_files(name):
    data = asset_bytes(name)
    entry = MANIFEST["files"][name]
    assert len(data) == entry["bytes"]
    assert hashlib.sha256(data).hexdigest() == entry["sha256"]


@pytest.mark.parametrize("name", CONFIGS)
def test_config2d_load_gives_every_field_and_default(tmp_path, name):
    j = json.loads(asset_bytes(name))
    c = F.Config2D()
    assert c.load(asset_file(tmp_path, name))
    p = c.get_params()
    for key, default in _PARAM_DEFAULTS.items():
        assert getattr(p, key) == value(j, key, default), key
    # std::vector<float>: the velocities pass through float
    bv = value(j, "boundary_velocities", [0.0] * 4)
    assert p.boundary_velocities == [float(np.float32(v)) for v in bv]
    fem = value(j, "global_fem_options", {})
    for key, default in _FEM_DEFAULTS.items():
        assert getattr(p.global_fem_options, key) == value(fem, key, default), key
    assert len(p.solids) == len(j["solids"])
    for got, js in zip(p.solids, j["solids"]):
        for key, default in _SOLID_DEFAULTS.items():
            want = value(js, key, default)
            assert getattr(got, key) == (float(want) if key == "rotate" else want), key
        lbs = value(js, "lbs_control_config", {})
        for key, default in _LBS_DEFAULTS.items():
            assert getattr(got.lbs_control_config, key) == value(lbs, key, default), key
    assert len(p.boundaries) == len(j["boundaries"])


def test_config_values_the_shipped_files_hold():
    """Spot values, so that a silent change of the fixtures or of the parser shows."""
    v = json.loads(asset_bytes("vortexstreet2d.json"))
    f = json.loads(asset_bytes("fish2d_lbs_control.json"))
    assert (v["fluid_nx"], v["fluid_ny"], v["dt"], v["fluid_dx"]) == (801, 201, 0.0025, 0.005)
    assert (f["fluid_nx"], f["fluid_ny"], f["solid_solver_type"]) == (1200, 400, "vbd")
    assert len(v["boundaries"]) == 2004 and len(f["boundaries"]) == 3200


@pytest.mark.parametrize("name", CONFIGS)
def test_flags_equal_the_reference_initialiser(tmp_path, name):
    j = json.loads(asset_bytes(name))
    c = F.Config2D()
    assert c.load(asset_file(tmp_path, name))
    got = F.flags_from_params(c.get_params())
    want = ref_flags(j)
    assert got.dtype == np.uint8 and np.array_equal(got, want)
    # the later entry wins where two entries name one cell (the corners of fish2d_lbs_control)
    seen = {}
    for bc in j["boundaries"]:
        seen[tuple(bc["pos"])] = bc["type"]
    nx = j["fluid_nx"]
    for (x, y), t in seen.items():
        assert got[y * nx + x] == _ENUM.index(t)


@pytest.mark.parametrize("name", MESHES)
def test_mesh_loads_as_the_reference_loader(tmp_path, name):
    text = asset_bytes(name).decode()
    verts, edges, tris = ref_load_mesh2d(text)
    with warnings.catch_warnings():
        warnings.simplefilter("error")     # every line of the shipped file is understood
        m = meshio.load_medit(asset_file(tmp_path, name), dimension=2)
    assert m.dimension == 2
    assert m.vertices.dtype == np.float64 and np.array_equal(m.vertices, verts)
    assert np.array_equal(m.triangles, tris)
    assert np.array_equal(m.edges, edges)
    assert len(tris) > 0 and tris.min() == 0 and tris.max() == len(verts) - 1


@pytest.mark.parametrize("config,mesh", [("fish2d_lbs_control.json", "fish2d.mesh"),
                                         ("vortexstreet2d.json", "sphere2d.mesh")])
def test_solid_scene_of_the_shipped_config(tmp_path, config, mesh):
    c = F.Config2D()
    assert c.load(asset_file(tmp_path, config))
    p = c.get_params()
    s = p.solids[0]
    assert os.path.basename(s.mesh_path) == mesh
    s.mesh_path = asset_file(tmp_path, mesh)
    sc = F.build_solid_scene(p, 2)
    verts, _, tris = ref_load_mesh2d(asset_bytes(mesh).decode())
    want = ref_place2d(verts, s.translate, s.rotate, s.scale)
    assert np.array_equal(sc.positions, want)
    assert np.array_equal(sc.elements, tris)
    # the surface: edges used by one triangle; a closed polygon through the map
    se, smap = sc.surface_elements.astype(np.int64), sc.surface_to_volume.astype(np.int64)
    e = np.sort(np.concatenate([tris[:, [0, 1]], tris[:, [1, 2]], tris[:, [2, 0]]]), axis=1)
    keys, cnt = np.unique(e, axis=0, return_counts=True)
    boundary = {tuple(k) for k in keys[cnt == 1]}
    assert {tuple(sorted(x)) for x in smap[se]} == boundary
    deg = np.bincount(se.reshape(-1), minlength=len(smap))
    assert (deg == 2).all()
    # the body lies inside the fluid box (lattice units)
    lat = sc.positions / p.fluid_dx
    assert lat.min() > 0 and lat[:, 0].max() < p.fluid_nx - 1 and lat[:, 1].max() < p.fluid_ny - 1
