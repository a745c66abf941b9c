"""The reference's Python interface (``fsi_simulator``) for the fluid path.

FreeFlow's pybind11 module (``src/python/bindings.cpp:133-328``) exposes the
following names; this module mirrors them over ``libffs_lbm.so``:

- ``Config2D`` / ``Config3D`` (``load``, ``get_params``);
- ``SimulationParameters2D`` / ``SimulationParameters3D``, with the JSON fields of
  ``include/FSI_Simulator/utils/Config.hpp:103-225``;
- ``fem.SolidBodyConfig2D`` / ``fem.SolidBodyConfig3D`` and ``fem.FemSolverOptions``
  (``include/FSI_Simulator/fem/FemConfig.hpp``);
- ``Simulator2D`` / ``Simulator3D``.

Existing configuration files and driver scripts therefore load and step unchanged.

Scope is the fluid step.

- Solids are read from Medit ``.mesh`` files (:mod:`freeflow_b200.meshio`) and kept as the
  reference's ``FemScene`` keeps them: the vertices of all meshes, placed and concatenated in
  mesh order (the volume mesh), its elements, and the surface that enters the fluid step (boundary
  edges in 2D, boundary faces in 3D) with its surface-to-volume vertex map.
- Each step is ``ffs_lbm_step_coupled``: the surface is gathered out of the volume vertices, the
  fluid steps, and the fluid force of the step is written to the surface's volume vertices.
- The accessors return what the reference's return (``ISolidSolver.hpp:49-105, 163-220``):
  ``getVertices``, ``getVelocity`` and ``getForce`` the volume arrays, ``getTriangles`` /
  ``getTetrahedra`` the volume elements, ``getBoundaryVertices``, ``getBoundaryElements`` and
  ``getBoundaryPointIdx`` the surface, its elements and its vertex map.
- The ``"static"`` solid solver is mirrored: a rigid body moved by ``apply_kinematic_control``
  (``src/fem/StaticBodySolver.cpp:122-151``).
- The deformable solvers (``"vbd"``, Newton) and LBS control are outside this package. A
  configuration that names one loads and steps with a warning; the solid keeps its placed rest shape
  until a caller that owns a solid model sets the volume vertices with ``set_surface``.

Differences from the reference that a caller can see:

- ``getForce`` holds the fluid force of the last step at the surface's volume vertices (zero
  elsewhere), what ``applyForces`` writes for a deformable solver (``VBDSolver.cpp:101-113``). The
  reference's static solver ignores the forces (``StaticBodySolver.cpp:153-156``), so its
  ``getForce`` stays zero.
- ``get_fluid_moments(buffer="A")`` returns buffer A as the reference does (``Simulator2D.hpp:41-43``);
  the default returns the current buffer.
"""
from __future__ import annotations

import json
import os
import sys
import warnings
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import _capi as A
from . import meshio

# LbmNodeFlag names accepted in "boundaries" (Config.hpp:23-62); anything else is Invalid (0)
NODE_FLAGS = {
    "Wall": 5, "InletLeft": 13, "InletRight": 14, "InletUp": 15, "InletDown": 16, "InletFront": 17,
    "InletBack": 18, "OutletLeft": 19, "OutletRight": 20, "OutletUp": 21, "OutletDown": 22, "OutletFront": 23,
    "OutletBack": 24,
}
FLUID, SOLID_DYNAMIC = 1, 4


# ------------------------------------------------------------ parameters
@dataclass
class FemSolverOptions:
    optimizer_type: str = "newton"
    iterations: int = 10
    line_search_method: str = "backtracking"
    ls_max_iter: int = 10
    ls_beta: float = 0.5
    ls_alpha: float = 1e-4
    linear_solver_type: str = "eigen_ldlt"
    force_density_abs_tol: float = 1e-3
    grad_check: bool = False
    thread_ct: int = 8
    substeps: int = 3
    omega: float = 0.8
    vbd_iterations: int = 30


@dataclass
class LBSControlConfig:
    cnum: int = 2
    lbs_distance_type: str = "geodesic"
    random_first: bool = False
    omega: float = 0.5
    stiffness: float = 10.0


@dataclass
class SolidBodyConfig2D:
    mesh_path: str = ""
    density: float = 1000.0
    youngs_modulus: float = 1.0e6
    poisson_ratio: float = 0.45
    translate: list = field(default_factory=lambda: [0.0, 0.0])
    rotate: float = 0.0
    scale: list = field(default_factory=lambda: [1.0, 1.0])
    initial_velocity: list = field(default_factory=lambda: [0.0, 0.0])
    lbs_control_config: LBSControlConfig = field(default_factory=LBSControlConfig)


@dataclass
class SolidBodyConfig3D:
    mesh_path: str = ""
    density: float = 1000.0
    youngs_modulus: float = 1.0e6
    poisson_ratio: float = 0.45
    translate: list = field(default_factory=lambda: [0.0, 0.0, 0.0])
    rotate: list = field(default_factory=lambda: [0.0, 0.0, 0.0])
    scale: list = field(default_factory=lambda: [1.0, 1.0, 1.0])
    initial_velocity: list = field(default_factory=lambda: [0.0, 0.0, 0.0])
    lbs_control_config: LBSControlConfig = field(default_factory=LBSControlConfig)


class fem:  # noqa: N801 -- the reference's submodule name
    FemSolverOptions = FemSolverOptions
    SolidBodyConfig2D = SolidBodyConfig2D
    SolidBodyConfig3D = SolidBodyConfig3D
    LBSControlConfig = LBSControlConfig


@dataclass
class BoundaryCondition:
    """One "boundaries" entry: the cell at `position` (Config.hpp:23-62).  `to`
    is an extension of the JSON format: when an entry also has "to", it
    covers the inclusive box from "pos" to "to" (a wall row of a 1200-cell
    channel is then one entry instead of 1200)."""
    position: list
    flag: int
    to: Optional[list] = None


@dataclass
class SimulationParameters2D:
    dimension: int = 2
    fluid_viscosity: float = 0.001
    fluid_density: float = 1000.0
    fluid_nx: int = 400
    fluid_ny: int = 400
    fluid_dx: float = 1.0
    solid_solver_type: str = "static"
    total_time: float = 10.0
    dt: float = 0.001
    output_frequency: int = 100
    output_path: str = "./output"
    log_level: str = "info"
    log_file: str = "simulation.log"
    use_newton: bool = True
    boundaries: list = field(default_factory=list)
    boundary_velocities: list = field(default_factory=lambda: [0.0] * 4)
    global_fem_options: FemSolverOptions = field(default_factory=FemSolverOptions)
    solids: list = field(default_factory=list)

    def get_cf(self) -> float:
        """Force scale rho dx^2 dx / dt^2, in float as ``getCf`` (Config.hpp:96-100)."""
        cm = np.float32(self.fluid_density * self.fluid_dx * self.fluid_dx)
        return float(np.float32(float(cm) * self.fluid_dx / (self.dt * self.dt)))


@dataclass
class SimulationParameters3D:
    dimension: int = 3
    fluid_viscosity: float = 0.001
    fluid_density: float = 1000.0
    fluid_nx: int = 128
    fluid_ny: int = 128
    fluid_nz: int = 128
    fluid_dx: float = 1.0
    solid_solver_type: str = "static"
    total_time: float = 10.0
    dt: float = 0.001
    output_frequency: int = 100
    output_path: str = "./output"
    log_level: str = "info"
    log_file: str = "simulation.log"
    use_newton: bool = True
    boundaries: list = field(default_factory=list)
    boundary_velocities: list = field(default_factory=list)
    global_fem_options: FemSolverOptions = field(default_factory=FemSolverOptions)
    solids: list = field(default_factory=list)

    def get_cf(self) -> float:
        """Force scale rho dx^3 dx / dt^2, in float as ``getCf`` (Config.hpp:154-158)."""
        cm = np.float32(self.fluid_density * self.fluid_dx * self.fluid_dx * self.fluid_dx)
        return float(np.float32(float(cm) * self.fluid_dx / (self.dt * self.dt)))


def _fill(obj, j: dict, keys):
    """obj.k = j.get(k, obj.k) with the type of the default (json ``value``)."""
    for k in keys:
        if k in j:
            cur = getattr(obj, k)
            v = j[k]
            if isinstance(cur, bool):
                v = bool(v)
            elif isinstance(cur, int):
                v = int(v)
            elif isinstance(cur, float):
                v = float(v)
            elif isinstance(cur, list):
                v = [float(x) for x in v]
            setattr(obj, k, v)
    return obj


def _solid(j: dict, dim: int):
    c = SolidBodyConfig2D() if dim == 2 else SolidBodyConfig3D()
    _fill(c, j, ["mesh_path", "density", "youngs_modulus", "poisson_ratio", "translate", "scale",
                 "initial_velocity"])
    if "rotate" in j:
        c.rotate = float(j["rotate"]) if dim == 2 else [float(x) for x in j["rotate"]]
    if isinstance(j.get("lbs_control_config"), dict):
        _fill(c.lbs_control_config, j["lbs_control_config"], list(LBSControlConfig.__dataclass_fields__))
    return c


def params_from_json(j: dict, dim: int):
    """``from_json`` of SimulationParameters2D / 3D (Config.hpp:103-123, :160-225)."""
    p = SimulationParameters2D() if dim == 2 else SimulationParameters3D()
    keys = ["dimension", "fluid_viscosity", "fluid_density", "fluid_nx", "fluid_ny", "fluid_dx",
            "solid_solver_type", "total_time", "dt", "output_path", "log_level", "log_file", "use_newton",
            "boundary_velocities"]
    keys += ["output_frequency"] if dim == 2 else ["fluid_nz"]
    _fill(p, j, keys)
    if dim == 2 and "boundary_velocities" not in j:
        p.boundary_velocities = [0.0] * 4
    # std::vector<float> in the reference: the values pass through float
    p.boundary_velocities = [float(np.float32(v)) for v in p.boundary_velocities]
    if isinstance(j.get("global_fem_options"), dict):
        _fill(p.global_fem_options, j["global_fem_options"], list(FemSolverOptions.__dataclass_fields__))
    for bc in j.get("boundaries", []) or []:
        if not isinstance(bc, dict):
            warnings.warn("item in 'boundaries' is not an object; skipped")
            continue
        to = [int(x) for x in bc["to"]] if "to" in bc else None
        p.boundaries.append(BoundaryCondition([int(x) for x in bc["pos"]], NODE_FLAGS.get(bc["type"], 0), to))
    for s in j.get("solids", []) or []:
        if isinstance(s, dict):
            p.solids.append(_solid(s, dim))
        else:
            warnings.warn("item in 'solids' is not an object; skipped")
    return p


class _ConfigBase:
    DIM = 2

    def __init__(self):
        self._params = SimulationParameters2D() if self.DIM == 2 else SimulationParameters3D()

    def load(self, filepath: str) -> bool:
        """Parses the JSON file; False (with a message on stderr) when the file is missing,
        unreadable or not valid for these parameters (Config.cpp:9-109)."""
        if not os.path.exists(filepath):
            print(f"[Config FATAL] Configuration file not found at path: '{filepath}'", file=sys.stderr)
            return False
        try:
            with open(filepath) as f:
                data = json.load(f)
        except (OSError, ValueError) as e:
            print(f"[Config FATAL] JSON parsing failed in file '{filepath}': {e}", file=sys.stderr)
            return False
        try:
            self._params = params_from_json(data, self.DIM)
        except (KeyError, TypeError, ValueError) as e:
            print(f"[Config] JSON validation failed for {self.DIM}D parameters in '{filepath}': {e}",
                  file=sys.stderr)
            return False
        self._post_process()
        return True

    def _post_process(self):
        for bc in self._params.boundaries:
            if len(bc.position) != self.DIM:
                warnings.warn(f"boundary position {bc.position} should have {self.DIM} entries")
            if bc.flag == 0:
                warnings.warn(f"boundary condition at {bc.position} has an unrecognized type")
        n = len(self._params.boundary_velocities)
        if n and n != 2 * self.DIM:
            warnings.warn(f"`boundary_velocities` for {self.DIM}D should have {2 * self.DIM} elements; found {n}")

    def get_params(self):
        return self._params


class Config2D(_ConfigBase):
    DIM = 2


class Config3D(_ConfigBase):
    DIM = 3


def flags_from_params(p) -> np.ndarray:
    """Per-cell node flags: Fluid everywhere, then each boundary entry in file order (a later entry
    wins); entries outside the grid are ignored (LbmInitializer2D.cu:103-124 and its 3D twin).
    An entry with `to` sets every cell of its box, clipped to the grid."""
    dim = 2 if isinstance(p, SimulationParameters2D) else 3
    nx, ny, nz = p.fluid_nx, p.fluid_ny, (p.fluid_nz if dim == 3 else 1)
    f = np.full((nz, ny, nx), FLUID, dtype=np.uint8)
    for bc in p.boundaries:
        lo = list(bc.position[:dim]) + [0] * (3 - dim)
        if bc.to is None:
            x, y, z = lo
            if 0 <= x < nx and 0 <= y < ny and 0 <= z < nz:
                f[z, y, x] = bc.flag
            else:
                warnings.warn(f"boundary condition at {bc.position} is outside the grid and is ignored")
            continue
        hi = list(bc.to[:dim]) + [0] * (3 - dim)
        a = [max(min(lo[k], hi[k]), 0) for k in range(3)]
        b = [min(max(lo[k], hi[k]), n - 1) for k, n in enumerate((nx, ny, nz))]
        if any(a[k] > b[k] for k in range(3)):
            warnings.warn(f"boundary box {bc.position}..{bc.to} is outside the grid and is ignored")
            continue
        f[a[2]:b[2] + 1, a[1]:b[1] + 1, a[0]:b[0] + 1] = bc.flag
    return f.reshape(-1)


# ----------------------------------------------------------------- solids
@dataclass
class SolidScene:
    """The solids as FemScene holds them: volume vertices of all meshes (placed, concatenated in
    mesh order), volume elements (triangles in 2D, tetrahedra in 3D) in volume numbering, the
    surface elements in compact surface numbering, and each surface vertex's volume index."""
    positions: np.ndarray          # (nvol, dim) float64
    elements: np.ndarray           # (ne, dim + 1) int64
    surface_elements: np.ndarray   # (ns, dim) uint32
    surface_to_volume: np.ndarray  # (nsv,) uint32
    mesh_of_vertex: np.ndarray     # (nvol,) int64


def build_solid_scene(params, dim: int) -> SolidScene:
    """Loads and places every solid of the configuration (FemScene2D/3D set-up)."""
    pos, elems, surf, smap, owner = [], [], [], [], []
    vbase = sbase = 0
    for mid, s in enumerate(params.solids):
        mesh = meshio.load_medit(s.mesh_path, dimension=dim)
        v = meshio.place(mesh.vertices, s.translate, s.rotate, s.scale)
        vol_el = mesh.triangles if dim == 2 else mesh.tetrahedra
        _, se, ids = meshio.surface_of(mesh)
        pos.append(v)
        elems.append(vol_el.astype(np.int64) + vbase)
        surf.append(se.astype(np.int64) + sbase)
        smap.append(ids.astype(np.int64) + vbase)
        owner.append(np.full(len(v), mid))
        vbase += len(v)
        sbase += len(ids)
    if not pos:
        z = np.zeros
        return SolidScene(z((0, dim)), z((0, dim + 1), np.int64), z((0, dim), np.uint32), z(0, np.uint32),
                          z(0, np.int64))
    return SolidScene(np.concatenate(pos), np.concatenate(elems), np.concatenate(surf).astype(np.uint32),
                      np.concatenate(smap).astype(np.uint32), np.concatenate(owner))


# ------------------------------------------------------------- simulators
class _SimulatorBase:
    DIM = 2

    def __init__(self, params, storage: str = "f32"):
        self.m_params = params
        self.storage = storage
        self._grid = None
        self._vs = None
        self._fluid_enabled = True
        self._profile_name = None
        self._targets, self._vel, self._target_index = [], 0.0, -1

    # -- set-up
    def initialize(self):
        from .grid import FluidGrid, VolumeSurface

        p = self.m_params
        if p.solid_solver_type not in ("static",):
            # a configuration written for a deformable solver (fish2d_lbs_control.json: "vbd") still
            # loads and steps: the solid keeps its placed rest shape until its owner sets the vertices
            warnings.warn(f"solid_solver_type '{p.solid_solver_type}': the deformable solid solvers are not part "
                          "of this package; the solid keeps its rest shape until set_surface() moves it")
        bc = list(p.boundary_velocities)
        if len(bc) != 2 * self.DIM:
            bc = [0.0] * (2 * self.DIM)
        self._grid = FluidGrid(dim=self.DIM, nx=p.fluid_nx, ny=p.fluid_ny, nz=getattr(p, "fluid_nz", 1),
                               fluid_viscosity=p.fluid_viscosity, fluid_density=p.fluid_density,
                               fluid_dx=p.fluid_dx, dt=p.dt, boundary_velocities=bc, storage=self.storage)
        self._flags = flags_from_params(p)
        self._grid.set_flags(self._flags)
        self._grid.initialize()
        self._scene = build_solid_scene(p, self.DIM)
        sc = self._scene
        if len(sc.positions):
            self._rest = sc.positions.copy()
            self._vel0 = np.concatenate([np.tile(np.asarray(s.initial_velocity, np.float64)[:self.DIM],
                                                 (int((sc.mesh_of_vertex == mid).sum()), 1))
                                         for mid, s in enumerate(p.solids)])
            self._pos = self._rest.copy()
            self._vel_now = self._vel0.copy()
            self._marker0 = self._rest[0].copy()   # the static solver's marker: the scene's first vertex
            self._marker = self._marker0.copy()
            self._vs = VolumeSurface(self._pos, self._vel_now, sc.surface_to_volume, sc.surface_elements)

    def reset(self):
        if self._grid is not None:
            self._grid.set_flags(self._flags)
            self._grid.initialize()
        if self._vs is not None:
            self._pos = self._rest.copy()
            self._vel_now = np.zeros_like(self._vel0)
            self._marker = self._marker0.copy()
            self._vs.update(self._pos, self._vel_now)
            self._vs.volume_forces.zero_()
        self._targets, self._vel, self._target_index = [], 0.0, -1

    def enableFluidSolver(self, enable: bool):  # noqa: N802 -- reference name
        self._fluid_enabled = bool(enable)

    # -- stepping (Simulator2D.cpp:88-130)
    def step(self):
        if self._fluid_enabled:
            if self._vs is not None:
                self._grid.step_coupled(self._vs)
            else:
                self._grid.step()
        self._advance_solid()

    def set_surface(self, vertices, velocities):
        """Positions and velocities of every vertex of the solids' volume mesh (physical units), for
        a caller that owns the solid model; the surface is gathered from them at every step."""
        self._pos = np.asarray(vertices, np.float64).reshape(-1, self.DIM)
        self._vel_now = np.asarray(velocities, np.float64).reshape(-1, self.DIM)
        self._vs.update(self._pos, self._vel_now)

    def apply_kinematic_control(self, mesh_id: int, target_pos, vel: float):
        """StaticBodySolver::applyKinematicControl (StaticBodySolver.cpp:158-180): the body moves
        rigidly through `target_pos` at speed `vel`, with the first mesh vertex as the marker."""
        if mesh_id < 0 or mesh_id >= len(self.m_params.solids):
            warnings.warn(f"invalid mesh_id {mesh_id} for kinematic control")
            return
        if len(target_pos) < 2:
            warnings.warn("at least two target positions are required for kinematic control")
            return
        if vel <= 0.0:
            warnings.warn("velocity must be positive for kinematic control")
            return
        self._targets = [np.asarray(t, np.float64) for t in target_pos]
        self._vel = float(vel)
        self._target_index = -1

    def _advance_solid(self):
        # StaticBodySolver2D/3D::advanceTimeStep (StaticBodySolver.cpp:122-151): every vertex of
        # the scene moves with the marker's velocity
        if not self._targets or self._vel <= 0.0 or self._vs is None:
            return
        dt = self.m_params.dt
        marker = self._marker
        if self._target_index < 0:
            self._target_index = 0
        target = self._targets[self._target_index]
        if np.linalg.norm(target - marker) < dt * self._vel:
            self._target_index = (self._target_index + 1) % len(self._targets)
            target = self._targets[self._target_index]
        d = target - marker
        v = self._vel * d / np.linalg.norm(d)
        self._vel_now[:] = v
        self._pos += v * dt
        self._marker = self._marker + v * dt
        self._vs.update(self._pos, self._vel_now)

    # -- accessors (bindings.cpp:307-321)
    def get_fluid_moments(self, buffer: str = "current") -> np.ndarray:
        """Moments in the reference layout, (ny, nx, 6) in 2D or (nz, ny, nx, 10) in 3D.
        buffer="A" returns buffer A, as the reference's getFluidMoment does."""
        which = A.BUF_A if buffer == "A" else A.BUF_CURRENT
        m = self._grid.get_moments(which=which)
        p = self.m_params
        shape = (p.fluid_ny, p.fluid_nx, 6) if self.DIM == 2 else (p.fluid_nz, p.fluid_ny, p.fluid_nx, 10)
        return m.reshape(shape)

    # ISolidSolver2D/3D accessors (ISolidSolver.hpp:49-105, 163-220)
    def _none(self, width=None):
        return np.zeros((0, width or self.DIM), np.float32)

    def getVertices(self):  # noqa: N802
        """Positions of every vertex of the solids' volume mesh."""
        return self._pos.astype(np.float32) if self._vs is not None else self._none()

    def getVelocity(self):  # noqa: N802
        return self._vel_now.astype(np.float32) if self._vs is not None else self._none()

    def getForce(self):  # noqa: N802
        """Fluid force of the last step on each volume vertex (zero off the surface)."""
        return self._vs.volume_forces.cpu().numpy() if self._vs is not None else self._none()

    def getBoundaryVertices(self):  # noqa: N802
        """Positions of the surface vertices (the surface the fluid step sees)."""
        if self._vs is None:
            return self._none()
        return self._pos[self._scene.surface_to_volume].astype(np.float32)

    def getBoundaryElements(self):  # noqa: N802
        """Surface elements, flattened, in surface-vertex numbering."""
        return self._scene.surface_elements.reshape(-1).copy() if self._vs is not None else np.zeros(0, np.uint32)

    def getBoundaryPointIdx(self):  # noqa: N802
        """Volume index of each surface vertex (the surface-to-volume map)."""
        return self._scene.surface_to_volume.copy() if self._vs is not None else np.zeros(0, np.uint32)

    def getControlPointIdx(self):  # noqa: N802
        """LBS control points; LBS control is not part of this package, so there are none."""
        return []

    def getLBSVertices(self):  # noqa: N802
        raise NotImplementedError("LBS control is not supported for the static solid solver")

    # solid-model controls of the reference that belong to the deformable solvers
    def apply_lbs_control(self, *args, **kwargs):
        """Simulator2D/3D::applyLBSControl (LBS control of a deformable solid): not part of the
        fluid step; a caller with its own solid model sets the vertices with set_surface()."""
        raise NotImplementedError("LBS control belongs to the deformable solid solvers, outside this package")

    def apply_active_strain(self, *args, **kwargs):
        """Simulator2D::applyActiveStrain (active strain of a deformable solid): not part of the
        fluid step."""
        raise NotImplementedError("active strain belongs to the deformable solid solvers, outside this package")

    def _surface_now(self):
        from .grid import DeviceSurface

        m = self._scene.surface_to_volume
        return DeviceSurface(self._pos[m], self._vel_now[m], self._scene.surface_elements)

    def status(self) -> int:
        """Device status bits (non-finite state, link overflow, force range, bad element); clears them."""
        return self._grid.status()

    def save_frame_data(self, frame_index: int):
        """Writes moments and surface of this frame to <output_path>/frame_<index>.npz (the
        reference's VTK writer is outside the fluid step)."""
        os.makedirs(self.m_params.output_path, exist_ok=True)
        np.savez(os.path.join(self.m_params.output_path, f"frame_{int(frame_index):06d}.npz"),
                 moments=self.get_fluid_moments(), vertices=self.getVertices(), velocities=self.getVelocity(),
                 forces=self.getForce(), boundary_elements=self.getBoundaryElements(),
                 boundary_point_idx=self.getBoundaryPointIdx())

    def begin_profiler(self, name: str):
        """Starts per-stage CUDA-event timing of the steps (detect, dense, link cells, forces)."""
        self._profile_name = name
        self._grid.profile(True)
        self._grid.profile_read(reset=True)

    def end_profiler(self) -> dict:
        """Stops timing; prints and returns {stage: (ms total, launches)}."""
        self._grid.profile(False)
        rep = self._grid.profile_read(reset=True)
        print(f"[profile {self._profile_name}] " +
              ", ".join(f"{k} {v[0]:.3f} ms / {v[1]}" for k, v in rep.items() if v[1]))
        return rep

    def close(self):
        if self._grid is not None:
            self._grid.close()
            self._grid = None


class Simulator2D(_SimulatorBase):
    DIM = 2

    def getTriangles(self):  # noqa: N802
        """Triangles of the solids' volume mesh, flattened, in volume numbering."""
        return self._scene.elements.reshape(-1).astype(np.uint32) if self._vs is not None else np.zeros(0, np.uint32)

    def fill_solid(self):
        """fillSolidFlags2D (FsiCoupling2D.cu:434-464): fluid cells inside the solid become
        SolidDynamic; returns their [x, y] list (Simulator2D.cpp:132-151)."""
        self._grid.fill_solid(self._surface_now())
        f = self._grid.get_flags()
        idx = np.nonzero(f == SOLID_DYNAMIC)[0]
        return [[int(i % self.m_params.fluid_nx), int(i // self.m_params.fluid_nx)] for i in idx]

    fillSolid = fill_solid


class Simulator3D(_SimulatorBase):
    DIM = 3

    def getTetrahedra(self):  # noqa: N802
        """Tetrahedra of the solids' volume mesh, flattened, in volume numbering (none for a
        solid given as a surface mesh)."""
        return self._scene.elements.reshape(-1).astype(np.uint32) if self._vs is not None else np.zeros(0, np.uint32)
