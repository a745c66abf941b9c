"""Python handle on one fluid grid, calling the C ABI (``include/ffs_lbm.h``).

This is the Python-side equivalent of FreeFlow's ``LbmFlowField2D/3D`` plus
``fsi_coupling::solveLbmAndFsiStep2D/3D``.  Device memory for surfaces comes
from torch tensors (plumbing only); every computation runs in the CUDA
kernels of ``libffs_lbm.so``.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _capi as A


def _stream_handle(stream) -> C.c_void_p:
    if stream is None:
        return C.c_void_p(0)
    if isinstance(stream, int):
        return C.c_void_p(stream)
    h = getattr(stream, "cuda_stream", None)
    if h is not None:
        return C.c_void_p(int(h))
    return C.c_void_p(int(stream))


def _np_ptr(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


class DeviceSurface:
    """Surface arrays on the device, the SolidGeometryProxy_Device view.

    vertices / velocities: (nv, dim) float32, physical units; elements:
    (ne, dim) uint32 vertex indices (segments in 2D, triangles in 3D).
    ``forces`` (nv, dim) float32 accumulates the fluid force (+=) and
    ``forces64`` (optional) the same in float64.
    """

    def __init__(self, vertices, velocities, elements, device="cuda", with_forces64=False):
        import torch

        # torch.tensor copies: the object never aliases the caller's arrays
        self.vertices = torch.tensor(np.ascontiguousarray(vertices, dtype=np.float32), device=device)
        self.dim = int(self.vertices.shape[1])
        self.velocities = torch.tensor(np.ascontiguousarray(velocities, dtype=np.float32), device=device)
        e = np.ascontiguousarray(elements, dtype=np.uint32).reshape(-1, self.dim)
        # torch has no uint32 arithmetic we need; keep raw bytes in int32
        self.elements = torch.tensor(e.view(np.int32), device=device)
        self.forces = torch.zeros_like(self.vertices)
        self.forces64 = torch.zeros(self.vertices.shape, dtype=torch.float64, device=device) if with_forces64 else None
        assert self.velocities.shape == self.vertices.shape

    @property
    def num_vertices(self) -> int:
        return int(self.vertices.shape[0])

    @property
    def num_elements(self) -> int:
        return int(self.elements.shape[0])

    def update(self, vertices=None, velocities=None):
        if vertices is not None:
            self.vertices.copy_(self._t(vertices))
        if velocities is not None:
            self.velocities.copy_(self._t(velocities))

    def _t(self, a):
        import torch
        if isinstance(a, torch.Tensor):
            return a.to(self.vertices.device, torch.float32)
        return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32))

    def c_struct(self) -> A.Surface:
        s = A.Surface()
        s.dim = self.dim
        s.vertices = self.vertices.data_ptr()
        s.velocities = self.velocities.data_ptr()
        s.elements = self.elements.data_ptr()
        s.num_vertices = self.num_vertices
        s.num_elements = self.num_elements
        s.forces = self.forces.data_ptr()
        s.forces64 = self.forces64.data_ptr() if self.forces64 is not None else None
        return s


class VolumeSurface:
    """A surface given as the boundary of a solid's volume mesh (the reference's
    FsiCouplingDataGpu view): the solid's vertex arrays on the device plus the
    surface-to-volume vertex map, for :meth:`FluidGrid.step_coupled`.

    volume_positions / volume_velocities: (nvol, dim) float32, physical units;
    surface_to_volume: (nv,) volume index of each surface vertex; elements:
    (ne, dim) surface-vertex indices.  After each coupled step
    ``volume_forces`` (nvol, dim) holds that step's fluid force at the mapped
    vertices and zero elsewhere; ``surface_positions`` / ``surface_velocities``
    hold the gathered surface.
    """

    def __init__(self, volume_positions, volume_velocities, surface_to_volume, elements, device="cuda"):
        import torch

        # torch.tensor copies: the object never aliases the caller's arrays
        vp = np.ascontiguousarray(volume_positions, dtype=np.float32)
        self.dim = int(vp.shape[1])
        self.volume_positions = torch.tensor(vp, device=device)
        self.volume_velocities = torch.tensor(np.ascontiguousarray(volume_velocities, dtype=np.float32), device=device)
        assert self.volume_velocities.shape == self.volume_positions.shape
        self.volume_forces = torch.zeros_like(self.volume_positions)
        m = np.ascontiguousarray(surface_to_volume, dtype=np.uint32).reshape(-1)
        self.surface_to_volume = torch.tensor(m.view(np.int32), device=device)
        e = np.ascontiguousarray(elements, dtype=np.uint32).reshape(-1, self.dim)
        self.elements = torch.tensor(e.view(np.int32), device=device)
        self.surface_positions = torch.zeros((m.size, self.dim), dtype=torch.float32, device=device)
        self.surface_velocities = torch.zeros_like(self.surface_positions)

    def update(self, volume_positions=None, volume_velocities=None):
        import torch

        for dst, a in ((self.volume_positions, volume_positions), (self.volume_velocities, volume_velocities)):
            if a is not None:
                dst.copy_(a.to(dst.device, torch.float32) if isinstance(a, torch.Tensor)
                          else torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32)))

    def c_struct(self) -> A.VolumeSurface:
        s = A.VolumeSurface()
        s.dim = self.dim
        s.num_volume_vertices = int(self.volume_positions.shape[0])
        s.volume_positions = self.volume_positions.data_ptr()
        s.volume_velocities = self.volume_velocities.data_ptr()
        s.volume_forces = self.volume_forces.data_ptr()
        s.num_vertices = int(self.surface_to_volume.shape[0])
        s.num_elements = int(self.elements.shape[0])
        s.surface_to_volume = self.surface_to_volume.data_ptr()
        s.elements = self.elements.data_ptr()
        s.surface_positions = self.surface_positions.data_ptr()
        s.surface_velocities = self.surface_velocities.data_ptr()
        return s


@dataclass
class GridInfo:
    ncell: int
    nm: int
    q: int
    omega: float
    cf: float


class FluidGrid:
    """One D2Q9 / D3Q27 fluid grid resident on the GPU."""

    def __init__(self, dim: int, nx: int, ny: int, nz: int = 1, fluid_viscosity: float = 0.001,
                 fluid_density: float = 1000.0, fluid_dx: float = 1.0, dt: float = 0.001,
                 boundary_velocities=None, storage: str = "f32", periodic: int = 0,
                 ref_half_populations: bool = False, ref_2d_wall_stream: bool = False):
        L = A.load()
        d = A.LbmDesc()
        d.dim, d.nx, d.ny, d.nz = dim, nx, ny, (1 if dim == 2 else nz)
        d.fluid_viscosity, d.fluid_density, d.fluid_dx, d.dt = fluid_viscosity, fluid_density, fluid_dx, dt
        bc = list(boundary_velocities or [])
        for i in range(6):
            d.boundary_velocities[i] = float(bc[i]) if i < len(bc) else 0.0
        d.storage = A.STORAGE[storage] if isinstance(storage, str) else int(storage)
        d.periodic_mask = int(periodic)
        d.ref_half_populations = int(bool(ref_half_populations))
        d.ref_2d_wall_stream = int(bool(ref_2d_wall_stream))
        self._h = C.c_void_p()
        A.check(L.ffs_lbm_create(C.byref(d), C.byref(self._h)), "ffs_lbm_create")
        self.dim, self.nx, self.ny, self.nz = dim, nx, ny, d.nz
        self.storage = storage
        self.info = self._info()

    # -- life cycle ---------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            A.load().ffs_lbm_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _info(self) -> GridInfo:
        n = C.c_int64()
        nm, q = C.c_int(), C.c_int()
        om, cf = C.c_double(), C.c_double()
        A.check(A.load().ffs_lbm_get_info(self._h, C.byref(n), C.byref(nm), C.byref(q), C.byref(om), C.byref(cf)),
                "ffs_lbm_get_info")
        return GridInfo(n.value, nm.value, q.value, om.value, cf.value)

    @property
    def ncell(self) -> int:
        return self.info.ncell

    @property
    def nm(self) -> int:
        return self.info.nm

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    # -- state ---------------------------------------------------------------
    def set_flags(self, flags, stream=None):
        f = np.ascontiguousarray(flags, dtype=np.uint8).reshape(-1)
        assert f.size == self.ncell
        A.check(A.load().ffs_lbm_set_flags(self._h, _np_ptr(f), A.MEM_HOST, _stream_handle(stream)), "set_flags")

    def get_flags(self, stream=None) -> np.ndarray:
        f = np.zeros(self.ncell, dtype=np.uint8)
        A.check(A.load().ffs_lbm_get_flags(self._h, _np_ptr(f), A.MEM_HOST, _stream_handle(stream)), "get_flags")
        return f

    def initialize(self, stream=None):
        A.check(A.load().ffs_lbm_initialize(self._h, _stream_handle(stream)), "initialize")

    def set_moments(self, m, which: int = A.BUF_BOTH, layout: int = A.LAYOUT_AOS, stream=None):
        a = np.ascontiguousarray(m, dtype=np.float32).reshape(-1)
        assert a.size == self.ncell * self.nm
        A.check(A.load().ffs_lbm_set_moments(self._h, _np_ptr(a), layout, A.MEM_HOST, which, _stream_handle(stream)),
                "set_moments")

    def get_moments(self, which: int = A.BUF_CURRENT, layout: int = A.LAYOUT_AOS, stream=None) -> np.ndarray:
        a = np.zeros(self.ncell * self.nm, dtype=np.float32)
        A.check(A.load().ffs_lbm_get_moments(self._h, _np_ptr(a), layout, A.MEM_HOST, which, _stream_handle(stream)),
                "get_moments")
        return a.reshape(self.ncell, self.nm) if layout == A.LAYOUT_AOS else a.reshape(self.nm, self.ncell)

    def reserve_surface(self, max_vertices: int, max_link_cells: int):
        A.check(A.load().ffs_lbm_reserve_surface(self._h, int(max_vertices), int(max_link_cells)), "reserve_surface")

    # -- stepping -------------------------------------------------------------
    def step(self, surface: DeviceSurface | None = None, stream=None):
        s = surface.c_struct() if surface is not None else None
        A.check(A.load().ffs_lbm_step(self._h, C.byref(s) if s is not None else None, _stream_handle(stream)), "step")

    def step_coupled(self, surface: VolumeSurface, stream=None):
        """One coupled step (ffs_lbm_step_coupled): gather the surface from the volume mesh,
        step the fluid, write this step's forces to ``surface.volume_forces``."""
        s = surface.c_struct()
        A.check(A.load().ffs_lbm_step_coupled(self._h, C.byref(s), _stream_handle(stream)), "step_coupled")

    def fill_solid(self, surface: DeviceSurface, stream=None):
        s = surface.c_struct()
        A.check(A.load().ffs_lbm_fill_solid(self._h, C.byref(s), _stream_handle(stream)), "fill_solid")

    def status(self, clear: bool = True, stream=None) -> int:
        v = C.c_uint32()
        A.check(A.load().ffs_lbm_get_status(self._h, C.byref(v), int(clear), _stream_handle(stream)), "get_status")
        return int(v.value)

    def profile(self, enable: bool = True, serial: bool = False):
        """Start/stop per-stage CUDA-event timing of the steps.  serial=True
        moves link detection off its side stream, ahead of the dense pass, so
        that each stage is timed alone (the step loses the overlap)."""
        mode = (2 if serial else 1) if enable else 0
        A.check(A.load().ffs_lbm_profile_enable(self._h, mode), "profile_enable")

    def profile_read(self, reset: bool = True) -> dict:
        """{stage: (milliseconds, launches)} summed since the last reset."""
        p = A.Profile()
        A.check(A.load().ffs_lbm_profile_read(self._h, C.byref(p), int(bool(reset))), "profile_read")
        return {name: (p.ms[i], int(p.launches[i])) for i, name in enumerate(A.PROFILE_STAGES)}

    def debug_links(self, surface: DeviceSurface, stream=None):
        s = surface.c_struct()
        n = C.c_int64()
        L = A.load()
        A.check(L.ffs_lbm_debug_links(self._h, C.byref(s), None, None, 0, C.byref(n), _stream_handle(stream)),
                "debug_links")
        cq = np.zeros(max(n.value, 1), dtype=np.uint64)
        key = np.zeros(max(n.value, 1), dtype=np.uint64)
        A.check(L.ffs_lbm_debug_links(self._h, C.byref(s), _np_ptr(cq), _np_ptr(key), n.value, C.byref(n),
                                      _stream_handle(stream)), "debug_links")
        return cq[: n.value], key[: n.value]
