"""Seeded synthetic inputs for the fluid-step configurations.

The reference ships no benchmark data, so these generators build the
configurations the benchmark and the tests run, following the shapes of the
reference's own demo scripts (``scripts/vortex_street_2d.py:54-132``,
``scripts/vortex_3d.py:25-97``, ``rl/env.py:90-128``):

  A  cylinder_channel_2d  D2Q9 256x128, fixed cylinder r=16 at (64,64)
  B  swimmer_2d           D2Q9 1200x400, travelling-wave fish outline
  C  taylor_green_3d      D3Q27 128^3 periodic Taylor-Green vortex
  D  swimmer_3d           D3Q27 384x192x192 channel, undulating ellipsoid

Node-flag values are FreeFlow's LbmNodeFlag (LbmDataTypes.cuh:17-56); boundary
cells are written in the demo scripts' order, so a later write wins at edges
and corners exactly as the reference's list of per-cell JSON entries does.
Everything is numpy; moments use the reference AoS layout.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

FLUID, SOLID, SOLID_DYNAMIC, WALL = 1, 3, 4, 5
INLET_LEFT, INLET_RIGHT, INLET_UP, INLET_DOWN, INLET_FRONT, INLET_BACK = 13, 14, 15, 16, 17, 18
OUTLET_LEFT, OUTLET_RIGHT, OUTLET_UP, OUTLET_DOWN, OUTLET_FRONT, OUTLET_BACK = 19, 20, 21, 22, 23, 24


@dataclass
class Workload:
    name: str
    dim: int
    nx: int
    ny: int
    nz: int
    fluid_viscosity: float
    fluid_density: float
    fluid_dx: float
    dt: float
    boundary_velocities: list
    flags: np.ndarray                 # (ncell,) uint8
    moments: np.ndarray               # (ncell, NM) float32, reference AoS layout
    periodic: int = 0
    elements: np.ndarray | None = None  # (ne, dim) uint32
    rest: np.ndarray | None = None      # (nv, dim) float32 rest positions (physical)
    kinematics: object = None           # t -> (vertices, velocities), physical units
    meta: dict = field(default_factory=dict)

    @property
    def ncell(self) -> int:
        return self.nx * self.ny * self.nz

    def surface_at(self, step: int):
        """Surface (vertices, velocities) at time step*dt, float32."""
        if self.kinematics is None:
            return self.rest.astype(np.float32), np.zeros_like(self.rest, dtype=np.float32)
        return self.kinematics(step * self.dt)

    def grid_kwargs(self, storage="f32", ref_half_populations=False, ref_2d_wall_stream=False):
        return dict(dim=self.dim, nx=self.nx, ny=self.ny, nz=self.nz, fluid_viscosity=self.fluid_viscosity,
                    fluid_density=self.fluid_density, fluid_dx=self.fluid_dx, dt=self.dt,
                    boundary_velocities=self.boundary_velocities, storage=storage, periodic=self.periodic,
                    ref_half_populations=ref_half_populations, ref_2d_wall_stream=ref_2d_wall_stream)


def equilibrium_moments(rho, u, dtype=np.float32):
    """Stored moments of an equilibrium state: pi_ab = u_a u_b."""
    rho = np.asarray(rho, dtype=np.float64)
    u = np.asarray(u, dtype=np.float64)
    dim = u.shape[-1]
    if dim == 2:
        ux, uy = u[..., 0], u[..., 1]
        m = np.stack([rho, ux, uy, ux * ux, uy * uy, ux * uy], axis=-1)
    else:
        ux, uy, uz = u[..., 0], u[..., 1], u[..., 2]
        m = np.stack([rho, ux, uy, uz, ux * ux, uy * uy, uz * uz, ux * uy, uy * uz, ux * uz], axis=-1)
    return m.astype(dtype)


# ------------------------------------------------------------------ config A
def channel_flags_2d(nx, ny):
    """Walls top/bottom, InletLeft, OutletRight (vortex_street_2d.py:105-117)."""
    f = np.full((ny, nx), FLUID, dtype=np.uint8)
    f[0, :] = WALL
    f[ny - 1, :] = WALL
    f[:, 0] = INLET_LEFT
    f[:, nx - 1] = OUTLET_RIGHT
    return f.reshape(-1)


def circle_polygon(cx, cy, r, nseg):
    th = 2.0 * np.pi * np.arange(nseg) / nseg
    v = np.stack([cx + r * np.cos(th), cy + r * np.sin(th)], axis=1)
    e = np.stack([np.arange(nseg), (np.arange(nseg) + 1) % nseg], axis=1)
    return v.astype(np.float32), e.astype(np.uint32)


def cylinder_channel_2d(nx=256, ny=128, radius=16.0, center=(64.0, 64.0), u_in=0.05, reynolds=100.0,
                        nseg=128, seed=0, fluid_dx=0.005, dt=0.0025, density=1000.0, perturbation=1e-3):
    """Config A: channel flow past a fixed circular cylinder (Re ~ 100)."""
    rng = np.random.default_rng(seed)
    flags = channel_flags_2d(nx, ny)
    nu = u_in * 2.0 * radius / reynolds
    # reference initializer: u = inlet velocity on inlet nodes, 0 on other
    # boundary nodes; fluid nodes start at the inlet velocity plus a seeded
    # uniform perturbation in [-perturbation, perturbation]^2
    u = np.zeros((flags.size, 2))
    fl = flags == FLUID
    u[flags == INLET_LEFT, 0] = u_in
    u[fl, 0] = u_in
    u[fl] += rng.uniform(-perturbation, perturbation, size=(int(fl.sum()), 2))
    m = equilibrium_moments(np.ones(flags.size), u)
    v, e = circle_polygon(center[0] * fluid_dx, center[1] * fluid_dx, radius * fluid_dx, nseg)
    return Workload(f"A:D2Q9 {nx}x{ny} cylinder", 2, nx, ny, 1, nu, density, fluid_dx, dt, [u_in, 0, 0, 0],
                    flags, m, 0, e, v, None, dict(seed=seed, reynolds=reynolds))


# ------------------------------------------------------------------ config B
def fish_outline(length, n_half, thickness=0.12, rng=None, jitter=0.0):
    """Closed NACA-00xx-like outline, head at x=0, body along +x (lattice units)."""
    s = 0.5 * (1.0 - np.cos(np.linspace(0.0, np.pi, n_half + 1)))  # cosine spacing head->tail
    yt = 5.0 * thickness * (0.2969 * np.sqrt(s) - 0.1260 * s - 0.3516 * s ** 2 + 0.2843 * s ** 3 - 0.1036 * s ** 4)
    top = np.stack([s, yt], axis=1)[:-1]            # head .. just before tail
    bot = np.stack([s[::-1], -yt[::-1]], axis=1)[:-1]  # tail .. just before head
    pts = np.concatenate([top, bot], axis=0) * length
    if rng is not None and jitter > 0:
        pts = pts + rng.uniform(-jitter, jitter, size=pts.shape)
    n = pts.shape[0]
    e = np.stack([np.arange(n), (np.arange(n) + 1) % n], axis=1).astype(np.uint32)
    return pts, e


def carangiform_envelope(s, length):
    """Lateral amplitude along the body, A(1) = 0.1 L."""
    return length * (0.02 - 0.0825 * s + 0.1625 * s * s)


def swimmer_2d(nx=1200, ny=400, body_frac=0.4, n_boundary=198, freq=1.0, seed=0, fluid_dx=0.005, dt=0.0025,
               density=10.0, viscosity=0.005, head=(0.25, 0.5)):
    """Config B: D2Q9 travelling-wave swimmer, outlets on all four sides."""
    rng = np.random.default_rng(seed)
    f = np.full((ny, nx), FLUID, dtype=np.uint8)
    # fish2d_lbs_control.json order: bottom/top rows, then left/right columns
    f[0, :] = OUTLET_DOWN
    f[ny - 1, :] = OUTLET_UP
    f[:, 0] = OUTLET_LEFT
    f[:, nx - 1] = OUTLET_RIGHT
    flags = f.reshape(-1)
    L = body_frac * ny
    pts, e = fish_outline(L, n_boundary // 2, rng=rng, jitter=1e-3)
    hx, hy = head[0] * nx, head[1] * ny
    X = pts[:, 0].copy()
    s = np.clip(X / L, 0.0, 1.0)
    amp = carangiform_envelope(s, L)
    k = 2.0 * np.pi / L
    om = 2.0 * np.pi * freq
    rest = np.stack([hx + pts[:, 0], hy + pts[:, 1]], axis=1) * fluid_dx

    def kin(t):
        ph = k * X - om * t
        y = hy + pts[:, 1] + amp * np.sin(ph)
        pos = np.stack([hx + pts[:, 0], y], axis=1) * fluid_dx
        vel = np.stack([np.zeros_like(X), -amp * om * np.cos(ph)], axis=1) * fluid_dx
        return pos.astype(np.float32), vel.astype(np.float32)

    m = equilibrium_moments(np.ones(flags.size), np.zeros((flags.size, 2)))
    return Workload(f"B:D2Q9 {nx}x{ny} swimmer", 2, nx, ny, 1, viscosity, density, fluid_dx, dt, [0, 0, 0, 0],
                    flags, m, 0, e, rest.astype(np.float32), kin, dict(seed=seed, body_length_cells=L))


# ------------------------------------------------------------------ config C
def taylor_green_3d(n=128, u0=0.04, viscosity=0.005, rho0=1.0):
    """Config C: periodic 3D Taylor-Green vortex, equilibrium initial state."""
    c = 2.0 * np.pi * (np.arange(n) + 0.5) / n
    z, y, x = np.meshgrid(c, c, c, indexing="ij")  # x fastest in memory
    ux = u0 * np.sin(x) * np.cos(y) * np.cos(z)
    uy = -u0 * np.cos(x) * np.sin(y) * np.cos(z)
    uz = np.zeros_like(ux)
    p = rho0 * u0 * u0 / 16.0 * (np.cos(2 * x) + np.cos(2 * y)) * (np.cos(2 * z) + 2.0)
    rho = rho0 + 3.0 * p
    u = np.stack([ux, uy, uz], axis=-1).reshape(-1, 3)
    m = equilibrium_moments(rho.reshape(-1), u)
    flags = np.full(n ** 3, FLUID, dtype=np.uint8)
    return Workload(f"C:D3Q27 {n}^3 Taylor-Green", 3, n, n, n, viscosity, 1.0, 1.0, 1.0, [0] * 6, flags, m, 7,
                    None, None, None, dict(u0=u0, k=2 * np.pi / n))


def tgv_kinetic_energy(m: np.ndarray) -> float:
    rho = m[:, 0].astype(np.float64)
    u2 = (m[:, 1:4].astype(np.float64) ** 2).sum(axis=1)
    return float(0.5 * (rho * u2).mean())


# ------------------------------------------------------------------ config D
def channel_flags_3d(nx, ny, nz):
    """vortex_3d.py:78-94: inlet on the middle of x=0, outlet at x=nx-1, walls elsewhere."""
    f = np.full((nz, ny, nx), FLUID, dtype=np.uint8)
    jj, kk = np.meshgrid(np.arange(ny), np.arange(nz), indexing="xy")
    inlet = (jj >= ny // 4) & (jj <= 3 * ny // 4) & (kk >= nz // 4) & (kk <= 3 * nz // 4)
    f[:, :, 0] = np.where(inlet, INLET_LEFT, WALL)
    f[:, :, nx - 1] = OUTLET_RIGHT
    f[:, 0, :] = WALL
    f[:, ny - 1, :] = WALL
    f[0, :, :] = WALL
    f[nz - 1, :, :] = WALL
    return f.reshape(-1)


def ellipsoid_mesh(a, b, c, nlat=64, nlon=64):
    """UV ellipsoid along x: (nlat-1)*nlon + 2 vertices, 2*nlon*(nlat-1) triangles."""
    th = np.pi * np.arange(1, nlat) / nlat
    ph = 2.0 * np.pi * np.arange(nlon) / nlon
    T, P = np.meshgrid(th, ph, indexing="ij")
    ring = np.stack([a * np.cos(T), b * np.sin(T) * np.cos(P), c * np.sin(T) * np.sin(P)], axis=-1).reshape(-1, 3)
    v = np.concatenate([[[a, 0.0, 0.0]], ring, [[-a, 0.0, 0.0]]], axis=0)
    tris = []
    top, bot = 0, v.shape[0] - 1
    idx = lambda i, j: 1 + i * nlon + (j % nlon)
    for j in range(nlon):
        tris.append([top, idx(0, j + 1), idx(0, j)])
    for i in range(nlat - 2):
        for j in range(nlon):
            a0, a1, b0, b1 = idx(i, j), idx(i, j + 1), idx(i + 1, j), idx(i + 1, j + 1)
            tris.append([a0, a1, b1])
            tris.append([a0, b1, b0])
    for j in range(nlon):
        tris.append([bot, idx(nlat - 2, j), idx(nlat - 2, j + 1)])
    return v, np.asarray(tris, dtype=np.uint32)


def swimmer_3d(nx=384, ny=192, nz=192, body_frac=0.3, freq=1.0, seed=0, fluid_dx=0.01, dt=0.005, density=500.0,
               viscosity=0.01, u_in=0.05, nlat=64, nlon=64, center=(0.35, 0.5, 0.5)):
    """Config D: D3Q27 channel with an undulating ellipsoid swimmer."""
    rng = np.random.default_rng(seed)
    flags = channel_flags_3d(nx, ny, nz)
    L = body_frac * nx
    v, e = ellipsoid_mesh(0.5 * L, 0.05 * ny, 0.05 * nz, nlat, nlon)
    v = v + rng.uniform(-1e-3, 1e-3, size=v.shape)
    cx, cy, cz = center[0] * nx, center[1] * ny, center[2] * nz
    X = v[:, 0] + 0.5 * L   # distance from the head (x = cx - L/2)
    s = np.clip(X / L, 0.0, 1.0)
    k = 2.0 * np.pi / L
    om = 2.0 * np.pi * freq
    amp = 0.08 * L * s * s
    rest = np.stack([cx + v[:, 0], cy + v[:, 1], cz + v[:, 2]], axis=1) * fluid_dx

    def kin(t):
        ph = k * X - om * t
        pos = np.stack([cx + v[:, 0], cy + v[:, 1], cz + v[:, 2] + amp * np.sin(ph)], axis=1) * fluid_dx
        vel = np.stack([np.zeros_like(X), np.zeros_like(X), -amp * om * np.cos(ph)], axis=1) * fluid_dx
        return pos.astype(np.float32), vel.astype(np.float32)

    u = np.zeros((flags.size, 3))
    u[flags == INLET_LEFT, 0] = u_in
    m = equilibrium_moments(np.ones(flags.size), u)
    return Workload(f"D:D3Q27 {nx}x{ny}x{nz} swimmer", 3, nx, ny, nz, viscosity, density, fluid_dx, dt,
                    [u_in, 0, 0, 0, 0, 0], flags, m, 0, e, rest.astype(np.float32), kin,
                    dict(seed=seed, body_length_cells=L, vertices=v.shape[0], triangles=e.shape[0]))


def small_variant(wl_fn, **kw):
    """Convenience: the same generator at a reduced size (tests)."""
    return wl_fn(**kw)
