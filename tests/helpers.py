"""Shared drivers for the GPU parity tests: run the CUDA path (through the
C ABI) and the CPU oracle side by side on identical seeded inputs."""
from __future__ import annotations

import numpy as np

from freeflow_b200 import workloads as W


def make_gpu(wl: W.Workload, storage="f32", ref_half=False, periodic=None, wall_stream=False):
    from freeflow_b200 import DeviceSurface, FluidGrid

    kw = wl.grid_kwargs(storage=storage, ref_half_populations=ref_half, ref_2d_wall_stream=wall_stream)
    if periodic is not None:
        kw["periodic"] = periodic
    g = FluidGrid(**kw)
    g.set_flags(wl.flags)
    g.set_moments(wl.moments)
    surf = None
    if wl.elements is not None:
        v, u = wl.surface_at(0)
        surf = DeviceSurface(v, u, wl.elements, with_forces64=True)
    return g, surf


def make_oracle(wl: W.Workload, precision="ref32", half_pops=False, periodic=None, wall_stream=False):
    from oracle.oracle import Oracle

    o = Oracle(wl.dim, wl.nx, wl.ny, wl.nz, viscosity=wl.fluid_viscosity, density=wl.fluid_density,
               dx=wl.fluid_dx, dt=wl.dt, boundary_velocities=wl.boundary_velocities,
               periodic=wl.periodic if periodic is None else periodic, half_pops=half_pops, precision=precision,
               wall_stream=wall_stream)
    o.set_flags(wl.flags)
    o.set_moments(wl.moments.astype(np.float64))
    return o


def run_pair(wl: W.Workload, steps: int, storage="f32", ref_half=False, precision="ref32", periodic=None):
    """Advance GPU and oracle `steps` steps with the workload's kinematics.
    Returns (gpu_moments, oracle_moments, gpu_forces64, oracle_forces, status)."""
    import torch

    g, surf = make_gpu(wl, storage, ref_half, periodic)
    o = make_oracle(wl, precision, ref_half, periodic)
    of = None
    if wl.elements is not None:
        of = np.zeros(wl.rest.size, dtype=np.float64)
    for s in range(steps):
        if wl.elements is not None:
            v, u = wl.surface_at(s)
            surf.update(v, u)
            g.step(surf)
            o.step(v, u, wl.elements, of)
        else:
            g.step()
            o.step()
    torch.cuda.synchronize()
    gm = g.get_moments().astype(np.float64)
    om = o.get_moments()
    gf = surf.forces64.cpu().numpy().reshape(-1) if surf is not None else None
    st = g.status()
    g.close()
    o.close()
    return gm, om, gf, of, st


def max_abs(a, b):
    return float(np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64)).max())


def rms(a, b):
    d = np.asarray(a, np.float64) - np.asarray(b, np.float64)
    return float(np.sqrt((d * d).mean()))
