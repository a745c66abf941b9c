"""Generates tgv128_fp64.npz: the FP64 oracle's run of the D3Q27 periodic
Taylor-Green vortex of config C (128^3, peak velocity 0.04, viscosity 0.005,
equilibrium start) for 5000 steps.

Stored (float64):
  ke_steps, ke     kinetic energy 0.5 <rho |u|^2> every 50 steps (0..5000)
  sample_idx       cell indices of an 8-cell-spaced sample lattice (16^3 cells)
  u_200, u_1000, u_5000   velocity at those cells after 200, 1000, 5000 steps

The GPU tests compare their own runs of the same workload against these.
Run from the repository root (about 12 minutes on 8 host cores):
    python tests/golden/make_tgv128_fp64.py
"""
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from freeflow_b200 import workloads as W  # noqa: E402
from oracle import oracle as O  # noqa: E402

N, STEPS, EVERY = 128, 5000, 50
SNAP = (200, 1000, 5000)


def sample_indices(n=N, stride=8):
    c = np.arange(stride // 2, n, stride)
    z, y, x = np.meshgrid(c, c, c, indexing="ij")
    return ((z * n + y) * n + x).reshape(-1)


def main():
    subprocess_make = os.path.join(ROOT, "oracle")
    os.system(f"make -s -C {subprocess_make}")
    O.set_threads(os.cpu_count() or 1)
    wl = W.taylor_green_3d(n=N, u0=0.04, viscosity=0.005)
    o = O.Oracle(3, N, N, N, viscosity=wl.fluid_viscosity, density=wl.fluid_density, dx=wl.fluid_dx, dt=wl.dt,
                 boundary_velocities=wl.boundary_velocities, periodic=wl.periodic, precision="phys64")
    o.set_flags(wl.flags)
    o.set_moments(wl.moments.astype(np.float64))
    idx = sample_indices()
    ke_steps, ke, snaps = [0], [W.tgv_kinetic_energy(wl.moments.astype(np.float64))], {}
    t0 = time.time()
    for s in range(1, STEPS + 1):
        o.step()
        if s % EVERY == 0 or s in SNAP:
            m = o.get_moments()
            if s % EVERY == 0:
                ke_steps.append(s)
                ke.append(W.tgv_kinetic_energy(m))
            if s in SNAP:
                snaps[f"u_{s}"] = m[idx, 1:4].copy()
            print(f"step {s} ke {ke[-1]:.9e} ({time.time() - t0:.0f} s)", flush=True)
    o.close()
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tgv128_fp64.npz")
    np.savez_compressed(out, ke_steps=np.array(ke_steps), ke=np.array(ke), sample_idx=idx, **snaps)
    print("wrote", out)


if __name__ == "__main__":
    main()
