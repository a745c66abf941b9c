"""The five benchmark configurations at their full sizes on the GPU, through
the C ABI, checked by properties that do not need the oracle to run at that
size (or, for the small config A, against the FP64 oracle itself):

  A  D2Q9 256x128 cylinder, FP32, 2000 steps: velocity and accumulated
     surface forces against the FP64 oracle (relative L2 <= 1e-3; measured
     1.8e-4 and 3.3e-4).
  B  D2Q9 1200x400 swimmer, 10k steps: FP32 and FP16 storage both stay
     healthy (status word clear), and their accumulated surface forces agree
     within 10 %.  The prescribed tail speed is about 0.25 lattice units at
     viscosity 0.005, so the flow is unsteady and fields of different
     precisions decorrelate; integral forces stay close.
  C  D3Q27 periodic Taylor-Green 128^3, 5000 steps: mass conserved to the
     rounding of FP32 (drift <= 2e-8 of the mass per step; the reference's
     FP32 weights give 7.4e-9), kinetic energy decreasing, and FP16 storage
     tracking the FP32 energy within 3 %.
  D  D3Q27 384x192x192 swimmer, 1000 steps: FP16 storage against FP32,
     velocity relative L2 <= 2e-3 (measured 5.3e-4) and accumulated forces
     <= 5e-4 (4.6e-5).
The serving mix (config E) is covered by test_gpu_serving.py.

At the end of the file, the full sizes against FP64 and the oracle: D (FP32
against the FP32 restatement, 10 steps; FP16/BF16 against FP64), C (FP32,
FP16, BF16 against FP64 after 200 steps and along 5000 steps of kinetic
energy) and B (100 steps from a developed state, FP32/FP16/BF16 against
FP64).

A long moving-wall run checks that no bias builds up over many steps: a
64x32x32 D3Q27 swimmer for 300 steps against the oracle's FP32 restatement
(velocity and accumulated forces within 1e-4 relative; at 96x48x48 and 500
steps the difference measured 9e-6 and 3e-6).
"""
import os

import numpy as np
import pytest

from freeflow_b200 import workloads as W

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(b))


def gpu_run(wl, steps, storage="f32", checkpoints=()):
    from freeflow_b200 import DeviceSurface, FluidGrid

    g = FluidGrid(**wl.grid_kwargs(storage=storage))
    g.set_flags(wl.flags)
    g.set_moments(wl.moments)
    surf = None
    if wl.elements is not None:
        v, u = wl.surface_at(0)
        surf = DeviceSurface(v, u, wl.elements, with_forces64=True)
    saved = []
    for s in range(steps):
        if surf is not None:
            if wl.kinematics is not None or s == 0:
                surf.update(*wl.surface_at(s))
            g.step(surf)
        else:
            g.step()
        if s + 1 in checkpoints:
            saved.append(g.get_moments().astype(np.float64))
    m = g.get_moments().astype(np.float64)
    st = g.status()
    F = surf.forces64.cpu().numpy().reshape(-1) if surf is not None else None
    g.close()
    return m, st, F, saved


def test_config_a_cylinder_2000_steps_vs_fp64(cuda):
    from oracle import oracle as O

    wl = W.cylinder_channel_2d()
    gm, st, gF, _ = gpu_run(wl, 2000)
    assert st == 0
    O.set_threads(os.cpu_count() or 1)
    o = O.Oracle(2, wl.nx, wl.ny, 1, viscosity=wl.fluid_viscosity, density=wl.fluid_density, dx=wl.fluid_dx,
                 dt=wl.dt, boundary_velocities=wl.boundary_velocities, periodic=wl.periodic, precision="phys64")
    o.set_flags(wl.flags)
    o.set_moments(wl.moments.astype(np.float64))
    F = np.zeros(wl.rest.size)
    v, u = wl.surface_at(0)
    for _ in range(2000):
        o.step(v, u, wl.elements, F)
    om = o.get_moments()
    o.close()
    assert rel(gm[:, 1:3], om[:, 1:3]) <= 1e-3
    assert rel(gF, F) <= 1e-3


def test_config_b_swimmer_10k_steps_fp32_and_fp16(cuda):
    wl = W.swimmer_2d()
    _, s32, F32, _ = gpu_run(wl, 10000, "f32")
    _, s16, F16, _ = gpu_run(wl, 10000, "f16")
    assert s32 == 0 and s16 == 0
    assert np.isfinite(F32).all() and np.isfinite(F16).all()
    assert rel(F16, F32) <= 0.1


def test_config_c_taylor_green_128_cubed_5000_steps(cuda):
    wl = W.taylor_green_3d(n=128, u0=0.04, viscosity=0.005)
    m0 = wl.moments.astype(np.float64)
    mass0 = m0[:, 0].sum()
    ke = lambda m: 0.5 * np.sum(m[:, 0] * np.sum(m[:, 1:4] ** 2, axis=1))
    marks = (1000, 2000, 3000, 4000, 5000)
    energies = {}
    for storage in ("f32", "f16"):
        _, st, _, saved = gpu_run(wl, 5000, storage, checkpoints=marks)
        assert st == 0
        drift = [(m[:, 0].sum() - mass0) / mass0 / t for m, t in zip(saved, marks)]
        assert max(abs(d) for d in drift) <= 2e-8, drift
        e = [ke(m) for m in saved]
        assert all(b < a for a, b in zip([ke(m0)] + e[:-1], e))
        energies[storage] = np.array(e)
    assert np.abs(energies["f16"] / energies["f32"] - 1.0).max() <= 0.03


def test_config_d_swimmer_fp16_vs_fp32_1000_steps(cuda):
    wl = W.swimmer_3d()
    m32, s32, F32, _ = gpu_run(wl, 1000, "f32")
    m16, s16, F16, _ = gpu_run(wl, 1000, "f16")
    assert s32 == 0 and s16 == 0
    assert rel(m16[:, 1:4], m32[:, 1:4]) <= 2e-3
    assert rel(F16, F32) <= 5e-4


def test_d3q27_swimmer_300_steps_vs_oracle(cuda):
    from oracle import oracle as O

    wl = W.swimmer_3d(nx=64, ny=32, nz=32, body_frac=0.4, nlat=16, nlon=24, seed=4)
    gm, st, gF, _ = gpu_run(wl, 300)
    assert st == 0
    O.set_threads(os.cpu_count() or 1)
    o = O.Oracle(3, wl.nx, wl.ny, wl.nz, viscosity=wl.fluid_viscosity, density=wl.fluid_density, dx=wl.fluid_dx,
                 dt=wl.dt, boundary_velocities=wl.boundary_velocities, periodic=wl.periodic, precision="ref32")
    o.set_flags(wl.flags)
    o.set_moments(wl.moments.astype(np.float64))
    F = np.zeros(wl.rest.size)
    for s in range(300):
        v, u = wl.surface_at(s)
        o.step(v, u, wl.elements, F)
    om = o.get_moments()
    o.close()
    assert rel(gm[:, 1:4], om[:, 1:4]) <= 1e-4
    assert rel(gF, F) <= 1e-4


# ------------------------------------------------ full sizes against FP64
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "tgv128_fp64.npz")


def test_config_d_full_size_vs_oracle(cuda):
    """Config D at its full size (384 x 192 x 192, the undulating 4034-vertex
    ellipsoid), 10 steps, against the oracle's FP32 restatement of the
    reference: moments max |diff| <= 4e-6 (measured 1.3e-6), accumulated
    surface forces <= 2e-4 x max |F| (the oracle's double sums against the
    product's fixed-point ones)."""
    from oracle import oracle as O

    wl = W.swimmer_3d()
    gm, st, gF, _ = gpu_run(wl, 10)
    assert st == 0
    O.set_threads(os.cpu_count() or 1)
    o = O.Oracle(3, wl.nx, wl.ny, wl.nz, viscosity=wl.fluid_viscosity, density=wl.fluid_density, dx=wl.fluid_dx,
                 dt=wl.dt, boundary_velocities=wl.boundary_velocities, periodic=wl.periodic, precision="ref32")
    o.set_flags(wl.flags)
    o.set_moments(wl.moments.astype(np.float64))
    F = np.zeros(wl.rest.size)
    for s in range(10):
        v, u = wl.surface_at(s)
        o.step(v, u, wl.elements, F)
    om = o.get_moments()
    o.close()
    assert float(np.abs(gm - om).max()) <= 4e-6
    assert float(np.abs(gF - F).max()) <= 2e-4 * float(np.abs(F).max())


def test_config_d_reduced_storage_vs_fp64(cuda):
    """Config D, 10 steps from the initial state, FP16 and BF16 storage against
    the FP64 oracle: relative L2 of u <= 1e-3 (FP16, measured 3.7e-4) and
    2e-3 (BF16, 7.3e-4); FP32 for scale (1.4e-6)."""
    from oracle import oracle as O

    wl = W.swimmer_3d()
    O.set_threads(os.cpu_count() or 1)
    o = O.Oracle(3, wl.nx, wl.ny, wl.nz, viscosity=wl.fluid_viscosity, density=wl.fluid_density, dx=wl.fluid_dx,
                 dt=wl.dt, boundary_velocities=wl.boundary_velocities, periodic=wl.periodic, precision="phys64")
    o.set_flags(wl.flags)
    o.set_moments(wl.moments.astype(np.float64))
    F = np.zeros(wl.rest.size)
    for s in range(10):
        v, u = wl.surface_at(s)
        o.step(v, u, wl.elements, F)
    ref = o.get_moments()[:, 1:4]
    o.close()
    for storage, tol in (("f32", 2e-5), ("f16", 1e-3), ("bf16", 2e-3)):
        m, st, gF, _ = gpu_run(wl, 10, storage)
        assert st == 0
        assert rel(m[:, 1:4], ref) <= tol, storage
        assert rel(gF, F) <= 10 * tol, storage


def test_config_c_full_size_vs_fp64(cuda):
    """Config C itself (128^3 periodic Taylor-Green, u0 0.04, viscosity 0.005)
    in FP32, FP16 and BF16 storage against FP64:
      * after 200 steps, relative L2 of u against the FP64 oracle run here;
      * the kinetic energy every 50 steps up to 5000, and u at an 8-cell
        lattice of 4096 cells after 1000 and 5000 steps, against the FP64
        oracle's run of the same 5000 steps (tests/golden/tgv128_fp64.npz,
        made by tests/golden/make_tgv128_fp64.py);
      * the early decay against the analytic viscous rate exp(-6 nu k^2 t)
        (k = 2 pi / 128); later the vortex decays faster through its own
        nonlinearity, as the FP64 run shows."""
    from oracle import oracle as O

    golden = np.load(GOLDEN)
    wl = W.taylor_green_3d(n=128, u0=0.04, viscosity=0.005)
    O.set_threads(os.cpu_count() or 1)
    o = O.Oracle(3, 128, 128, 128, viscosity=wl.fluid_viscosity, density=1.0, dx=1.0, dt=1.0,
                 boundary_velocities=[0] * 6, periodic=7, precision="phys64")
    o.set_flags(wl.flags)
    o.set_moments(wl.moments.astype(np.float64))
    for _ in range(200):
        o.step()
    u200 = o.get_moments()[:, 1:4]
    o.close()
    ke64 = golden["ke"]
    idx = golden["sample_idx"]
    e0 = ke64[0]
    kk = 2.0 * np.pi / 128
    tols = {"f32": (2e-5, 1e-3, 5e-3), "f16": (1e-3, 3e-2, 5e-2), "bf16": (2e-3, 3e-2, 5e-2)}
    ke = {}
    for storage, (tol200, tol_ke, tol_u) in tols.items():
        from freeflow_b200 import FluidGrid

        g = FluidGrid(**wl.grid_kwargs(storage=storage))
        g.set_flags(wl.flags)
        g.set_moments(wl.moments)
        curve = [W.tgv_kinetic_energy(wl.moments.astype(np.float64))]
        for s in range(1, 5001):
            g.step()
            if s % 50 == 0 or s == 200:
                m = g.get_moments().astype(np.float64)
                if s == 200:
                    assert rel(m[:, 1:4], u200) <= tol200, (storage, rel(m[:, 1:4], u200))
                if s % 50 == 0:
                    curve.append(W.tgv_kinetic_energy(m))
                if s in (1000, 5000):
                    ref = golden[f"u_{s}"]
                    assert rel(m[idx, 1:4], ref) <= tol_u, (storage, s, rel(m[idx, 1:4], ref))
        assert g.status() == 0
        g.close()
        curve = np.array(curve)
        ke[storage] = curve
        assert np.abs(curve / ke64 - 1.0).max() <= tol_ke, storage
        t = golden["ke_steps"]
        early = t <= 200
        assert np.abs(curve[early] / (e0 * np.exp(-6 * wl.fluid_viscosity * kk * kk * t[early])) - 1.0).max() <= 5e-3
    # BF16 keeps decaying with FP32 (its velocity is stored in binary16)
    assert np.abs(ke["bf16"] / ke["f32"] - 1.0).max() <= 0.03


def test_config_b_from_developed_state_vs_fp64(cuda):
    """Config B (1200 x 400 swimmer): the FP32 state after 2000 steps, then 100
    steps from that identical state in FP32, FP16 and BF16 storage against the
    FP64 oracle fed the same surfaces: relative L2 of u <= 2e-5 (FP32,
    measured 4.4e-6), 1e-3 (FP16, 6.9e-4), 3e-3 (BF16, 1.6e-3)."""
    from oracle import oracle as O

    wl = W.swimmer_2d()
    from freeflow_b200 import DeviceSurface, FluidGrid

    g = FluidGrid(**wl.grid_kwargs())
    g.set_flags(wl.flags)
    g.set_moments(wl.moments)
    v, u = wl.surface_at(0)
    surf = DeviceSurface(v, u, wl.elements)
    for s in range(2000):
        surf.update(*wl.surface_at(s))
        g.step(surf)
    state = g.get_moments().astype(np.float32)
    assert g.status() == 0
    g.close()
    O.set_threads(os.cpu_count() or 1)
    o = O.Oracle(2, wl.nx, wl.ny, 1, viscosity=wl.fluid_viscosity, density=wl.fluid_density, dx=wl.fluid_dx,
                 dt=wl.dt, boundary_velocities=wl.boundary_velocities, periodic=wl.periodic, precision="phys64")
    o.set_flags(wl.flags)
    o.set_moments(state.astype(np.float64))
    F = np.zeros(wl.rest.size)
    for s in range(2000, 2100):
        v, u = wl.surface_at(s)
        o.step(v, u, wl.elements, F)
    ref = o.get_moments()[:, 1:3]
    o.close()
    for storage, tol in (("f32", 2e-5), ("f16", 1e-3), ("bf16", 3e-3)):
        g = FluidGrid(**wl.grid_kwargs(storage=storage))
        g.set_flags(wl.flags)
        g.set_moments(state)
        v, u = wl.surface_at(2000)
        sf = DeviceSurface(v, u, wl.elements, with_forces64=True)
        for s in range(2000, 2100):
            sf.update(*wl.surface_at(s))
            g.step(sf)
        m = g.get_moments().astype(np.float64)
        assert g.status() == 0
        assert rel(m[:, 1:3], ref) <= tol, (storage, rel(m[:, 1:3], ref))
        assert rel(sf.forces64.cpu().numpy().reshape(-1), F) <= 10 * tol, storage
        g.close()
