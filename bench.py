"""Benchmark of the moment-encoded LBM fluid step on B200.

Default workload (one GPU): D3Q27 384x192x192 channel with an undulating
ellipsoid swimmer (~4k vertices, 8k triangles), FP32 moment storage: one
step = link detection + fused stream/reconstruct/collide/re-encode pass +
moving-wall links with surface forces + outlet update.  Metric: MLUPS
(million lattice-cell updates per second, whole job), with the dense kernel's
fraction of the measured HBM peak.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload D|C|B|A] [--storage f32|f16|bf16] [--small]

N > 1 runs one independent replica per GPU (one grid per GPU: the grid is not
sharded, so there is no exchange step), one process per GPU: started by
torchrun, or by bench.py itself when no launcher set WORLD_SIZE; the time is
the max over ranks and value = all cells updated / that time ("weak").
``--check-ranks`` only joins the ranks over gloo (no GPU work) and prints
what every rank saw, a check of the launch.

``--impl reference`` times the reference's algorithm on the host cores: the
FP32 restatement in oracle/ (the reference's CUDA sources do not build here)
with all host threads, each step a z-slab sample of the same workload.

The default line (N = 1) also carries:
  storage                 config D with FP16 and BF16 moment storage (GPU);
  coupled_step            config D stepped through ffs_lbm_step_coupled
                          (surface gathered from a volume mesh, forces
                          scattered back, one stream) against the same stages
                          with the reference's two host synchronisations (GPU);
  serving                 config E, the batched FP16 pool against the plain
                          per-episode FP32 path (GPU);
  cpu_baseline and        the CPU leg, the only part of the GPU arm that runs
  storage_errors_vs_fp64  the oracle: its FP32 restatement timed on the host
                          cores, and its FP64 build as the checker of the
                          reduced-storage GPU results (skipped with
                          --no-cpu-baseline).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from freeflow_b200 import workloads as W  # noqa: E402

PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0

# DRAM bytes (read + write) per cell of the dense kernel from one ncu capture
# (dram__bytes_read.sum + dram__bytes_write.sum), scaled to a launch by the
# cells it processes; the capture and its command are in the named profile.
DENSE_TRAFFIC_PER_CELL = {
    (3, "f32"): (75.20, "profiles/dense3d_link_kernels_D3Q27_256x128x128_swimmer_f32.md"),
    (3, "f16"): (35.98, "profiles/dense3d_D3Q27_256x128x128_swimmer_f16.md"),
}


def algorithmic_bytes_per_cell(dim: int, storage: str) -> int:
    """2 * NM * s + 1: read and write NM moments of s bytes, read one flag byte."""
    nm = 6 if dim == 2 else 10
    s = 4 if storage == "f32" else 2
    return 2 * nm * s + 1


def run_config(wl, storage: str, world: int) -> dict:
    """The `config` object of both arms' JSON lines (the same dict, so the two
    lines name the same workload)."""
    bpc = algorithmic_bytes_per_cell(wl.dim, storage)
    small = wl.ncell * bpc <= 2 * 126e6   # one moment buffer can sit in the 126 MB L2
    surface = None
    if wl.elements is not None:
        surface = f"{wl.rest.shape[0]} vertices / {wl.elements.shape[0]} elements"
    return {"workload": wl.name, "cells": wl.ncell, "storage": storage, "surface": surface,
            "l2": ("moment buffers exceed L2 (no flush needed)" if not small
                   else "L2 flushed before every step (256 MB write outside the timed spans)"),
            "parallelism": f"replicas x{world}"}


def make_workload(name: str, small: bool):
    if name == "D":
        return W.swimmer_3d(nx=256, ny=128, nz=128) if small else W.swimmer_3d()
    if name == "C":
        return W.taylor_green_3d(n=96 if small else 128)
    if name == "B":
        return W.swimmer_2d(nx=600, ny=200) if small else W.swimmer_2d()
    if name == "A":
        return W.cylinder_channel_2d()
    raise ValueError(name)


def hbm_peak():
    try:
        with open(PEAKS_FILE) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """SM clock and clock-event (throttle) samples while the timed region runs.

    Polls NVML every 2 ms from a thread (reads only; no setting is changed), so
    that timed regions of a fraction of a second still get tens of samples;
    falls back to ``nvidia-smi -lms 100`` when NVML is not importable."""

    REASONS = (("hw_slowdown", 0x8), ("sw_thermal_slowdown", 0x20), ("hw_thermal_slowdown", 0x40),
               ("sw_power_cap", 0x4), ("hw_power_brake_slowdown", 0x80))
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, cuda_index: int):
        self.cuda_index = cuda_index
        self.sm, self.mask = [], 0
        self.smax = None
        self.proc = None
        self.lines = []
        self._stop = threading.Event()
        self._t = None
        self._nvml = None

    def _handle(self):
        import pynvml
        import torch

        pynvml.nvmlInit()
        try:
            uuid = str(torch.cuda.get_device_properties(self.cuda_index).uuid)
            return pynvml, pynvml.nvmlDeviceGetHandleByUUID("GPU-" + uuid)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.cuda_index)

    def _poll(self, nv, h):
        while not self._stop.is_set():
            try:
                self.sm.append(float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)))
                self.mask |= int(nv.nvmlDeviceGetCurrentClocksEventReasons(h))
            except Exception:
                pass
            self._stop.wait(0.002)

    def start(self):
        try:
            nv, h = self._handle()
            self.smax = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self._nvml = nv
            self._t = threading.Thread(target=self._poll, args=(nv, h), daemon=True)
            self._t.start()
            return
        except Exception:
            self._nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.cuda_index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self._nvml is not None:
            self._stop.set()
            self._t.join(timeout=2)
            reasons = sorted(n for n, bit in self.REASONS if self.mask & bit)
            return {"sm_mhz": statistics.median(self.sm) if self.sm else None, "sm_max_mhz": self.smax,
                    "reasons": reasons, "samples": len(self.sm), "source": "nvml 2 ms"}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clock sampling unavailable"], "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self._t:
            self._t.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvidia-smi 100 ms"}


# ------------------------------------------------------------ CPU (oracle)
def oracle_slab_run(wl: W.Workload, steps: int, warmup: int, nz_slab: int, threads: int, precision="ref32"):
    """Time the oracle on a z-slab of the workload (3D) or the whole grid (2D).
    Returns (MLUPS, cells per step, seconds)."""
    from oracle import oracle as O

    O.set_threads(threads)
    if wl.dim == 3:
        nz_slab = max(3, min(nz_slab, wl.nz))
        z0 = max(0, wl.nz // 2 - nz_slab // 2)
        nxy = wl.nx * wl.ny
        flags = wl.flags[z0 * nxy:(z0 + nz_slab) * nxy]
        mom = wl.moments[z0 * nxy:(z0 + nz_slab) * nxy]
        shift = np.array([0.0, 0.0, z0 * wl.fluid_dx], dtype=np.float32)
        nz = nz_slab
    else:
        flags, mom, shift, nz = wl.flags, wl.moments, None, 1
    o = O.Oracle(wl.dim, wl.nx, wl.ny, nz, viscosity=wl.fluid_viscosity, density=wl.fluid_density,
                 dx=wl.fluid_dx, dt=wl.dt, boundary_velocities=wl.boundary_velocities, periodic=wl.periodic,
                 precision=precision)
    o.set_flags(flags)
    o.set_moments(mom.astype(np.float64))
    F = np.zeros(wl.rest.size, dtype=np.float64) if wl.elements is not None else None

    def one(s):
        if wl.elements is None:
            o.step()
            return
        v, u = wl.surface_at(s)
        if shift is not None:
            v = v - shift
        o.step(v, u, wl.elements, F)

    for s in range(warmup):
        one(s)
    t0 = time.perf_counter()
    for s in range(steps):
        one(warmup + s)
    dt = time.perf_counter() - t0
    cells = wl.nx * wl.ny * nz
    return cells * steps / dt / 1e6, cells, dt


def serving_velocity_error(storage: str, control_steps: int = 20, sides: str = "walls"):
    """Relative L2 velocity error of a pool episode (256x128 swimmer) against
    the FP64 oracle run on the same surfaces, after `control_steps` x 10 substeps."""
    from freeflow_b200 import serving as S
    from oracle.oracle import Oracle

    sp = S.make_episode(256, 128, seed=51, length=control_steps, sides=sides)
    pool = S.Pool(storage=storage, budget_bytes=256 << 20, max_episodes=2)
    slot = pool.admit(sp)
    o = Oracle(2, sp.nx, sp.ny, 1, viscosity=sp.viscosity, density=sp.density, dx=sp.dx, dt=sp.dt,
               boundary_velocities=[0, 0, 0, 0], periodic=0, precision="phys64")
    o.set_flags(sp.flags)
    o.set_moments(pool.get_moments(slot).astype(np.float64))
    q = 0
    for c in range(control_steps):
        a = np.random.default_rng(c).uniform(-1, 1, 8).astype(np.float32)
        pool.set_action(slot, a)
        pool.advance()
        for _ in range(pool.substeps):
            V, U = S.swimmer_surface(sp, a, q)
            o.step(V, U, sp.elements, None)
            q += 1
    g = pool.get_moments(slot).astype(np.float64)
    ref = o.get_moments()
    err = float(np.linalg.norm(g[:, 1:3] - ref[:, 1:3]) / np.linalg.norm(ref[:, 1:3]))
    o.close()
    pool.close()
    return err


def tgv_velocity_errors(storages=("f32", "f16", "bf16"), n: int = 48, steps: int = 100):
    """Relative L2 velocity error of a D3Q27 periodic Taylor-Green vortex (n^3,
    peak velocity 0.04, viscosity 0.005) after `steps` steps on the GPU with
    each moment storage, against one run of the oracle's FP64 build."""
    from freeflow_b200 import FluidGrid
    from oracle.oracle import Oracle

    wl = W.taylor_green_3d(n=n, u0=0.04, viscosity=0.005)
    o = Oracle(3, n, n, n, viscosity=wl.fluid_viscosity, density=wl.fluid_density, dx=wl.fluid_dx, dt=wl.dt,
               boundary_velocities=wl.boundary_velocities, periodic=wl.periodic, precision="phys64")
    o.set_flags(wl.flags)
    o.set_moments(wl.moments.astype(np.float64))
    for _ in range(steps):
        o.step()
    ref = o.get_moments()[:, 1:4]
    o.close()
    out = {}
    for st in storages:
        g = FluidGrid(**wl.grid_kwargs(storage=st))
        g.set_flags(wl.flags)
        g.set_moments(wl.moments)
        for _ in range(steps):
            g.step()
        got = g.get_moments().astype(np.float64)[:, 1:4]
        g.close()
        out[st] = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
    return out


def cpu_leg(wl: W.Workload, threads: int):
    """The CPU leg of the GPU arm, the one place where this arm runs the oracle:
    the oracle's FP64 build timed on the host cores at all threads and at one
    (the CPU baseline: an FP64 run of the same update), its FP32 restatement
    beside it, each on a z-slab sample of the workload sized to about 10-20 s
    of CPU work; and the FP64 build as the checker of the reduced-storage GPU
    outputs.  Returns (cpu_baseline, errors against FP64)."""
    def slab(seconds, rate):
        return int(seconds * rate / 3 / (wl.nx * wl.ny)) if wl.dim == 3 else 1

    rate_all = 2.0e6 * threads          # cell updates / s of the oracle, measured order
    mlups64, cells64, sec64 = oracle_slab_run(wl, 3, 1, slab(15.0, rate_all), threads, precision="phys64")
    mlups32, cells32, sec32 = oracle_slab_run(wl, 3, 1, slab(15.0, rate_all), threads, precision="ref32")
    mlups1, cells1, sec1 = oracle_slab_run(wl, 3, 1, slab(10.0, 2.0e6), 1, precision="phys64")
    nxy = wl.nx * wl.ny

    def sample(cells, sec, what):
        return ((f"3 steps of a {cells // nxy}-plane z-slab of {wl.name}" if wl.dim == 3 else f"3 steps of {wl.name}")
                + f", {what}, {sec:.1f} s")

    cpu = {"value": round(mlups64, 3), "unit": "MLUPS", "cores": threads, "kind": "port",
           "sample": sample(cells64, sec64, "FP64 oracle"),
           "fp64_1_thread": {"value": round(mlups1, 3), "cores": 1, "sample": sample(cells1, sec1, "FP64 oracle")},
           "fp32_all_threads": {"value": round(mlups32, 3), "cores": threads,
                                "sample": sample(cells32, sec32, "FP32 restatement of the reference's arithmetic")}}
    errors = {
        "serving_2d": {
            "closed_tank": {"f16": serving_velocity_error("f16"), "f32": serving_velocity_error("f32")},
            "outlets": {"f16": serving_velocity_error("f16", sides="outlets"),
                        "f32": serving_velocity_error("f32", sides="outlets")},
            "case": "pool episode, 256x128 swimmer, 200 substeps, same surfaces as the FP64 oracle; with outlets "
                    "the reference's sign-switched outlet rule makes even FP32 differ from FP64 (branch flips)"},
        "taylor_green_3d": tgv_velocity_errors(n=128, steps=200),
        "taylor_green_3d_case": "config C itself: D3Q27 periodic 128^3, u0 0.04, viscosity 0.005, 200 steps, "
                                "relative L2 of u against the FP64 oracle",
        "target": "f16 relative velocity error <= 1e-3",
    }
    return cpu, errors


def run_reference(args):
    from freeflow_b200 import replicas as R

    rank, _, _ = R.env_ranks()
    if rank != 0:  # the CPU reference arm runs once, on rank 0; other ranks exit without work
        return 0
    wl = make_workload(args.workload, args.small)
    threads = os.cpu_count() or 1
    # size the slab so that the whole (K + W)-step run stays near two minutes
    rate = 4.0e6 * threads / 8.0  # cell updates / s, measured order of the oracle
    budget_s = 120.0
    nz_slab = int(budget_s * rate / max(1, args.steps + args.warmup) / (wl.nx * wl.ny))
    mlups, cells, sec = oracle_slab_run(wl, args.steps, args.warmup, nz_slab, threads)
    sample = (f"{'z-slab ' + str(cells // (wl.nx * wl.ny)) + ' of ' + str(wl.nz) + ' planes' if wl.dim == 3 else 'full grid'}"
              f" of {wl.name} ({cells} cells per step), {args.steps} steps")
    out = {
        "metric": "MLUPS", "value": round(mlups, 3), "unit": "MLUPS", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(1e3 * sec / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
        "impl": "reference",
        "config": run_config(wl, "f32", args.gpus),
        "cpu_baseline": {"value": round(mlups, 3), "unit": "MLUPS", "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": round(mlups, 3), "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)
    return 0



# ---------------------------------------------------------------- serving
def run_serving(iterations: int, warmup: int, concurrencies=(64, 256, 512), plain_steps: int = 20,
                plain_seconds: float = 1.0, seed: int = 0, pipelined_at=(256,)):
    """Config E: Poisson stream of 2D swimmer episodes (grids uniform over
    256x128, 512x192, 1200x400; 8 actions per control step; 10 substeps per
    action; lengths uniform in 200..2000 control steps) through the FP16 pool
    with continuous batching, at each mean concurrency, against the plain
    per-episode FP32 path (one episode of each grid size at a time, at least
    `plain_seconds` of control steps each).  At the concurrencies in
    `pipelined_at` the same stream also runs through serve_pipelined (two
    pools stepping in turn); its iterations each serve one of the two groups,
    so it runs twice the iterations for the same number of control steps."""
    import torch
    from freeflow_b200 import serving as S

    t0 = time.perf_counter()
    peak, peak_kind = hbm_peak()
    sample = [S.make_episode(nx, ny, seed=1000 + i, length=plain_steps) for i, (nx, ny) in enumerate(S.SERVING_SIZES)]
    plain = S.plain_rate(sample, plain_steps, min_seconds=plain_seconds)
    by_c = {}
    for concurrency in concurrencies:
        mean_len = 1100.0
        per_iter = concurrency / mean_len
        n_specs = concurrency + int(per_iter * (iterations + warmup) * 1.5) + 16
        specs = S.serving_mix(n_specs, seed=seed)
        max_episodes = min(1000, 2 * concurrency)   # the pool holds at most 1000 episodes
        pool = S.Pool(storage="f16", budget_bytes=6 << 30, max_episodes=max_episodes, substeps=10, num_actions=8)
        r = S.serve(pool, specs, iterations=iterations, initial=concurrency, arrivals_per_iter=per_iter, seed=seed,
                    warmup_iterations=warmup)
        info = r.pop("pool_info_at_end")
        pool.close()
        torch.cuda.synchronize()
        dense_gbs = info["tuned_cells"] * 25 / (info["dense_ms"] * 1e-3) / 1e9 if info["dense_ms"] > 0 else None
        piped = None
        if concurrency in pipelined_at:
            # the same request stream over two pools stepping in turn: host
            # work on one group overlaps the GPU step of the other
            pools = [S.Pool(storage="f16", budget_bytes=3 << 30, max_episodes=min(1000, concurrency), substeps=10,
                            num_actions=8) for _ in range(2)]
            rp = S.serve_pipelined(pools, specs, iterations=2 * iterations, initial=concurrency,
                                   arrivals_per_iter=per_iter, seed=seed, warmup_iterations=2 * warmup)
            for pl in pools:
                pl.close()
            torch.cuda.synchronize()
            piped = {k: (round(v, 3) if isinstance(v, float) else v) for k, v in rp.items()}
            piped["speedup_vs_plain"] = round(rp["env_steps_per_s"] / plain["env_steps_per_s"], 2)
        by_c[str(concurrency)] = {
            "batched": {k: (round(v, 3) if isinstance(v, float) else v) for k, v in r.items()},
            "pipelined_two_pools": piped,
            "speedup_vs_plain": round(r["env_steps_per_s"] / plain["env_steps_per_s"], 2),
            "pool": {"tile": f"{info['tile_x']}x{info['tile_y']}" + (" strip" if info["strip"] else ""),
                     "graph_builds": info["graph_builds"], "max_episodes": max_episodes,
                     "dense_ms_at_tuning": round(info["dense_ms"], 4), "cells_at_tuning": info["tuned_cells"],
                     "dense_roofline": ({"achieved": round(dense_gbs, 1), "peak": peak, "unit": "GB/s",
                                         "frac": round(dense_gbs / peak, 4), "bytes_per_cell": 25,
                                         "peak_kind": peak_kind} if dense_gbs else None)},
        }
    return {
        "workload": "E: D2Q9 swimmer mix {256x128, 512x192, 1200x400}, 198-edge fish, 8 actions x 10 substeps",
        "storage": "f16",
        "by_concurrency": by_c,
        "plain_f32": {k: (round(v, 3) if isinstance(v, float) else v) for k, v in plain.items()},
        "seconds": round(time.perf_counter() - t0, 1),
    }


def run_storage_d(wl: W.Workload, storage: str, steps: int = 40, warmup: int = 5):
    """Config D with reduced moment storage (scaled deviations, FP32 compute):
    whole-step MLUPS and the dense kernel's time and bandwidth, device-resident
    surfaces, CUDA events."""
    import torch
    from freeflow_b200 import DeviceSurface, FluidGrid

    g = FluidGrid(**wl.grid_kwargs(storage=storage))
    g.set_flags(wl.flags)
    g.set_moments(wl.moments)
    v0, u0 = wl.surface_at(0)
    surf = DeviceSurface(v0, u0, wl.elements)
    g.reserve_surface(surf.num_vertices, max(4096, surf.num_elements * 40))
    Vd = torch.from_numpy(np.stack([wl.surface_at(s)[0] for s in range(steps + warmup)])).cuda()
    Ud = torch.from_numpy(np.stack([wl.surface_at(s)[1] for s in range(steps + warmup)])).cuda()
    stream = torch.cuda.Stream()

    def step(s):
        surf.vertices, surf.velocities = Vd[s], Ud[s]
        g.step(surf, stream=stream)

    with torch.cuda.stream(stream):
        for s in range(warmup):
            step(s)
    torch.cuda.synchronize()
    g.profile(True)
    g.profile_read(reset=True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    with torch.cuda.stream(stream):
        for s in range(steps):
            step(warmup + s)
    e1.record(stream)
    torch.cuda.synchronize()
    g.profile(False)
    prof = g.profile_read(reset=True)
    ms = e0.elapsed_time(e1)
    status = g.status(clear=True)
    g.close()
    peak, peak_kind = hbm_peak()
    bpc = algorithmic_bytes_per_cell(3, storage)
    dense_ms = prof["dense"][0] / max(1, prof["dense"][1])
    return {"mlups": round(wl.ncell * steps / (ms * 1e-3) / 1e6, 1), "ms_per_step": round(ms / steps, 4),
            "dense_ms": round(dense_ms, 4), "bytes_per_cell": bpc,
            "dense_gbs": round(wl.ncell * bpc / (dense_ms * 1e-3) / 1e9, 1),
            "dense_frac": round(wl.ncell * bpc / (dense_ms * 1e-3) / 1e9 / peak, 4), "peak_kind": peak_kind,
            "device_status": status}


def run_coupled(wl: W.Workload, steps: int = 40, warmup: int = 5):
    """The coupled step (surface gathered from a volume mesh, fluid step, forces
    scattered back) on config D, against the same three stages issued the way
    the reference's Simulator3D::step issues them: gather, stream synchronise,
    fluid step, zero + scatter + zero, stream synchronise.  The volume mesh is
    the surface plus as many interior vertices; the body moves as in the main
    measurement (per-step volume arrays resident on the device).  CUDA events
    bracket each loop, so the host synchronisations show up as device idle
    time."""
    import torch
    from freeflow_b200 import DeviceSurface, FluidGrid, VolumeSurface

    nv = wl.rest.shape[0]
    nvol = 2 * nv
    perm = np.random.default_rng(1).permutation(nvol)[:nv].astype(np.uint32)
    n = steps + warmup
    vp = np.zeros((n, nvol, 3), np.float32)
    vv = np.zeros((n, nvol, 3), np.float32)
    for s in range(n):
        vp[s, perm], vv[s, perm] = wl.surface_at(s)
    VP, VV = torch.from_numpy(vp).cuda(), torch.from_numpy(vv).cuda()
    idx = torch.from_numpy(perm.astype(np.int64)).cuda()
    stream = torch.cuda.Stream()
    out = {}
    for mode in ("coupled", "synchronised"):
        g = FluidGrid(**wl.grid_kwargs())
        g.set_flags(wl.flags)
        g.set_moments(wl.moments)
        vol = VolumeSurface(vp[0], vv[0], perm, wl.elements)
        surf = DeviceSurface(vp[0][perm], vv[0][perm], wl.elements)
        g.reserve_surface(nv, max(4096, surf.num_elements * 40))

        def step(s):
            if mode == "coupled":
                vol.volume_positions, vol.volume_velocities = VP[s], VV[s]
                g.step_coupled(vol, stream=stream)
            else:
                torch.index_select(VP[s], 0, idx, out=surf.vertices)
                torch.index_select(VV[s], 0, idx, out=surf.velocities)
                stream.synchronize()
                g.step(surf, stream=stream)
                vol.volume_forces.zero_()
                vol.volume_forces.index_copy_(0, idx, surf.forces)
                surf.forces.zero_()
                stream.synchronize()

        with torch.cuda.stream(stream):
            for s in range(warmup):
                step(s)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
            for s in range(steps):
                step(warmup + s)
            e1.record(stream)
        torch.cuda.synchronize()
        out[mode] = {"ms_per_step": round(e0.elapsed_time(e1) / steps, 4), "device_status": g.status(clear=True)}
        g.close()
    out["case"] = (f"{wl.name}, {nvol}-vertex volume mesh ({nv} on the surface), {steps} steps; synchronised = "
                   "gather, sync, step, zero + scatter + zero, sync per step")
    return out


def run_serving_line(args):
    """`--workload E`: the serving measurement as its own JSON line (the
    headline value is the concurrency-256 mix)."""
    import torch

    torch.cuda.set_device(0)
    r = run_serving(iterations=args.steps, warmup=args.warmup)
    c = r["by_concurrency"]["256"]
    b = c["batched"]
    line = {
        "metric": "env_steps_per_s", "value": b["env_steps_per_s"], "unit": "env-steps/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1e3 * b["seconds"] / max(1, args.steps), 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f16", "data": "synthetic (seeded)",
        "config": {"workload": r["workload"], "storage": "f16", "concurrency_mean": b["concurrency_mean"],
                   "l2": "episode state exceeds L2 at this concurrency"},
        "p50_ms": b["p50_ms"], "p99_ms": b["p99_ms"],
        # per control step the pool uploads one 576-byte parameter row per episode
        # and reads back the 48-byte output records of all its slots
        "e2e": {"value": b["env_steps_per_s"], "unit": "env-steps/s", "h2d_bytes_per_step": 576,
                "d2h_bytes_per_step": round(48 * c["pool"]["max_episodes"] / max(1.0, b["concurrency_mean"]), 1)},
        "serving": r,
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------- GPU
def run_ours(args):
    import torch

    from freeflow_b200 import replicas as R

    rank, world, local = R.env_ranks()
    torch.cuda.set_device(local if world > 1 else 0)
    R.init("nccl", timeout_s=300.0, device=torch.device("cuda", local) if world > 1 else None)
    from freeflow_b200 import DeviceSurface, FluidGrid

    wl = make_workload(args.workload, args.small)
    K, Wm = args.steps, args.warmup
    storage = args.storage
    g = FluidGrid(**wl.grid_kwargs(storage=storage))
    g.set_flags(wl.flags)
    g.set_moments(wl.moments)
    stream = torch.cuda.Stream()
    surf = None
    link_stats = None
    nsteps_total = K + Wm
    if wl.elements is not None:
        v0, u0 = wl.surface_at(0)
        surf = DeviceSurface(v0, u0, wl.elements)
        g.reserve_surface(surf.num_vertices, max(4096, surf.num_elements * 40))
        # per-step surfaces for the device-resident run
        V = np.empty((nsteps_total,) + v0.shape, np.float32)
        U = np.empty_like(V)
        for s in range(nsteps_total):
            V[s], U[s] = wl.surface_at(s)
        Vd = torch.from_numpy(V).cuda()
        Ud = torch.from_numpy(U).cuda()
        cq, _ = g.debug_links(surf)
        link_stats = {"links": int(cq.size), "link_cells": int(np.unique(cq // g.info.q).size)}

    def step(s):
        if surf is not None:
            surf.vertices = Vd[s]
            surf.velocities = Ud[s]
            g.step(surf, stream=stream)
        else:
            g.step(stream=stream)

    with torch.cuda.stream(stream):
        for s in range(Wm):
            step(s)
    torch.cuda.synchronize()
    if g.status(clear=True):
        print(json.dumps({"warning": "device status set during warm-up"}), file=sys.stderr)

    # ---- timed region: inputs resident in HBM (both moment buffers exceed L2)
    clocks = ClockSampler(torch.cuda.current_device())
    R.barrier()
    torch.cuda.synchronize()
    g.profile(True)
    g.profile_read(reset=True)
    clocks.start()
    bpc = algorithmic_bytes_per_cell(wl.dim, storage)
    small = wl.ncell * bpc <= 2 * 126e6   # one moment buffer can sit in the 126 MB L2
    if not small:
        # both moment buffers exceed L2: the steps run back to back
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        with torch.cuda.stream(stream):
            for s in range(K):
                step(Wm + s)
        ev1.record(stream)
        torch.cuda.synchronize()
        elapsed = ev0.elapsed_time(ev1)
    else:
        # L2 is flushed before every step (a 256 MB write, outside the timed
        # spans) and each step is timed by its own pair of events
        scratch = torch.empty(64 << 20, dtype=torch.float32, device="cuda")
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
        with torch.cuda.stream(stream):
            for s in range(K):
                scratch.fill_(float(s))
                evs[s][0].record(stream)
                step(Wm + s)
                evs[s][1].record(stream)
        torch.cuda.synchronize()
        elapsed = sum(a.elapsed_time(b) for a, b in evs)
        del scratch
    clk = clocks.stop()
    g.profile(False)
    prof = g.profile_read(reset=True)
    ms = R.max_over_ranks(elapsed, device="cuda")
    R.barrier()
    status = g.status(clear=True)

    # ---- each stage alone: detection moved onto the step's stream ahead of
    # the dense pass (profile mode 2), a few steps after the timed region
    stages_alone = None
    if surf is not None:
        n_alone = min(K, 10)
        g.profile(True, serial=True)
        g.profile_read(reset=True)
        with torch.cuda.stream(stream):
            for s in range(n_alone):
                step(Wm + s)
        torch.cuda.synchronize()
        pa = g.profile_read(reset=True)
        g.profile(False)
        stages_alone = {k: round(v[0] / max(1, v[1]), 4) for k, v in pa.items() if v[1]}

    # ---- end to end: host surface in pinned memory -> step -> forces to host
    e2e = None
    if surf is not None:
        Vh = torch.from_numpy(V).pin_memory()
        Uh = torch.from_numpy(U).pin_memory()
        Fh = torch.empty(surf.forces.shape, dtype=torch.float32).pin_memory()
        vbuf = torch.empty_like(surf.forces)
        ubuf = torch.empty_like(surf.forces)
        surf.vertices, surf.velocities = vbuf, ubuf

        def e2e_step(s):
            vbuf.copy_(Vh[s], non_blocking=True)
            ubuf.copy_(Uh[s], non_blocking=True)
            surf.forces.zero_()
            g.step(surf, stream=stream)
            Fh.copy_(surf.forces, non_blocking=True)

        with torch.cuda.stream(stream):
            for s in range(Wm):
                e2e_step(s)
        torch.cuda.synchronize()
        R.barrier()
        if not small:
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            with torch.cuda.stream(stream):
                for s in range(K):
                    e2e_step(Wm + s)
            e1.record(stream)
            torch.cuda.synchronize()
            e_elapsed = e0.elapsed_time(e1)
        else:
            scratch = torch.empty(64 << 20, dtype=torch.float32, device="cuda")
            evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
            with torch.cuda.stream(stream):
                for s in range(K):
                    scratch.fill_(float(s))
                    evs[s][0].record(stream)
                    e2e_step(Wm + s)
                    evs[s][1].record(stream)
            torch.cuda.synchronize()
            e_elapsed = sum(a.elapsed_time(b) for a, b in evs)
            del scratch
        ems = R.max_over_ranks(e_elapsed, device="cuda")
        nb = surf.num_vertices * wl.dim * 4
        e2e = {"value": round(R.whole_job_rate(wl.ncell * K, ems * 1e-3, world) / 1e6, 1), "unit": "MLUPS",
               "h2d_bytes_per_step": 2 * nb, "d2h_bytes_per_step": nb,
               "copies": "serial: each step's uploads, step and read-back in order on one stream"}
        if not small:
            ems_p = R.max_over_ranks(e2e_pipelined(g, surf, stream, Vh, Uh, Wm, K), device="cuda")
            serial = e2e["value"]
            piped = round(R.whole_job_rate(wl.ncell * K, ems_p * 1e-3, world) / 1e6, 1)
            # both loops keep every upload and read-back inside their timed
            # region; the line reports the faster and lists both
            e2e["serial_value"] = serial
            e2e["pipelined_value"] = piped
            e2e["value"] = max(serial, piped)
            e2e["copies"] = ("the faster of two loops: serial (each step's uploads, step and read-back in order on one "
                             "stream) and pipelined (step s+1's surface uploaded and step s's forces read back on a "
                             "copy stream while step s runs, double-buffered device arrays); all K uploads and K "
                             "read-backs are inside either timed region")
            e2e["note"] = ("the device-timed value records per-stage CUDA events in its timed region (for the "
                           "roofline's kernel time); these end-to-end loops record none, so they can come out "
                           "a few percent above it")
    else:
        # no surface: the step's inputs are the moments themselves; e2e = upload
        # the initial state once, step, read back the density field once
        e2e = None

    value = R.whole_job_rate(wl.ncell * K, ms * 1e-3, world) / 1e6
    peak, peak_kind = hbm_peak()
    dense_ms, dense_n = prof["dense"]
    dense_avg_s = dense_ms * 1e-3 / max(1, dense_n)
    achieved = wl.ncell * bpc / dense_avg_s / 1e9
    # dense pass, plus detection, link cells and (for surfaces of more than
    # 2048 force components) the force conversion
    launches_per_step = 1 + ((3 if surf.num_vertices * wl.dim > 2048 else 2) if surf is not None else 0)
    tpc = DENSE_TRAFFIC_PER_CELL.get((wl.dim, storage))
    traffic = round(tpc[0] * wl.ncell) if tpc else None
    traffic_src = f"{tpc[0]} B/cell measured by ncu, scaled to {wl.ncell} cells ({tpc[1]})" if tpc else None
    out = None
    if rank == 0:
        cpu, errors = None, None
        if world == 1 and not args.no_cpu_baseline:
            cpu, errors = cpu_leg(wl, os.cpu_count() or 1)
        out = {
            "metric": "MLUPS", "value": round(value, 1), "unit": "MLUPS", "n_gpus": world, "steps": K,
            "warmup": Wm, "ms_per_step": round(ms / K, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": storage, "data": "synthetic (seeded)",
            "config": run_config(wl, storage, world),
            "links_at_step0": link_stats,
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": traffic, "traffic_source": traffic_src,
                         "peak_kind": peak_kind,
                         "kernel": "dense3d_kernel" if wl.dim == 3 else "dense2d_kernel",
                         "bytes_per_cell": bpc, "kernel_ms": round(dense_ms / max(1, dense_n), 4)},
            "stages_ms_per_step": {k: round(v[0] / max(1, v[1]), 4) for k, v in prof.items() if v[1]},
            "stages_alone_ms_per_step": stages_alone,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches_per_step * K,
            "clocks": clk,
            "device_status": status,
        }
        if errors is not None:
            out["storage_errors_vs_fp64"] = errors
        if world == 1 and not args.small and args.workload == "D" and storage == "f32":
            out["storage"] = {st: run_storage_d(wl, st) for st in ("f16", "bf16")}
            out["coupled_step"] = run_coupled(wl)
        if world == 1 and not args.no_serving and not args.small:
            out["serving"] = run_serving(iterations=150, warmup=20)
        print(json.dumps(out), flush=True)
    g.close()
    R.shutdown()
    return 0


def e2e_pipelined(g, surf, stream, Vh, Uh, first, K):
    """K end-to-end steps with the copies overlapped: step s+1's vertices and
    velocities go up, and step s's forces come back, on a copy stream while
    step s runs.  Device arrays are double-buffered; events order each slot's
    upload before its step, and its read-back before the slot is zeroed for
    the step after next.  Returns the device milliseconds of the K steps,
    every upload and read-back included."""
    import torch

    cs = torch.cuda.Stream()
    vb = [torch.empty_like(surf.forces) for _ in range(2)]
    ub = [torch.empty_like(surf.forces) for _ in range(2)]
    fb = [torch.zeros_like(surf.forces) for _ in range(2)]
    Fh = [torch.empty(surf.forces.shape, dtype=torch.float32).pin_memory() for _ in range(2)]
    uploaded = [torch.cuda.Event() for _ in range(2)]
    stepped = [torch.cuda.Event() for _ in range(2)]
    read = [torch.cuda.Event() for _ in range(2)]

    def upload(s):
        j = s & 1
        cs.wait_event(stepped[j])          # the step that last used slot j has consumed it
        with torch.cuda.stream(cs):
            vb[j].copy_(Vh[s], non_blocking=True)
            ub[j].copy_(Uh[s], non_blocking=True)
        uploaded[j].record(cs)

    def run(s, last):
        j = s & 1
        stream.wait_event(uploaded[j])
        stream.wait_event(read[j])         # step s-2's forces are on the host
        with torch.cuda.stream(stream):
            fb[j].zero_()
            surf.vertices, surf.velocities, surf.forces = vb[j], ub[j], fb[j]
            g.step(surf, stream=stream)
        stepped[j].record(stream)
        if not last:
            upload(s + 1)
        cs.wait_event(stepped[j])
        with torch.cuda.stream(cs):
            Fh[j].copy_(fb[j], non_blocking=True)
        read[j].record(cs)

    # untimed pass through the same code, then the timed one
    n0 = min(3, K)
    torch.cuda.synchronize()
    upload(first)
    for s in range(n0):
        run(first + s, s == n0 - 1)
    stream.wait_event(read[(first + n0 - 1) & 1])
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    cs.wait_event(e0)
    upload(first)
    for s in range(K):
        run(first + s, s == K - 1)
    stream.wait_event(read[(first + K - 1) & 1])
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)


def check_ranks():
    """`--check-ranks`: join the ranks over gloo and print what each one saw."""
    from freeflow_b200 import replicas as R

    rank, world, local = R.env_ranks()
    R.init("gloo", timeout_s=60.0)
    seen = R.all_gather_objects({"rank": rank, "world": world, "local_rank": local, "pid": os.getpid()})
    if rank == 0:
        print(json.dumps({"check_ranks": seen}), flush=True)
    R.shutdown()
    return 0


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=200)
    p.add_argument("--warmup", type=int, default=10)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default="D", choices=["A", "B", "C", "D", "E"])
    p.add_argument("--storage", default="f32", choices=["f32", "f16", "bf16"])
    p.add_argument("--small", action="store_true", help="reduced grid (profiling captures)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-serving", action="store_true", help="skip the serving (config E) sub-measurement")
    p.add_argument("--check-ranks", action="store_true", help="only join the ranks (gloo) and report them")
    args = p.parse_args()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # no launcher: start one process per GPU here, as torchrun would
        from freeflow_b200 import replicas as R

        return R.launch_local_ranks([os.path.abspath(__file__), *sys.argv[1:]], args.gpus)
    if args.check_ranks:
        return check_ranks()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "E":
        return run_serving_line(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
