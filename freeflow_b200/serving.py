"""Batched serving of many swimmer episodes, and the plain per-episode path.

FreeFlow serves reinforcement learning with one simulator process per
environment (``rl/env.py:163-217``).  Each control step applies an action,
runs ``itrnum_per_step`` fluid steps and reads the forces back after each of
them.  Here a :class:`Pool` (the C ABI in ``include/ffs_pool.h``) keeps every
admitted episode on the device and advances all of them by one control step
with one CUDA-graph launch.  :func:`serve` is the request loop around it:

- episodes arrive as a Poisson stream;
- they are admitted while the pool's device-memory budget and slots allow;
- each gets its next action as soon as its previous outputs are back;
- it leaves the pool when it ends or diverges.

The loop reports aggregate env-steps/s and the p50/p99 latency from action
submission to outputs.  :class:`PlainEnv` is the baseline: one FP32 grid per
episode through ``ffs_lbm_step``, sequential launches, with a host sync per
control step.

An episode of the serving mix is a D2Q9 swimmer:

- a fish outline of ``n_boundary`` edges, 0.4 of the channel height long;
- a travelling body wave on that outline;
- outlets on all four sides.

Its 8 actions in [-1, 1] scale the wave amplitude of 8 body segments by
(1 + a/2).  This mapping is project-defined: the reference's LBS/VBD
actuation is outside the fluid step.
"""
from __future__ import annotations

import ctypes as C
import math
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from . import _capi as A
from . import workloads as W

SERVING_SIZES = ((256, 128), (512, 192), (1200, 400))

# ffs_pool_output as a numpy record (48 bytes)
OUTPUT_DTYPE = np.dtype([("energy", "<f8"), ("force", "<f8", (2,)), ("torque", "<f8"), ("status", "<u4"),
                         ("pad", "<u4")])


def _ptr(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


@dataclass
class EpisodeSpec:
    """One swimmer episode: grid, flags, swimmer arrays and its length."""
    nx: int
    ny: int
    flags: np.ndarray
    viscosity: float
    density: float
    dx: float
    dt: float
    rest: np.ndarray        # (nv, 2) float32, physical
    elements: np.ndarray    # (ne, 2) uint32
    amplitude: np.ndarray   # (nv,) float32, physical lateral amplitude
    sin_kx: np.ndarray      # (nv,) float32
    cos_kx: np.ndarray      # (nv,) float32
    segment: np.ndarray     # (nv,) int32
    omega: float
    length: int             # control steps
    seed: int
    t0: float = 0.0
    meta: dict = field(default_factory=dict)

    @property
    def ncell(self) -> int:
        return self.nx * self.ny

    def grid_kwargs(self, storage="f32") -> dict:
        return dict(dim=2, nx=self.nx, ny=self.ny, nz=1, fluid_viscosity=self.viscosity,
                    fluid_density=self.density, fluid_dx=self.dx, dt=self.dt, boundary_velocities=[0, 0, 0, 0],
                    storage=storage, periodic=0)

    def c_swimmer(self) -> A.Swimmer:
        s = A.Swimmer()
        s.num_vertices = int(self.rest.shape[0])
        s.num_elements = int(self.elements.shape[0])
        s.rest, s.elements, s.amplitude = _ptr(self.rest), _ptr(self.elements), _ptr(self.amplitude)
        s.sin_kx, s.cos_kx, s.segment = _ptr(self.sin_kx), _ptr(self.cos_kx), _ptr(self.segment)
        s.omega, s.t0 = float(self.omega), float(self.t0)
        return s

    def c_episode(self) -> A.EpisodeDesc:
        e = A.EpisodeDesc()
        g = e.grid
        g.dim, g.nx, g.ny, g.nz = 2, self.nx, self.ny, 1
        g.fluid_viscosity, g.fluid_density, g.fluid_dx, g.dt = self.viscosity, self.density, self.dx, self.dt
        e.flags = _ptr(self.flags)
        e.swimmer = self.c_swimmer()
        return e


def make_episode(nx: int, ny: int, seed: int, length: int | None = None, n_boundary: int = 198,
                 num_actions: int = 8, viscosity: float = 0.01, density: float = 10.0, dx: float = 0.005,
                 dt: float = 0.0025, tail_velocity: float = 0.05, sides: str = "outlets") -> EpisodeSpec:
    """A seeded serving episode.

    - The body is 0.4 ny cells long, with its head at (0.25 nx, 0.5 ny).
    - The four sides are outlets, as in config B, or walls (`sides="walls"`, a closed tank).
    - The body wave has wavelength L and tail amplitude 0.1 L. Its frequency makes the tail's
      lattice speed `tail_velocity` at zero action.
    """
    rng = np.random.default_rng(seed)
    f = np.full((ny, nx), W.FLUID, dtype=np.uint8)
    if sides == "walls":
        f[0, :] = f[ny - 1, :] = f[:, 0] = f[:, nx - 1] = W.WALL
    else:
        f[0, :] = W.OUTLET_DOWN
        f[ny - 1, :] = W.OUTLET_UP
        f[:, 0] = W.OUTLET_LEFT
        f[:, nx - 1] = W.OUTLET_RIGHT
    L = 0.4 * ny
    pts, e = W.fish_outline(L, n_boundary // 2, rng=rng, jitter=1e-3)
    hx, hy = 0.25 * nx, 0.5 * ny
    s = np.clip(pts[:, 0] / L, 0.0, 1.0)
    amp_cells = W.carangiform_envelope(s, L)
    k = 2.0 * math.pi / L
    tail_amp = float(W.carangiform_envelope(np.array([1.0]), L)[0])
    omega = tail_velocity / (tail_amp * dt)       # lattice tail speed = A omega dt / dx (A in cells * dx)
    rest = (np.stack([hx + pts[:, 0], hy + pts[:, 1]], axis=1) * dx).astype(np.float32)
    seg = np.minimum((s * num_actions).astype(np.int32), num_actions - 1).astype(np.int32)
    if length is None:
        length = int(rng.integers(200, 2001))
    return EpisodeSpec(nx=nx, ny=ny, flags=f.reshape(-1), viscosity=viscosity, density=density, dx=dx, dt=dt,
                       rest=rest, elements=np.ascontiguousarray(e, dtype=np.uint32),
                       amplitude=(amp_cells * dx).astype(np.float32),
                       sin_kx=np.sin(k * pts[:, 0]).astype(np.float32),
                       cos_kx=np.cos(k * pts[:, 0]).astype(np.float32),
                       segment=np.ascontiguousarray(seg), omega=float(omega), length=int(length), seed=int(seed),
                       meta=dict(body_length_cells=L))


def serving_mix(n: int, seed: int = 0, sizes=SERVING_SIZES, lengths=(200, 2000)) -> list[EpisodeSpec]:
    """n episodes with grid sizes uniform over `sizes` and lengths uniform in `lengths`."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        nx, ny = sizes[int(rng.integers(0, len(sizes)))]
        out.append(make_episode(nx, ny, seed=int(rng.integers(0, 2**31)),
                                length=int(rng.integers(lengths[0], lengths[1] + 1))))
    return out


def swimmer_surface(spec: EpisodeSpec, actions, q: int):
    """Surface (vertices, velocities) of episode substep q, with the pool's arithmetic."""
    L = A.load()
    nv = spec.rest.shape[0]
    V = np.empty((nv, 2), np.float32)
    U = np.empty((nv, 2), np.float32)
    a = np.ascontiguousarray(actions, dtype=np.float32)
    sw = spec.c_swimmer()
    A.check(L.ffs_swimmer_surface(C.byref(sw), _ptr(a), int(a.size), int(q), float(spec.dt), _ptr(V), _ptr(U)),
            "ffs_swimmer_surface")
    return V, U


# ----------------------------------------------------------------- the pool
class Pool:
    """Device pool of swimmer episodes (``include/ffs_pool.h``)."""

    def __init__(self, storage: str = "f16", budget_bytes: int = 8 << 30, max_episodes: int = 512,
                 substeps: int = 10, num_actions: int = 8, max_link_cells: int = 0):
        L = A.load()
        d = A.PoolDesc()
        d.storage = A.STORAGE[storage]
        d.budget_bytes, d.max_episodes = int(budget_bytes), int(max_episodes)
        d.substeps, d.num_actions, d.max_link_cells = int(substeps), int(num_actions), int(max_link_cells)
        d.stream = None
        self._h = C.c_void_p()
        A.check(L.ffs_pool_create(C.byref(d), C.byref(self._h)), "ffs_pool_create")
        self.storage, self.substeps, self.num_actions = storage, substeps, num_actions
        self.specs: dict[int, EpisodeSpec] = {}

    def close(self):
        if self._h:
            A.load().ffs_pool_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def episode_bytes(self, spec: EpisodeSpec) -> int:
        n = C.c_int64()
        ep = spec.c_episode()
        A.check(A.load().ffs_pool_episode_bytes(self._h, C.byref(ep), C.byref(n)), "ffs_pool_episode_bytes")
        return int(n.value)

    def admit(self, spec: EpisodeSpec):
        """Slot of the admitted episode, or None when the pool is full."""
        slot = C.c_int(-1)
        ep = spec.c_episode()
        r = A.load().ffs_pool_admit(self._h, C.byref(ep), C.byref(slot))
        if r == 4:  # FFS_ERR_CAPACITY
            return None
        A.check(r, "ffs_pool_admit")
        self.specs[slot.value] = spec
        return slot.value

    def evict(self, slot: int):
        A.check(A.load().ffs_pool_evict(self._h, int(slot)), "ffs_pool_evict")
        self.specs.pop(slot, None)

    def set_action(self, slot: int, actions):
        a = np.ascontiguousarray(actions, dtype=np.float32)
        A.check(A.load().ffs_pool_set_action(self._h, int(slot), _ptr(a), int(a.size)), "ffs_pool_set_action")

    def set_actions(self, slots, actions):
        """Actions of many slots in one call: actions is (len(slots), num_actions)."""
        sl = np.ascontiguousarray(slots, dtype=np.int32)
        a = np.ascontiguousarray(actions, dtype=np.float32).reshape(len(sl), self.num_actions)
        A.check(A.load().ffs_pool_set_actions(self._h, int(sl.size), _ptr(sl), _ptr(a)), "ffs_pool_set_actions")

    def collect_many(self, slots) -> np.ndarray:
        """Output records of many slots (a structured array with the fields of ffs_pool_output)."""
        sl = np.ascontiguousarray(slots, dtype=np.int32)
        out = np.zeros(sl.size, dtype=OUTPUT_DTYPE)
        A.check(A.load().ffs_pool_collect_many(self._h, int(sl.size), _ptr(sl), _ptr(out)), "ffs_pool_collect_many")
        return out

    def advance(self):
        A.check(A.load().ffs_pool_advance(self._h), "ffs_pool_advance")

    def collect(self, slot: int, forces: bool = False):
        """(output record, per-vertex forces of the last substep or None)."""
        out = A.PoolOutput()
        F = None
        fp = None
        if forces:
            F = np.empty((self.specs[slot].rest.shape[0], 2), np.float64)
            fp = _ptr(F)
        A.check(A.load().ffs_pool_collect(self._h, int(slot), C.byref(out), fp), "ffs_pool_collect")
        return out, F

    def get_moments(self, slot: int) -> np.ndarray:
        spec = self.specs[slot]
        m = np.empty((spec.ncell, 6), np.float32)
        A.check(A.load().ffs_pool_get_moments(self._h, int(slot), _ptr(m)), "ffs_pool_get_moments")
        return m

    def tune(self):
        A.check(A.load().ffs_pool_tune(self._h), "ffs_pool_tune")

    def info(self) -> dict:
        i = A.PoolInfo()
        A.check(A.load().ffs_pool_get_info(self._h, C.byref(i)), "ffs_pool_get_info")
        return {k: getattr(i, k) for k, _ in A.PoolInfo._fields_}


# ---------------------------------------------------------- plain baseline
class PlainEnv:
    """One episode on its own FP32 grid through ffs_lbm_step: the surface of
    every substep is computed on the host and copied in, and the forces are
    read back with a host sync once per control step."""

    def __init__(self, spec: EpisodeSpec, storage: str = "f32"):
        from .grid import DeviceSurface, FluidGrid

        self.spec = spec
        self.g = FluidGrid(**spec.grid_kwargs(storage))
        self.g.set_flags(spec.flags)
        self.g.initialize()
        self.surf = DeviceSurface(spec.rest, np.zeros_like(spec.rest), spec.elements, with_forces64=True)
        self.q = 0
        self.actions = np.zeros(8, np.float32)

    def set_action(self, actions):
        self.actions = np.ascontiguousarray(actions, dtype=np.float32)

    def control_step(self, substeps: int = 10) -> np.ndarray:
        """Runs one control step; returns the last substep's per-vertex forces."""
        for j in range(substeps):
            V, U = swimmer_surface(self.spec, self.actions, self.q)
            self.surf.update(V, U)
            if j == substeps - 1:
                self.surf.forces64.zero_()
            self.g.step(self.surf)
            self.q += 1
        return self.surf.forces64.cpu().numpy()  # the host sync of the control step

    def close(self):
        self.g.close()


# -------------------------------------------------------------- the loop
@dataclass
class _Live:
    spec: EpisodeSpec
    rng: np.random.Generator
    done_steps: int
    submitted: float


def serve(pool: Pool, specs: list[EpisodeSpec], iterations: int, initial: int, arrivals_per_iter: float,
          seed: int = 0, warmup_iterations: int = 0) -> dict:
    """Continuous-batching request loop over `pool`.

    - `initial` episodes are queued at the start. Each has already made a uniform random share of its
      length, which models a loop in steady state.
    - Each loop iteration, Poisson(`arrivals_per_iter`) more episodes arrive from `specs`.
    - Queued episodes are admitted in arrival order while the pool accepts them.
    - Every admitted episode gets a new action as soon as its previous outputs are back.
    - An episode leaves on its last control step or on a divergence (status bit 1).

    The first `warmup_iterations` iterations are not timed. Returns throughput, latency percentiles and
    concurrency figures.
    """
    rng = np.random.default_rng(seed)
    feed = deque(specs)
    queue: deque = deque()
    live: dict[int, _Live] = {}
    for _ in range(min(initial, len(feed))):
        sp = feed.popleft()
        queue.append((sp, int(rng.integers(0, max(1, sp.length)))))
    lat: list[float] = []
    conc: list[int] = []
    steps = finished = diverged = refused = 0
    t_begin = None
    for it in range(iterations + warmup_iterations):
        if it == warmup_iterations:
            t_begin = time.perf_counter()
            lat.clear()
            conc.clear()
            steps = 0
        for _ in range(int(rng.poisson(arrivals_per_iter)) if it else 0):
            if feed:
                queue.append((feed.popleft(), 0))
        while queue:
            sp, done = queue[0]
            slot = pool.admit(sp)
            if slot is None:
                refused += 1
                break
            queue.popleft()
            er = np.random.default_rng(sp.seed)
            pool.set_action(slot, er.uniform(-1.0, 1.0, pool.num_actions).astype(np.float32))
            live[slot] = _Live(sp, er, done, time.perf_counter())
        if not live:
            if not feed and not queue:
                break
            continue
        conc.append(len(live))
        pool.advance()
        slots = list(live)
        if hasattr(pool, "collect_many"):
            status = pool.collect_many(slots)["status"]
        else:
            status = [pool.collect(sl)[0].status for sl in slots]
        t = time.perf_counter()
        cont, acts = [], []
        for slot, stat in zip(slots, status):
            st = live[slot]
            lat.append(t - st.submitted)
            steps += 1
            st.done_steps += 1
            if int(stat) & A.STATUS_NONFINITE:
                diverged += 1
                pool.evict(slot)
                del live[slot]
            elif st.done_steps >= st.spec.length:
                finished += 1
                pool.evict(slot)
                del live[slot]
            else:
                cont.append(slot)
                acts.append(st.rng.uniform(-1.0, 1.0, pool.num_actions).astype(np.float32))
        if cont:
            if hasattr(pool, "set_actions"):
                pool.set_actions(cont, np.stack(acts))
            else:
                for slot, a in zip(cont, acts):
                    pool.set_action(slot, a)
            now = time.perf_counter()
            for slot in cont:
                live[slot].submitted = now
    wall = time.perf_counter() - (t_begin if t_begin is not None else time.perf_counter())
    info = pool.info() if hasattr(pool, "info") else None
    for slot in list(live):
        pool.evict(slot)
    lat_ms = np.array(lat) * 1e3
    return {
        "env_steps": steps, "seconds": wall, "env_steps_per_s": steps / wall if wall > 0 else 0.0,
        "p50_ms": float(np.percentile(lat_ms, 50)) if lat else None,
        "p99_ms": float(np.percentile(lat_ms, 99)) if lat else None,
        "concurrency_mean": float(np.mean(conc)) if conc else 0.0,
        "concurrency_min": int(np.min(conc)) if conc else 0, "concurrency_max": int(np.max(conc)) if conc else 0,
        "finished": finished, "diverged": diverged, "admission_waits": refused, "pool_info_at_end": info,
    }


def serve_pipelined(pools: list, specs: list[EpisodeSpec], iterations: int, initial: int, arrivals_per_iter: float,
                    seed: int = 0, warmup_iterations: int = 0) -> dict:
    """serve() with the live episodes split over several pools that step in
    turn, so that the host's work on one group's outputs (and the next
    actions, admissions and evictions) overlaps the GPU's control step of
    the others.  Each pool has its own stream; ffs_pool_advance returns at
    once, so every group's step is queued while the host serves the next.

    One loop iteration serves one group: collect its last control step,
    retire finished or diverged episodes, admit queued ones (keeping the
    groups even), set the next actions and advance.  `arrivals_per_iter` is
    the arrival rate per control step of the whole set, spread over the
    groups' iterations.  Latency is measured as in serve(): from action
    submission to the output being on the host.
    """
    G = len(pools)
    rng = np.random.default_rng(seed)
    feed = deque(specs)
    queue: deque = deque()
    live: list[dict] = [dict() for _ in range(G)]
    pending = [False] * G
    for _ in range(min(initial, len(feed))):
        sp = feed.popleft()
        queue.append((sp, int(rng.integers(0, max(1, sp.length)))))
    lat: list[float] = []
    conc: list[int] = []
    steps = finished = diverged = refused = 0
    t_begin = None
    for it in range(iterations + warmup_iterations):
        if it == warmup_iterations:
            t_begin = time.perf_counter()
            lat.clear()
            conc.clear()
            steps = 0
        g = it % G
        pool, lv = pools[g], live[g]
        # outputs of this group's last control step (queued G iterations ago)
        cont, acts = [], []
        if pending[g]:
            slots = list(lv)
            status = pool.collect_many(slots)["status"]
            t = time.perf_counter()
            for slot, stat in zip(slots, status):
                st = lv[slot]
                lat.append(t - st.submitted)
                steps += 1
                st.done_steps += 1
                if int(stat) & A.STATUS_NONFINITE:
                    diverged += 1
                    pool.evict(slot)
                    del lv[slot]
                elif st.done_steps >= st.spec.length:
                    finished += 1
                    pool.evict(slot)
                    del lv[slot]
                else:
                    cont.append(slot)
                    acts.append(st.rng.uniform(-1.0, 1.0, pool.num_actions).astype(np.float32))
            pending[g] = False
        for _ in range(int(rng.poisson(arrivals_per_iter / G)) if it else 0):
            if feed:
                queue.append((feed.popleft(), 0))
        # admit while this group holds fewer than its share of live and queued episodes
        share = -(-(sum(len(x) for x in live) + len(queue)) // G)
        while queue and len(lv) < share:
            sp, done = queue[0]
            slot = pool.admit(sp)
            if slot is None:
                refused += 1
                break
            queue.popleft()
            er = np.random.default_rng(sp.seed)
            cont.append(slot)
            acts.append(er.uniform(-1.0, 1.0, pool.num_actions).astype(np.float32))
            lv[slot] = _Live(sp, er, done, 0.0)
        if not lv:
            if not feed and not queue and not any(live):
                break
            continue
        conc.append(sum(len(x) for x in live))
        pool.set_actions(cont, np.stack(acts))
        now = time.perf_counter()
        for slot in cont:
            lv[slot].submitted = now
        pool.advance()
        pending[g] = True
    for g, pool in enumerate(pools):
        if pending[g]:
            pool.collect_many(list(live[g]))
    wall = time.perf_counter() - (t_begin if t_begin is not None else time.perf_counter())
    for g, pool in enumerate(pools):
        for slot in list(live[g]):
            pool.evict(slot)
    lat_ms = np.array(lat) * 1e3
    return {
        "env_steps": steps, "seconds": wall, "env_steps_per_s": steps / wall if wall > 0 else 0.0,
        "p50_ms": float(np.percentile(lat_ms, 50)) if lat else None,
        "p99_ms": float(np.percentile(lat_ms, 99)) if lat else None,
        "concurrency_mean": float(np.mean(conc)) if conc else 0.0,
        "concurrency_min": int(np.min(conc)) if conc else 0, "concurrency_max": int(np.max(conc)) if conc else 0,
        "finished": finished, "diverged": diverged, "admission_waits": refused, "groups": G,
    }


def plain_rate(specs: list[EpisodeSpec], control_steps: int, substeps: int = 10, min_seconds: float = 0.0) -> dict:
    """Plain per-episode path over `specs`, one episode at a time: env-steps/s
    and per-step latency percentiles (each control step ends with a host sync).

    Each episode runs at least `control_steps` control steps and at least
    `min_seconds` of timed control steps.  The rate weights every spec equally
    (the mix of the batched path draws its grid sizes uniformly): one env-step
    of the mix costs the mean, over the specs, of their mean step times."""
    import torch

    lat = []
    per_spec = []
    t0 = time.perf_counter()
    for sp in specs:
        env = PlainEnv(sp)
        rng = np.random.default_rng(sp.seed)
        env.set_action(rng.uniform(-1.0, 1.0, 8).astype(np.float32))
        env.control_step(substeps)  # warm: first-step set-up of this grid
        torch.cuda.synchronize()
        mine = []
        while len(mine) < control_steps or sum(mine) < min_seconds:
            a = time.perf_counter()
            env.set_action(rng.uniform(-1.0, 1.0, 8).astype(np.float32))
            env.control_step(substeps)
            mine.append(time.perf_counter() - a)
        env.close()
        lat.extend(mine)
        per_spec.append({"grid": f"{sp.nx}x{sp.ny}", "env_steps": len(mine), "seconds": round(sum(mine), 3),
                         "env_steps_per_s": round(len(mine) / sum(mine), 1),
                         "p50_ms": round(float(np.percentile(np.array(mine) * 1e3, 50)), 4)})
    mean_step = float(np.mean([s["seconds"] / s["env_steps"] for s in per_spec]))
    lat_ms = np.array(lat) * 1e3
    return {"env_steps": len(lat), "seconds": float(sum(lat)),
            "env_steps_per_s": 1.0 / mean_step if mean_step > 0 else 0.0,
            "p50_ms": float(np.percentile(lat_ms, 50)), "p99_ms": float(np.percentile(lat_ms, 99)),
            "per_grid": per_spec, "wall_including_setup_s": time.perf_counter() - t0}
