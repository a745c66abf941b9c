"""Host-side logic of the serving path (no GPU): episode generation, the
swimmer kinematics shared by the pool and the plain path, and the
continuous-batching request loop driven against an in-memory pool."""
import math

import numpy as np

from freeflow_b200 import _capi as A
from freeflow_b200 import serving as S
from freeflow_b200 import workloads as W


def test_episode_shapes_and_tail_speed():
    sp = S.make_episode(256, 128, seed=3, length=50)
    nv = sp.rest.shape[0]
    assert sp.flags.shape == (256 * 128,) and sp.flags.dtype == np.uint8
    assert sp.elements.shape == (nv, 2) and sp.elements.max() < nv
    assert sp.segment.min() >= 0 and sp.segment.max() <= 7
    assert (sp.flags.reshape(128, 256)[0, 1:-1] == W.OUTLET_DOWN).all()  # corners: the columns win
    # lattice speed of the tail at zero action: A omega dt / dx
    tail = float(sp.amplitude.max()) * sp.omega * sp.dt / sp.dx
    assert abs(tail - 0.05) < 1e-3


def _numpy_surface(sp, actions, q):
    """The kinematics restated with float32 numpy operations, one rounding per
    operation in the order of swimmer_vertex."""
    f = np.float32
    beta = sp.omega * (sp.t0 + q * sp.dt)
    sb, cb = f(math.sin(beta)), f(math.cos(beta))
    a = np.where(sp.segment >= 0, np.asarray(actions, f)[np.maximum(sp.segment, 0)], f(0))
    A_ = sp.amplitude * (f(1) + f(0.5) * a)
    sn = sp.sin_kx * cb - sp.cos_kx * sb
    cs = sp.cos_kx * cb + sp.sin_kx * sb
    y = sp.rest[:, 1] + A_ * sn
    vy = -((A_ * f(sp.omega)) * cs)
    V = np.stack([sp.rest[:, 0], y], axis=1).astype(f)
    U = np.stack([np.zeros_like(y), vy], axis=1).astype(f)
    return V, U


def test_swimmer_surface_matches_float32_restatement():
    sp = S.make_episode(512, 192, seed=5, length=10)
    rng = np.random.default_rng(0)
    for q in (0, 1, 37, 9999):
        act = rng.uniform(-1, 1, 8).astype(np.float32)
        V, U = S.swimmer_surface(sp, act, q)
        V2, U2 = _numpy_surface(sp, act, q)
        assert np.array_equal(V, V2)
        assert np.array_equal(U, U2)


def test_swimmer_surface_rejects_short_action_vector():
    sp = S.make_episode(256, 128, seed=1, length=10)
    try:
        S.swimmer_surface(sp, np.zeros(3, np.float32), 0)
    except A.FfsError as e:
        assert "segment" in str(e)
    else:
        raise AssertionError("a segment index beyond the actions must be rejected")


class FakePool:
    """In-memory stand-in with the Pool interface: a slot and byte budget,
    one output per advance, divergence injected for chosen episodes."""

    def __init__(self, max_episodes, budget, diverge_seeds=()):
        self.num_actions = 8
        self.max, self.budget, self.used = max_episodes, budget, 0
        self.slots = {}
        self.diverge = set(diverge_seeds)
        self.advances = 0
        self.actions_seen = {}

    def admit(self, sp):
        if len(self.slots) >= self.max or self.used + sp.ncell > self.budget:
            return None
        s = next(i for i in range(self.max) if i not in self.slots)
        self.slots[s] = sp
        self.used += sp.ncell
        return s

    def evict(self, s):
        self.used -= self.slots.pop(s).ncell

    def set_action(self, s, a):
        assert s in self.slots and len(a) == 8
        self.actions_seen[s] = self.actions_seen.get(s, 0) + 1

    def advance(self):
        self.advances += 1

    def collect(self, s, forces=False):
        o = A.PoolOutput()
        o.status = A.STATUS_NONFINITE if self.slots[s].seed in self.diverge else 0
        return o, None


def test_request_loop_admits_as_memory_frees():
    specs = [S.EpisodeSpec(nx=10, ny=10, flags=None, viscosity=0.01, density=1, dx=1, dt=1, rest=None,
                           elements=None, amplitude=None, sin_kx=None, cos_kx=None, segment=None, omega=1.0,
                           length=5 + (i % 4), seed=i) for i in range(40)]
    pool = FakePool(max_episodes=8, budget=600, diverge_seeds={7})
    r = S.serve(pool, specs, iterations=200, initial=12, arrivals_per_iter=0.5, seed=1)
    assert r["concurrency_max"] <= 6                 # the byte budget binds before the slot count
    assert r["admission_waits"] > 0                  # arrivals queued while the pool was full
    assert r["diverged"] == 1
    assert r["finished"] + r["diverged"] == 40       # every episode ran to its end or diverged
    assert r["env_steps"] > 0 and pool.advances > 0
    assert not pool.slots and pool.used == 0         # everything evicted
    assert r["p50_ms"] is not None and r["p99_ms"] >= r["p50_ms"]


def test_request_loop_counts_every_control_step():
    specs = [S.EpisodeSpec(nx=4, ny=4, flags=None, viscosity=0.01, density=1, dx=1, dt=1, rest=None,
                           elements=None, amplitude=None, sin_kx=None, cos_kx=None, segment=None, omega=1.0,
                           length=3, seed=i) for i in range(5)]
    pool = FakePool(max_episodes=16, budget=10**6)
    r = S.serve(pool, specs, iterations=50, initial=5, arrivals_per_iter=0.0, seed=0)
    # initial episodes start part-way through their length: 1..3 steps each
    assert 5 <= r["env_steps"] <= 15
    assert r["finished"] == 5
