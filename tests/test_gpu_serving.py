"""The batched serving pool on the GPU, through the C ABI (include/ffs_pool.h).

  * pool (FP32 storage) vs one grid per episode through ffs_lbm_step, fed the
    same surface: moments and last-substep forces identical (the batched
    kernels run the single-grid bodies on the same inputs)
  * pool vs the ref32 oracle: moments max |diff| <= 2e-6, forces <= 1e-4 x max |F|
  * an episode alone and in a mix of other episodes: every output identical
  * FP16 storage vs the FP64 oracle: relative L2 velocity error <= 1e-3
    (closed tank; FP32 storage, for scale, <= 5e-4)
  * admission by device memory, eviction, and graph reuse across mixes
The identity tests run once per dense work unit (FFS_POOL_SHAPE pins it): the
five tile shapes and the three row-marching strips must all give the same bits.
"""
import numpy as np
import pytest

from freeflow_b200 import serving as S

from helpers import max_abs

pytestmark = pytest.mark.gpu

TILES, STRIPS = [0, 1, 2, 3, 4], [5, 6, 7]


@pytest.fixture
def pin_shape(monkeypatch):
    def pin(shape):
        monkeypatch.setenv("FFS_POOL_SHAPE", str(shape))
    return pin


def _actions(sp, step):
    return np.random.default_rng(sp.seed * 1000 + step).uniform(-1, 1, 8).astype(np.float32)


def _run_pool(pool, slots_specs, control_steps):
    """Advances the pool; returns per slot the output records and forces of every control step."""
    outs = {s: [] for s, _ in slots_specs}
    for c in range(control_steps):
        for s, sp in slots_specs:
            pool.set_action(s, _actions(sp, c))
        pool.advance()
        for s, sp in slots_specs:
            o, F = pool.collect(s, forces=True)
            outs[s].append((o.energy, o.force[0], o.force[1], o.torque, o.status, F))
    return outs


@pytest.mark.parametrize("shape,storage", [(s, "f32") for s in TILES + STRIPS] + [(1, "f16"), (6, "f16"), (6, "bf16")])
def test_pool_f32_matches_single_grid_step(cuda, pin_shape, shape, storage):
    """Pool episodes against single grids of the same storage (FP32, and the
    16-bit paths with their codec), unit by unit: identical bits."""
    pin_shape(shape)
    specs = [S.make_episode(256, 128, seed=11, length=10), S.make_episode(512, 192, seed=12, length=10)]
    pool = S.Pool(storage=storage, budget_bytes=1 << 30, max_episodes=8)
    slots = [(pool.admit(sp), sp) for sp in specs]
    outs = _run_pool(pool, slots, 3)
    for (s, sp) in slots:
        env = S.PlainEnv(sp, storage)
        for c in range(3):
            env.set_action(_actions(sp, c))
            F = env.control_step(pool.substeps)
        assert np.array_equal(pool.get_moments(s), env.g.get_moments()), "moments differ from ffs_lbm_step"
        assert np.array_equal(outs[s][-1][5], F), "forces differ from ffs_lbm_step"
        assert np.abs(F).max() > 0
        env.close()
    pool.close()


@pytest.mark.parametrize("shape", [1] + STRIPS)
def test_pool_matches_oracle(cuda, pin_shape, shape):
    from oracle.oracle import Oracle

    pin_shape(shape)
    sp = S.make_episode(256, 128, seed=21, length=10)
    pool = S.Pool(storage="f32", budget_bytes=256 << 20, max_episodes=2)
    s = pool.admit(sp)
    o = Oracle(2, sp.nx, sp.ny, 1, viscosity=sp.viscosity, density=sp.density, dx=sp.dx, dt=sp.dt,
               boundary_velocities=[0, 0, 0, 0], periodic=0, precision="ref32")
    o.set_flags(sp.flags)
    o.set_moments(pool.get_moments(s).astype(np.float64))
    F = np.zeros(sp.rest.size)
    q = 0
    for c in range(2):
        a = _actions(sp, c)
        pool.set_action(s, a)
        pool.advance()
        for j in range(pool.substeps):
            V, U = S.swimmer_surface(sp, a, q)
            if j == pool.substeps - 1:
                F[:] = 0.0
            o.step(V, U, sp.elements, F)
            q += 1
    _, Fg = pool.collect(s, forces=True)
    assert max_abs(pool.get_moments(s), o.get_moments()) <= 2e-6
    assert max_abs(Fg.reshape(-1), F) <= 1e-4 * np.abs(F).max()
    o.close()
    pool.close()


@pytest.mark.parametrize("storage", ["f16", "f32"])
def test_strip_and_tile_units_agree_on_odd_widths(cuda, pin_shape, storage):
    """Odd row widths: 2-byte moments cannot be staged two per 4-byte copy, so
    the strip kernel copies them one by one; walls on every side exercise the
    bounce-back path of the strip kernel too."""
    res = []
    for sides in ("outlets", "walls"):
        sp = S.make_episode(255, 131, seed=51, length=10, sides=sides)
        for shape in (1, 5, 6):
            pin_shape(shape)
            pool = S.Pool(storage=storage, budget_bytes=256 << 20, max_episodes=2)
            s = pool.admit(sp)
            out = _run_pool(pool, [(s, sp)], 2)[s]
            res.append((sides, out, pool.get_moments(s)))
            pool.close()
    for k in (0, 3):
        for j in (1, 2):
            (_, oa, ma), (_, ob, mb) = res[k], res[k + j]
            for a, b in zip(oa, ob):
                assert a[:5] == b[:5]
                assert np.array_equal(a[5], b[5])
            assert np.array_equal(ma, mb)


@pytest.mark.parametrize("shape", [1] + STRIPS)
def test_episode_alone_and_in_mix_identical(cuda, pin_shape, shape):
    pin_shape(shape)
    target = S.make_episode(512, 192, seed=31, length=10)
    others = [S.make_episode(n[0], n[1], seed=40 + i, length=10)
              for i, n in enumerate([(256, 128), (1200, 400), (512, 192), (256, 128), (1200, 400)])]
    alone = S.Pool(storage="f16", budget_bytes=1 << 30, max_episodes=8)
    sa = alone.admit(target)
    out_a = _run_pool(alone, [(sa, target)], 4)[sa]
    m_a = alone.get_moments(sa)
    alone.close()

    mix = S.Pool(storage="f16", budget_bytes=1 << 30, max_episodes=8)
    pairs = [(mix.admit(sp), sp) for sp in others[:3]]
    sm = mix.admit(target)                       # a different slot and table position
    pairs += [(sm, target)] + [(mix.admit(sp), sp) for sp in others[3:]]
    assert sm != sa
    out_m = _run_pool(mix, pairs, 4)[sm]
    m_m = mix.get_moments(sm)
    mix.close()
    for a, m in zip(out_a, out_m):
        assert a[:5] == m[:5]
        assert np.array_equal(a[5], m[5])
    assert np.array_equal(m_a, m_m)


@pytest.mark.parametrize("storage,tol", [("f16", 1e-3), ("f32", 5e-4)])
def test_reduced_storage_velocity_error_vs_fp64(cuda, storage, tol):
    """Relative L2 velocity error of the pool's state against the FP64 oracle,
    fed the same surfaces, after 20 control steps (200 substeps) of a 256x128
    swimmer in a closed tank.

    The tank has walls because the reference's outlet rule switches on the
    sign of the neighbour's normal velocity: where that velocity is near zero,
    any two precisions, FP32 against FP64 included, take different branches.
    With outlets, the FP32 oracle already differs from the FP64 one by 1.5e-4
    relative after 200 substeps (the FP32 GPU path by 3e-3), whatever the
    storage.  The closed tank isolates the storage error."""
    from oracle.oracle import Oracle

    sp = S.make_episode(256, 128, seed=51, length=50, sides="walls")
    pool = S.Pool(storage=storage, budget_bytes=256 << 20, max_episodes=2)
    s = pool.admit(sp)
    o = Oracle(2, sp.nx, sp.ny, 1, viscosity=sp.viscosity, density=sp.density, dx=sp.dx, dt=sp.dt,
               boundary_velocities=[0, 0, 0, 0], periodic=0, precision="phys64")
    o.set_flags(sp.flags)
    o.set_moments(pool.get_moments(s).astype(np.float64))
    q = 0
    for c in range(20):
        a = _actions(sp, c)
        pool.set_action(s, a)
        pool.advance()
        for _ in range(pool.substeps):
            V, U = S.swimmer_surface(sp, a, q)
            o.step(V, U, sp.elements, None)
            q += 1
    out, _ = pool.collect(s)
    assert out.status == 0
    g, ref = pool.get_moments(s).astype(np.float64), o.get_moments()
    du = g[:, 1:3] - ref[:, 1:3]
    rel = np.linalg.norm(du) / np.linalg.norm(ref[:, 1:3])
    assert np.linalg.norm(ref[:, 1:3]) > 0
    assert rel <= tol, f"{storage}: relative velocity error {rel:.3e}"
    o.close()
    pool.close()


def test_admission_by_memory_and_eviction(cuda):
    big = S.make_episode(1200, 400, seed=61, length=10)
    small = S.make_episode(256, 128, seed=62, length=10)
    probe = S.Pool(storage="f16", budget_bytes=64 << 20, max_episodes=4)
    nb = probe.episode_bytes(big)
    probe.close()
    pool = S.Pool(storage="f16", budget_bytes=2 * nb + nb // 2, max_episodes=8)
    a = pool.admit(big)
    b = pool.admit(big)
    assert a is not None and b is not None
    assert pool.admit(big) is None               # over budget: refused, nothing changed
    assert pool.info()["active_episodes"] == 2
    c = pool.admit(small)                        # a smaller episode still fits
    assert c is not None
    pool.set_action(a, np.zeros(8, np.float32))
    pool.advance()
    pool.evict(a)
    d = pool.admit(big)                          # memory freed by the eviction
    assert d is not None
    pool.advance()
    for s in (b, c, d):
        o, _ = pool.collect(s)
        assert o.status == 0
    pool.close()


def test_graph_reused_across_mixes(cuda):
    specs = [S.make_episode(512, 192, seed=70 + i, length=10) for i in range(6)]
    pool = S.Pool(storage="f16", budget_bytes=1 << 30, max_episodes=8)
    slots = [pool.admit(sp) for sp in specs[:4]]
    pool.advance()
    builds = pool.info()["graph_builds"]
    pool.evict(slots[0])
    slots.append(pool.admit(specs[4]))
    pool.advance()
    pool.evict(slots[1])
    slots.append(pool.admit(specs[5]))
    pool.advance()
    info = pool.info()
    assert info["graph_builds"] == builds        # the mix changed, the graph did not
    assert info["advances"] == 3
    assert info["active_episodes"] == 4
    pool.close()


def test_batched_action_and_output_calls_match_per_slot_calls(cuda):
    specs = [S.make_episode(256, 128, seed=80 + i, length=10) for i in range(3)]
    a = S.Pool(storage="f16", budget_bytes=256 << 20, max_episodes=4)
    b = S.Pool(storage="f16", budget_bytes=256 << 20, max_episodes=4)
    sa = [a.admit(sp) for sp in specs]
    sb = [b.admit(sp) for sp in specs]
    for c in range(3):
        acts = np.stack([_actions(sp, c) for sp in specs])
        for s, act in zip(sa, acts):
            a.set_action(s, act)
        b.set_actions(sb, acts)
        a.advance()
        b.advance()
        ra = [a.collect(s)[0] for s in sa]
        rb = b.collect_many(sb)
        for o, r in zip(ra, rb):
            assert (o.energy, o.force[0], o.force[1], o.torque, o.status) == \
                (r["energy"], r["force"][0], r["force"][1], r["torque"], r["status"])
    with pytest.raises(Exception, match="no such episode"):
        b.set_actions([sb[0], 3], np.zeros((2, 8), np.float32))
    a.close()
    b.close()


def test_back_to_back_advances_without_collect(cuda):
    """Double-buffered pinned buffers: a second control step enqueued before
    the first is collected gives the same episode state and the same latest
    outputs as collecting after every step."""
    specs = [S.make_episode(256, 128, seed=90 + i, length=10) for i in range(2)]
    a = S.Pool(storage="f16", budget_bytes=256 << 20, max_episodes=4)
    b = S.Pool(storage="f16", budget_bytes=256 << 20, max_episodes=4)
    sa = [a.admit(sp) for sp in specs]
    sb = [b.admit(sp) for sp in specs]
    for c in range(0, 6, 2):
        for step in (c, c + 1):
            acts = np.stack([_actions(sp, step) for sp in specs])
            a.set_actions(sa, acts)
            a.advance()
            ra = a.collect_many(sa)
            b.set_actions(sb, acts)
            b.advance()          # the second of these runs while the first is in flight
        rb = b.collect_many(sb)
        assert ra.tobytes() == rb.tobytes()
    for s1, s2 in zip(sa, sb):
        assert np.array_equal(a.get_moments(s1), b.get_moments(s2))
    a.close()
    b.close()


def test_pipelined_serving_loop_runs_every_episode(cuda):
    """serve_pipelined: two pools stepping alternately, every admitted
    episode advanced and finished or still live at the end."""
    specs = S.serving_mix(24, seed=5, lengths=(6, 6))
    pools = [S.Pool(storage="f16", budget_bytes=1 << 30, max_episodes=16) for _ in range(2)]
    r = S.serve_pipelined(pools, specs, iterations=40, initial=12, arrivals_per_iter=0.5, seed=1)
    assert r["env_steps"] > 0 and r["diverged"] == 0
    assert r["finished"] >= 12
    assert r["p50_ms"] is not None and r["p99_ms"] >= r["p50_ms"]
    for p in pools:
        p.close()
