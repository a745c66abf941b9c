"""Known-answer and invariant tests of the CPU oracle (no GPU).

The reference ships no tests or golden data for the fluid step, so the oracle
is pinned here by facts that follow from the reference's own equations:
exact equilibrium reproduction, the equilibrium fixed point of the
collision, lattice symmetries, conservation on a periodic box, analytic
Taylor-Green decay, hand-checked link geometry and the momentum-exchange
force of a single moving-wall link.
"""
import numpy as np
import pytest

from oracle import oracle as O
from freeflow_b200 import workloads as W

EX2 = np.array([0, 1, 0, -1, 0, 1, -1, -1, 1])
EY2 = np.array([0, 0, 1, 0, -1, 1, 1, -1, -1])
INV2 = np.array([0, 3, 4, 1, 2, 7, 8, 5, 6])
EX3 = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1])
EY3 = np.array([0, 0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1])
EZ3 = np.array([0, 0, 0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1])
INV3 = np.array([0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17, 20, 19, 22, 21, 24, 23, 26, 25])


def moments_of(dim, f):
    f = np.asarray(f, dtype=np.float64)
    if dim == 2:
        rho = f.sum()
        jx, jy = (f * EX2).sum(), (f * EY2).sum()
        return np.array([rho, jx / rho, jy / rho, (f * EX2 * EX2).sum() / rho - 1 / 3,
                         (f * EY2 * EY2).sum() / rho - 1 / 3, (f * EX2 * EY2).sum() / rho])
    rho = f.sum()
    c = [EX3, EY3, EZ3]
    out = [rho] + [(f * c[a]).sum() / rho for a in range(3)]
    out += [(f * c[a] * c[a]).sum() / rho - 1 / 3 for a in range(3)]
    out += [(f * c[0] * c[1]).sum() / rho, (f * c[1] * c[2]).sum() / rho, (f * c[0] * c[2]).sum() / rho]
    return np.array(out)


def random_state(dim, rng, neq=True):
    rho = 1.0 + rng.uniform(-0.02, 0.02)
    u = rng.uniform(-0.05, 0.05, size=dim)
    m = W.equilibrium_moments(np.array([rho]), u[None, :], dtype=np.float64)[0]
    if neq:
        m[1 + dim:] += rng.uniform(-1e-3, 1e-3, size=m.size - 1 - dim)
    return m


def test_lattice_tables():
    for ex, ey, ez, inv in ((EX2, EY2, 0 * EX2, INV2), (EX3, EY3, EZ3, INV3)):
        assert np.all(inv[inv] == np.arange(inv.size))
        assert np.all(ex[inv] == -ex) and np.all(ey[inv] == -ey) and np.all(ez[inv] == -ez)


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("precision", ["ref32", "phys64"])
def test_reconstruction_reproduces_moments(dim, precision):
    """The third-order Hermite reconstruction carries rho, u and pi exactly."""
    rng = np.random.default_rng(1)
    tol = 1e-6 if precision == "ref32" else 1e-13
    for _ in range(20):
        m = random_state(dim, rng)
        f = O.reconstruct(dim, m, precision)
        assert np.allclose(moments_of(dim, f), m, rtol=0, atol=tol)


@pytest.mark.parametrize("dim", [2, 3])
def test_reconstruct_at_matches_all(dim):
    rng = np.random.default_rng(2)
    m = random_state(dim, rng)
    f = O.reconstruct(dim, m, "phys64")
    q = 9 if dim == 2 else 27
    at = np.array([O.reconstruct_at(dim, m, i, "phys64") for i in range(q)])
    assert np.allclose(at, f, atol=1e-15)


@pytest.mark.parametrize("dim", [2, 3])
def test_collision_equilibrium_fixed_point(dim):
    rng = np.random.default_rng(3)
    for nu in (0.005, 0.016, 0.1):
        omega = 1.0 / (3 * nu + 0.5)
        m = random_state(dim, rng, neq=False)
        out = O.collide_pops(dim, O.reconstruct(dim, m, "phys64"), omega, "phys64")
        assert np.allclose(out, m, atol=1e-14)


@pytest.mark.parametrize("dim", [2, 3])
def test_collision_relaxes_nonequilibrium(dim):
    """Off-diagonal non-equilibrium stress relaxes by exactly (1 - omega)."""
    rng = np.random.default_rng(4)
    omega = 1.0 / (3 * 0.02 + 0.5)
    m = random_state(dim, rng, neq=False)
    neq = m.copy()
    k = 5 if dim == 2 else 7
    neq[k] += 1e-3
    out = O.collide_pops(dim, O.reconstruct(dim, neq, "phys64"), omega, "phys64")
    assert out[k] - m[k] == pytest.approx((1 - omega) * 1e-3, rel=1e-9)


def test_half_rounding_matches_numpy():
    rng = np.random.default_rng(5)
    for v in rng.uniform(-1, 1, size=200).astype(np.float32):
        assert O.lib().ffo_round_half(float(v)) == float(np.float32(np.float16(v)))


@pytest.mark.parametrize("precision", ["ref32", "phys64"])
def test_uniform_flow_is_invariant(precision):
    o = O.Oracle(3, 6, 5, 4, viscosity=0.02, precision=precision)
    u = np.array([0.04, -0.01, 0.02])
    dt = np.float32 if precision == "ref32" else np.float64
    m = np.tile(W.equilibrium_moments(np.array([1.0]), u[None, :], dtype=dt)[0], (o.ncell, 1))
    o.set_moments(m)
    for _ in range(3):
        o.step()
    assert np.abs(o.get_moments() - m).max() < (2e-6 if precision == "ref32" else 1e-14)


@pytest.mark.parametrize("dim", [2, 3])
def test_periodic_box_conserves_mass_and_momentum(dim):
    rng = np.random.default_rng(6)
    n = (12, 10, 8) if dim == 3 else (16, 12, 1)
    o = O.Oracle(dim, *n, viscosity=0.02, periodic=7, precision="phys64")
    ncell = o.ncell
    rho = 1 + rng.uniform(-0.01, 0.01, ncell)
    u = rng.uniform(-0.03, 0.03, (ncell, dim))
    o.set_moments(W.equilibrium_moments(rho, u))
    m0 = o.get_moments()
    mass0 = m0[:, 0].sum()
    mom0 = (m0[:, 0:1] * m0[:, 1:1 + dim]).sum(axis=0)
    for _ in range(20):
        o.step()
    m = o.get_moments()
    assert m[:, 0].sum() == pytest.approx(mass0, rel=1e-12)
    assert np.allclose((m[:, 0:1] * m[:, 1:1 + dim]).sum(axis=0), mom0, atol=1e-11)


def _tgv_rate_ratio(dim, n, nu=0.02, u0=0.001, base_steps=25, base_n=16):
    """log(KE ratio) of the simulated TGV over the analytic log ratio."""
    steps = int(base_steps * (n / base_n) ** 2)  # same nu k^2 t at every n
    k = 2 * np.pi / n
    if dim == 3:
        wl = W.taylor_green_3d(n=n, u0=u0, viscosity=nu)
        m0 = W.equilibrium_moments(wl.moments[:, 0].astype(np.float64), wl.moments[:, 1:4].astype(np.float64),
                                   dtype=np.float64)
        o = O.Oracle(3, n, n, n, viscosity=nu, periodic=7, precision="phys64")
        ke = W.tgv_kinetic_energy
        expected = -6 * nu * k * k * steps
    else:
        c = 2 * np.pi * (np.arange(n) + 0.5) / n
        y, x = np.meshgrid(c, c, indexing="ij")
        u = np.stack([u0 * np.sin(x) * np.cos(y), -u0 * np.cos(x) * np.sin(y)], -1).reshape(-1, 2)
        rho = 1 + 3 * (u0 ** 2 / 4) * (np.cos(2 * x) + np.cos(2 * y)).reshape(-1)
        m0 = W.equilibrium_moments(rho, u, dtype=np.float64)
        o = O.Oracle(2, n, n, viscosity=nu, periodic=3, precision="phys64")
        ke = lambda m: 0.5 * (m[:, 0] * (m[:, 1] ** 2 + m[:, 2] ** 2)).mean()
        expected = -4 * nu * k * k * steps
    o.set_moments(m0)
    e0 = ke(o.get_moments())
    for _ in range(steps):
        o.step()
    return np.log(ke(o.get_moments()) / e0) / expected


@pytest.mark.parametrize("dim,n0", [(2, 32), (3, 16)])
def test_taylor_green_decay_converges_second_order(dim, n0):
    """Taylor-Green decay, KE ~ exp(-2 nu |k|^2 t): the rate error of the
    lattice solution falls ~4x per grid doubling (second order) and is within
    a few percent on the finer grid."""
    r1 = _tgv_rate_ratio(dim, n0)
    r2 = _tgv_rate_ratio(dim, 2 * n0)
    e1, e2 = abs(r1 - 1), abs(r2 - 1)
    assert 3.2 < e1 / e2 < 4.8
    assert e2 < (0.015 if dim == 2 else 0.05)


def test_walls_bounce_back_channel():
    """A closed box with walls keeps a resting fluid at rest and conserves mass."""
    o = O.Oracle(2, 12, 10, viscosity=0.05, precision="phys64")
    f = np.full((10, 12), W.FLUID, np.uint8)
    f[0, :] = f[-1, :] = f[:, 0] = f[:, -1] = W.WALL
    o.set_flags(f)
    o.initialize()
    for _ in range(5):
        o.step()
    m = o.get_moments()
    assert np.abs(m[:, 1:3]).max() < 1e-15
    assert np.allclose(m[:, 0], 1.0, atol=1e-14)


def test_initializer_sets_inlet_equilibrium():
    wl = W.cylinder_channel_2d(nx=32, ny=16, radius=3, center=(8, 8))
    o = O.Oracle(2, 32, 16, boundary_velocities=[0.05, 0, 0, 0], precision="ref32")
    o.set_flags(wl.flags)
    o.initialize()
    m = o.get_moments()
    inlet = wl.flags == W.INLET_LEFT
    assert np.allclose(m[inlet, 1], 0.05) and np.allclose(m[inlet, 3], 0.05 ** 2, atol=1e-7)
    assert np.allclose(m[~inlet, 1:], 0.0, atol=1e-7)  # FP32: one ulp of 1/3 survives in pi_aa
    assert np.allclose(m[:, 0], 1.0)


def test_outlet_rule_copies_outward_velocity():
    """OutletRight copies u_x of its inner neighbour when positive and sets pi_xx = u^2."""
    nx, ny = 8, 3
    f = np.full((ny, nx), W.FLUID, np.uint8)
    f[:, nx - 1] = W.OUTLET_RIGHT
    o = O.Oracle(2, nx, ny, viscosity=0.05, precision="phys64")
    o.set_flags(f)
    u = np.zeros((nx * ny, 2))
    u[:, 0] = 0.03
    u[f.reshape(-1) == W.OUTLET_RIGHT, 0] = 0.0
    o.set_moments(W.equilibrium_moments(np.ones(nx * ny), u))
    o.step()
    m = o.get_moments().reshape(ny, nx, 6)
    assert np.allclose(m[:, nx - 1, 1], m[:, nx - 2, 1])
    assert np.allclose(m[:, nx - 1, 3], m[:, nx - 2, 1] ** 2)


def test_segment_link_geometry():
    """A vertical-ish wall segment between x=2 and x=3 cuts the +x links of cells at x=3."""
    # segment from (2.5, -5) to (2.6, 5) in lattice units, dx = 1
    V = np.array([[2.5, -5.0], [2.6, 5.0]], np.float32)
    E = np.array([[0, 1]], np.uint32)
    o = O.Oracle(2, 6, 4, viscosity=0.05, precision="ref32")
    o.step(V, np.zeros_like(V), E)
    cq, key = o.links()
    cells, dirs = cq // 9, cq % 9
    xs, ys = cells % 6, cells // 6
    # links from x=3 looking back along -c: c=(1,*) dirs 1,5,8 pull from x=2
    got = set(zip(xs.tolist(), ys.tolist(), dirs.tolist()))
    for y in range(4):
        assert (3, y, 1) in got
        assert (2, y, 3) in got
    # depth = fraction from the cell to the wall, element 0
    for x, d, k in zip(xs, dirs, key):
        assert (int(k) & 0xFFFFFFFF) == 0
        dq = int(k) >> 32
        assert 0 <= dq <= 32768


def test_segment_parallel_to_link_misses():
    """The reference's x-extent test rejects segments with equal x (vertical)."""
    V = np.array([[2.5, -5.0], [2.5, 5.0]], np.float32)
    E = np.array([[0, 1]], np.uint32)
    o = O.Oracle(2, 6, 4, viscosity=0.05, precision="ref32")
    o.step(V, np.zeros_like(V), E)
    cq, _ = o.links()
    dirs = cq % 9
    assert not np.any(dirs == 1)  # purely horizontal links never register


def test_triangle_link_geometry():
    """A large triangle in the plane z = 2.5 cuts every +-z link between z=2 and z=3."""
    V = np.array([[-10, -10, 2.5], [30, -10, 2.5], [-10, 30, 2.5]], np.float32)
    E = np.array([[0, 1, 2]], np.uint32)
    o = O.Oracle(3, 4, 4, 6, viscosity=0.05, precision="ref32")
    o.step(V, np.zeros_like(V), E)
    cq, key = o.links()
    cells, dirs = cq // 27, cq % 27
    zs = cells // 16
    # every link that crosses z=2.5 belongs to a cell at z=3 (c_z=+1) or z=2 (c_z=-1)
    assert set(zs.tolist()) == {2, 3}
    assert np.all((EZ3[dirs] == 1) == (zs == 3))
    # depth 0.5 for straight z links
    straight = (dirs == 5) | (dirs == 6)
    assert np.all((key[straight] >> np.uint64(32)) == 16384)


def test_moving_wall_link_force_sign():
    """A wall moving in +x pushes the fluid: the fluid force on the wall points to -x."""
    nx, ny = 10, 6
    o = O.Oracle(2, nx, ny, viscosity=0.05, density=1.0, dx=1.0, dt=1.0, precision="phys64", periodic=2)
    f = np.full((ny, nx), W.FLUID, np.uint8)
    o.set_flags(f)
    o.set_moments(W.equilibrium_moments(np.ones(nx * ny), np.zeros((nx * ny, 2))))
    V = np.array([[4.55, -3.0], [4.45, 9.0]], np.float32)
    U = np.array([[0.01, 0.0], [0.01, 0.0]], np.float32)
    E = np.array([[0, 1]], np.uint32)
    F = np.zeros(4)
    o.step(V, U, E, F)
    fx = F[0] + F[2]
    assert fx < 0
    assert abs(F[1] + F[3]) < abs(fx)
