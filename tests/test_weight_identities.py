"""Float identities the D3Q27 dense pass relies on, checked on the CPU in
IEEE single precision:

* the reference's lattice weights, one float constant per class
  (8/27, 2/27, 1/54, 1/216), are exactly fl(8/27) times 4^-n for n non-zero
  velocity components, so populations can be stored without their weights and
  the weights applied by powers of two in the pulls;
* those constants sum over the 27 directions to 1 + 7.4e-9 (the reference's
  own mass bias), where the products of the float-rounded 1D weights 2/3 and
  1/6 would sum to 1 + 1.1e-7;
* the power-of-two scales of the scaled raw-moment sums times fl(8/27) are
  exact products;
* the kernel's accumulation of unweighted populations (slice sums with their
  1/4 factors, the c_z = 0 slice added as 4 Y, completion by W0 s_k) gives
  the raw moments of the weighted populations.
"""
import itertools

import numpy as np

W0 = np.float32(8.0) / np.float32(27.0)
CLASS = [np.float32(8.0 / 27.0), np.float32(2.0 / 27.0), np.float32(1.0 / 54.0), np.float32(1.0 / 216.0)]


def test_class_weights_are_powers_of_four_of_one_constant():
    assert CLASS[0] == W0
    for n, w in enumerate(CLASS):
        assert w == W0 * np.float32(4.0 ** -n)
        assert w / np.float32(4.0 ** -n) == W0


def test_weight_sum_bias_matches_the_reference():
    s = np.float64(0.0)
    for c in itertools.product((-1, 0, 1), repeat=3):
        s += np.float64(CLASS[sum(x != 0 for x in c)])
    assert abs(s - 1.0) < 1e-8
    assert abs(s - 1.0 - 7.4e-9) < 1e-9
    w1 = {0: np.float32(2.0 / 3.0), 1: np.float32(1.0 / 6.0)}
    p = np.float64(0.0)
    for c in itertools.product((-1, 0, 1), repeat=3):
        p += np.float64(w1[c[0] != 0] * w1[c[1] != 0] * w1[c[2] != 0])
    assert abs(p - 1.0) > 1e-7


def test_scaled_sum_factors_are_exact():
    scales = [0.25, 0.0625, 0.0625, 0.25, 0.0625, 0.0625, 0.25, 0.015625, 0.0625, 0.0625]
    for sc in scales:
        f = W0 * np.float32(sc)
        assert np.float64(f) == np.float64(W0) * sc
        # scaling a sum by the factor equals scaling by W0 and the power of two separately
        x = np.float32(0.3712345)
        assert x * f == (x * W0) * np.float32(sc)


def _scaled_raw_moments(F):
    """The single-plane dense kernel's accumulation, restated in float64: unweighted
    populations F[kx, ky, kz] (k = c + 1, clamped), slice sums with the 1/4 factors,
    the c_z = 0 slice added as 4 Y, the others as Y, then R_k = W0 s_k R''_k."""
    s = [0.25, 0.0625, 0.0625, 0.25, 0.0625, 0.0625, 0.25, 0.015625, 0.0625, 0.0625]
    R = np.zeros(10)
    for kz in range(3):
        X0, X1, X2 = np.zeros(3), np.zeros(3), np.zeros(3)
        for ky in range(3):
            fm, f0, fp = (max(F[k, ky, kz], 0.0) for k in range(3))
            sm = fp + fm
            X1[ky], X0[ky], X2[ky] = fp - fm, 0.25 * sm + f0, sm
        s0 = X0[2] + X0[0]
        Y = [0.25 * s0 + X0[1], X0[2] - X0[0], s0, 0.25 * (X1[2] + X1[0]) + X1[1], X1[2] - X1[0],
             0.25 * (X2[2] + X2[0]) + X2[1]]
        cz = kz - 1
        if cz == 0:
            for k, y in zip((0, 2, 5, 1, 7, 4), Y):
                R[k] += 4.0 * y
        else:
            for k, y in zip((0, 2, 5, 1, 7, 4), Y):
                R[k] += y
            R[3] += cz * Y[0]
            R[6] += Y[0]
            R[8] += cz * Y[1]
            R[9] += cz * Y[3]
    return np.array([float(W0) * sk * r for sk, r in zip(s, R)])


def test_scaled_slice_sums_equal_the_weighted_raw_moments():
    """The kernel's scaled sums of unweighted populations are the raw moments
    {rho, jx, jy, jz, Pxx, Pyy, Pzz, Pxy, Pyz, Pxz} of the weighted populations
    (real-number identity, checked in float64 on seeded populations, some negative
    so that the clamp matters)."""
    rng = np.random.default_rng(7)
    for _ in range(20):
        F = rng.uniform(-0.2, 1.5, (3, 3, 3))
        direct = np.zeros(10)
        for kx, ky, kz in itertools.product(range(3), repeat=3):
            cx, cy, cz = kx - 1, ky - 1, kz - 1
            w = float(CLASS[(cx != 0) + (cy != 0) + (cz != 0)])
            f = w * max(F[kx, ky, kz], 0.0)
            direct += f * np.array([1, cx, cy, cz, cx * cx, cy * cy, cz * cz, cx * cy, cy * cz, cx * cz])
        assert np.allclose(_scaled_raw_moments(F), direct, rtol=1e-13, atol=1e-15)
