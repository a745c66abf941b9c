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
  exact products.
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
