"""CPU tests of the warm-start network's oracle (oracle/mlp_oracle.py).

The device kernels' gradients are checked against this restatement on the
GPU (tests/test_gpu_learn.py); here the restatement itself is checked: its
backward pass in float64 without BF16 rounding against central finite
differences of its forward pass, and its BF16 form against the float64 form.
"""
import numpy as np
import pytest

import mlp_oracle as M
from solfec_b200 import learn


def _problem(seed, n=24):
    rng = np.random.default_rng(seed)
    P = M.init_params(seed).astype(np.float64)
    P[M.PW3:M.PB3] = rng.normal(0, 0.1, size=M.PB3 - M.PW3)
    P[M.PW3 + 3 * M.HID:M.PB3] = 0.0      # rows 3..15 of W3 stay zero, as on the device
    P[M.PB2:M.PW3] = rng.normal(0, 0.1, size=M.HID)
    P[M.PB3:M.PB3 + 3] = rng.normal(0, 0.1, size=3)
    X = rng.normal(0, 1, size=(n, M.IN))
    X[:, M.BIAS_COL] = 1.0
    X[:, M.BIAS_COL + 1:] = 0.0
    T = rng.normal(0, 1, size=(n, 3))
    return P, X, T


def test_layout_matches_package():
    assert learn.NPARAMS == M.NPARAMS
    assert (learn.PW1, learn.PW2, learn.PB2, learn.PW3, learn.PB3) == (M.PW1, M.PW2, M.PB2, M.PW3, M.PB3)
    np.testing.assert_array_equal(learn.init_params(7), M.init_params(7))


@pytest.mark.parametrize('seed', [0, 1])
def test_oracle_backward_against_finite_differences(seed):
    P, X, T = _problem(seed)
    loss, g = M.loss_and_grad(P, X, T, rounding=False)
    rng = np.random.default_rng(100 + seed)
    live = np.r_[np.arange(M.PW1, M.PW2).reshape(M.HID, M.IN)[:, :M.BIAS_COL + 1].ravel(),
                 np.arange(M.PW2, M.PW3), np.arange(M.PW3, M.PW3 + 3 * M.HID), np.arange(M.PB3, M.PB3 + 3)]
    idx = rng.choice(live, size=60, replace=False)
    h = 1e-6
    for p in idx:
        Pp, Pm = P.copy(), P.copy()
        Pp[p] += h; Pm[p] -= h
        fd = (M.loss_and_grad(Pp, X, T, rounding=False)[0] - M.loss_and_grad(Pm, X, T, rounding=False)[0]) / (2 * h)
        assert abs(fd - g[p]) <= 1e-6 * max(1.0, abs(fd)), (p, fd, g[p])


def test_bf16_gradient_close_to_float64():
    P, X, T = _problem(3, n=256)
    l64, g64 = M.loss_and_grad(P, X, T, rounding=False)
    l16, g16 = M.loss_and_grad(P.astype(np.float32), X.astype(np.float32), T.astype(np.float32), rounding=True)
    assert abs(l16 - l64) <= 2e-2 * l64
    for a, b in ((M.PW1, M.PW2), (M.PW2, M.PB2), (M.PB2, M.PW3), (M.PW3, M.PB3), (M.PB3, M.NPARAMS)):
        assert np.linalg.norm(g16[a:b] - g64[a:b]) <= 3e-2 * np.linalg.norm(g64[a:b]) + 1e-12, (a, b)


def test_bf16_rounding_is_nearest_even():
    # BF16 spacing near 1 is 2**-7: 1 + 2**-8 and 1 + 3 * 2**-8 are ties
    x = np.array([1.0, 1.00390625, 1.01171875, 1.005859375, 1.001953125, -2.5], dtype=np.float32)
    r = M.bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0            # tie, even mantissa below
    assert r[2] == 1.015625       # tie, even mantissa above
    assert r[3] == 1.0078125 and r[4] == 1.0
    assert r[5] == -2.5
