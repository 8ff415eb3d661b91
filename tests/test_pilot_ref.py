"""The CPU reference of the learned pilot (oracle/pilot_ref.py), no GPU.

Its backward pass is checked against central finite differences of its own
forward pass in exact float64 (no bf16 rounding), so the reference the GPU
gradients are compared with is itself pinned.
"""
import os
import sys

import numpy as np

from oracle import pilot_ref as R  # noqa: E402


def test_param_layout():
    assert R.param_count() == 9 * 48 * 2 + 48 + 6 * (9 * 48 * 48 + 48) + 9 * 48 + 1
    p = R.init_params(0)
    parts = R.unpack(p)
    assert [W.shape for W, _ in parts][0] == (9, 48, 2) and parts[-1][0].shape == (9, 1, 48)


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(1)
    p = R.init_params(3).astype(np.float64)
    p[-(9 * 48 + 1):] *= 10  # a last layer large enough for clear gradients
    img = rng.uniform(0, 255, (1, 6, 7))
    sig = np.array([20.0])
    tgt = img + rng.normal(0, 5, img.shape)
    g, _ = R.gradients(p, img, sig, tgt, rounding=False)
    off = np.cumsum([0] + [9 * co * ci + co for ci, co in R.LAYERS])
    picks = [off[0] + 5, off[0] + 9 * 48 * 2 + 3, off[3] + 777, off[7] + 11, off[8] - 1]
    for k in picks:
        h = 1e-4 * max(1.0, abs(p[k]))
        pp, pm = p.copy(), p.copy()
        pp[k] += h
        pm[k] -= h
        lp = np.mean((R.forward(pp, img, sig, rounding=False)[0] - tgt) ** 2)
        lm = np.mean((R.forward(pm, img, sig, rounding=False)[0] - tgt) ** 2)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[k]) <= 1e-5 * max(1.0, abs(fd)) + 1e-7, (k, fd, g[k])


def test_conv_is_a_correlation_with_zero_padding():
    x = np.zeros((1, 5, 5, 1))
    x[0, 2, 2, 0] = 1.0
    W = np.zeros((9, 1, 1))
    W[0, 0, 0] = 1.0  # tap (dy, dx) = (-1, -1): y[p] = x[p + (-1, -1)]
    y = R.conv(x, W)
    assert y[0, 3, 3, 0] == 1.0 and y.sum() == 1.0
