"""The band proposer's network restatement (tests/proposer_net.py), on the CPU.

Its hand-derived gradient (the same chain of GEMMs, col2im, un-pooling and
ReLU masks the CUDA training kernels run) must equal central finite
differences of its own loss in float64, and its BF16 mode must stay close to
float64; the GPU tests then compare the CUDA forward pass and gradient with
this restatement.
"""
import numpy as np
import pytest

from tests import proposer_net as net


@pytest.mark.parametrize("seed", [1, 2])
def test_gradient_matches_finite_differences(seed):
    w, X, Y = net.random_problem(seed, 3)
    loss, g = net.loss_and_gradient(w, X, Y, use_bf16=False)
    rng = np.random.default_rng(seed + 100)
    # every layer's weights and biases: a sample of each block
    idx, o = [], 0
    for name, shape in net.SHAPES:
        k = int(np.prod(shape))
        idx.extend((o + rng.choice(k, min(k, 12), replace=False)).tolist())
        o += k
    eps = 1e-6
    for i in idx:
        wp, wm = w.copy(), w.copy()
        wp[i] += eps
        wm[i] -= eps
        lp, _ = net.loss_and_gradient(wp, X, Y, use_bf16=False)
        lm, _ = net.loss_and_gradient(wm, X, Y, use_bf16=False)
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(fd), (i, fd, g[i])


def test_bf16_mode_tracks_float64():
    w, X, Y = net.random_problem(3, 16)
    y64 = net.predict(w, X, use_bf16=False)
    y16 = net.predict(w, X, use_bf16=True)
    assert np.max(np.abs(y64 - y16)) <= 0.05 * np.max(np.abs(y64)) + 1e-3
    _, g64 = net.loss_and_gradient(w, X, Y, use_bf16=False)
    _, g16 = net.loss_and_gradient(w, X, Y, use_bf16=True)
    cos = float(g64 @ g16 / np.linalg.norm(g64) / np.linalg.norm(g16))
    assert cos > 0.999


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.00390625, 1.005859375, 1.0078125, -3.1415926], dtype=np.float32)
    r = net.bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0            # exactly half an ulp above 1.0: ties to even (1.0)
    assert r[2] == 1.0078125      # above half: rounds up
    assert r[3] == 1.0078125      # representable
    assert abs(r[4] + 3.140625) < 1e-7
