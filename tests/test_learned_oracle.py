"""The NumPy restatement of the learned predictor (oracle/learned.py) pinned before it is
used as the checker of the CUDA kernels: its analytic gradient against central finite
differences, its BF16 rounding against the definition, its features on hand-made cases."""
import numpy as np
import pytest

from oracle import learned as L


def _problem(seed, N=2, H=5, W=7):
    rng = np.random.default_rng(seed)
    _, P = L.layout()
    params = rng.normal(0, 0.05, P)
    x = rng.normal(0, 1, (N, 81, H, W))
    label = rng.normal(0, 1, (N, 2, H, W))
    mask = (rng.random((N, H, W)) > 0.2).astype(np.float64)
    return params, x, label, mask


def test_parameter_count():
    lay, P = L.layout()
    assert P == 881922
    assert len(lay) == 13


def test_gradient_matches_finite_differences():
    params, x, label, mask = _problem(1)
    loss, grad, _ = L.loss_and_grad(params, x, label, mask, use_bf16=False)
    lay, _ = L.layout()
    rng = np.random.default_rng(2)
    # a few weights and the bias of every layer
    picks = []
    for (w_off, b_off, cout, cin) in lay:
        picks += list(rng.integers(w_off, w_off + cout * cin * 9, 3)) + [b_off]
    h = 1e-6
    for k in picks:
        p1, p2 = params.copy(), params.copy()
        p1[k] += h
        p2[k] -= h
        l1 = L.loss_and_grad(p1, x, label, mask, use_bf16=False)[0]
        l2 = L.loss_and_grad(p2, x, label, mask, use_bf16=False)[0]
        fd = (l1 - l2) / (2 * h)
        assert abs(fd - grad[k]) <= 1e-5 + 1e-4 * abs(fd), (k, fd, grad[k])


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 3.0e-3, 65504.0], np.float32)
    r = L.bf16(x)
    # exactly representable values stay; ties go to even; others to the nearest
    assert r[0] == 1.0 and r[3] == -2.5
    assert r[1] == 1.0 + 2 ** -7 or r[1] == 1.0  # tie between 1 and 1+2^-7: even mantissa is 1.0
    assert r[1] == 1.0
    assert r[2] == 1.0 + 2 ** -7
    assert (r.view(np.uint32) & 0xFFFF == 0).all()
    assert abs(r[4] - 3.0e-3) <= 3.0e-3 * 2 ** -8


def test_features_shift_and_normalisation():
    # frame 2 = frame 1 moved by (+8, -4) image px = (+2, -1) downsampled px: the
    # cost volume of an interior vector peaks at that shift, near 1 (the frame-2 energy is
    # the zero-shift window's, and the zero band moves frame 2's mean)
    rng = np.random.default_rng(3)
    img1 = rng.integers(0, 256, (256, 256)).astype(np.uint8)
    img2 = np.zeros_like(img1)
    img2[0:252, 8:256] = img1[4:256, 0:248]
    cv = L.features(img1, img2, Nx_vec=7, Ny_vec=7, sp_x=32, sp_y=32, Nx_left=16, Ny_left=16, ws_x=64, ws_y=64)
    assert cv.shape == (81, 7, 7)
    c = cv[:, 3, 3]
    k = int(np.argmax(c))
    assert (k // 9 - 4, k % 9 - 4) == (-1, 2)
    assert 0.85 < c[k] <= 1.05
    assert np.sort(c)[-2] < 0.5 * c[k]
    # a blank frame gives zeros, not NaN
    z = L.features(img1, np.zeros_like(img1), 3, 3, 32, 32, 16, 16, 64, 64)
    assert np.isfinite(z).all() and (z == 0).all()
