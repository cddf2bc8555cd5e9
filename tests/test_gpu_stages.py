"""Stage-by-stage parity of the CUDA engine against the CPU oracle, through the C-ABI.

Each test feeds one stage identical inputs on both sides:
  MHE                         bit-exact (integer path)
  correlation planes          FP32 engine vs FP64 oracle, relative 2e-6 of the window peak
  candidate search / top-N    on the engine's own FP32 planes: counts and peak indices
                              bit-exact, displacements within 1e-4 px (FP32 log numerator
                              vs FP64), windows with exact value ties or slot overflow
                              excluded (the reference itself is order-dependent there)
  deformation, upsampling     FP32 with FMA contraction vs without: 2e-3 grey levels / 1e-5 px
  validation                  bit-exact (FP32 arithmetic written as the reference writes it)
"""
import numpy as np
import pytest

import piv_b200 as P
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def c0_params(N=256, ws=32, sp=16, **kw):
    d = dict(Nx=N, Ny=N, ws_x1=ws, ws_y1=ws, spacing_x1=sp, spacing_y1=sp, Npass1=1, ws_x2=ws, ws_y2=ws,
             spacing_x2=sp, spacing_y2=sp, Npass2=0, max_dispx_win_percent1=0.25, max_dispy_win_percent1=0.25,
             max_dispx_win_percent2=0.25, max_dispy_win_percent2=0.25, insert_threshold_p1=2.0,
             insert_threshold_p2=2.0)
    d.update(kw)
    return P.default_params(**d)


def gather_windows(img, geom, grid, wsx, wsy, spx, spy):
    """organize_data_fft2d_multi: window (ix, iy) pixel (i, j) = image(ix*sp + i - Nx_left, ...), 0 outside."""
    Ny, Nx = img.shape
    nxv, nyv = geom["Nx_vec"][grid], geom["Ny_vec"][grid]
    xl, yl = geom["Nx_left"][grid], geom["Ny_left"][grid]
    pad = max(wsx, wsy) + max(xl, yl) + 4
    big = np.zeros((Ny + 2 * pad, Nx + 2 * pad), np.float64)
    big[pad:pad + Ny, pad:pad + Nx] = img
    out = np.empty((nyv * nxv, wsy, wsx))
    for iy in range(nyv):
        for ix in range(nxv):
            y0 = iy * spy - yl + pad
            x0 = ix * spx - xl + pad
            out[iy * nxv + ix] = big[y0:y0 + wsy, x0:x0 + wsx]
    return out


@pytest.mark.parametrize("shape,ws,thresh", [((200, 400), 40, 0.91), ((253, 317), 40, 0.91), ((128, 96), 16, 0.5)])
def test_mhe_bitexact(cuda, shape, ws, thresh):
    import torch

    rng = np.random.default_rng(3)
    s = P.synth_params(shape[1], shape[0], ppp=0.05, seed=5)
    img, _ = P.synth_pair(s)
    img = np.ascontiguousarray(img)
    img[:10, :10] = rng.integers(0, 256, (10, 10))
    want = O.mhe(img, ws, thresh)
    m = P.mhe_gpu()
    assert m.init(shape[1], shape[0], ws, thresh)
    d = torch.from_numpy(img).cuda()
    assert m.processsing(d)
    torch.cuda.synchronize()
    got = m.d_enhanced.cpu().numpy()
    m.freemem()
    assert np.array_equal(got, want)


@pytest.mark.parametrize("ws,sp", [(32, 16), (64, 32), (16, 8), (24, 12), (48, 24)])
def test_cc_planes_vs_fp64(cuda, ws, sp):
    s = P.synth_params(192, 160, ppp=0.05, a=2.4, b=-1.3, seed=21)
    f1, f2 = P.synth_pair(s)
    p = c0_params(N=192, ws=ws, sp=sp, Ny=160)
    with P.Engine(p) as e:
        e.set_images(f1, f2)
        e.prep()
        e.pass_grid1(0)
        nt = e.geom["Nt_vec"][0]
        got = e.cc_planes(0, 0, nt)
    w1 = gather_windows(f1, e.geom, 0, ws, ws, sp, sp)
    w2 = gather_windows(f2, e.geom, 0, ws, ws, sp, sp)
    for w in range(0, nt, max(1, nt // 40)):
        want = O.xcorr_plane(w1[w], w2[w])
        scale = max(want.max(), 1.0)
        assert np.abs(got[w] - want).max() <= 2e-6 * scale, f"window {w}"


@pytest.mark.parametrize("ws,sp,nps", [(32, 16, 4), (64, 32, 4), (24, 12, 6), (16, 8, 4)])
def test_peaks_on_engine_planes(cuda, ws, sp, nps):
    s = P.synth_params(256, 192, ppp=0.05, a=3.3, b=-1.7, seed=31)
    f1, f2 = P.synth_pair(s)
    p = c0_params(N=256, Ny=192, ws=ws, sp=sp, Npeak_save=nps)
    with P.Engine(p) as e:
        e.set_images(f1, f2)
        e.prep()
        e.pass_grid1(0)
        nt = e.geom["Nt_vec"][0]
        planes = e.cc_planes(0, 0, nt)
        _, _, dx, dy, v = e.field(0)
        cnt, idx, val = e.peaks(0)
    op = O.params_from(p)
    _, g = O.geometry(op)
    z = np.zeros(nt, np.float32)
    c = O.peaks_from_planes(planes, op, g, 0, z, z)
    ok = c.flags == 0
    assert ok.mean() > 0.9
    assert np.array_equal(cnt, c.count)
    assert np.array_equal(idx[ok], c.peak_index[ok])
    assert np.array_equal(val[ok], c.peak_value[ok])
    assert np.array_equal(v[ok], c.valid[ok])
    both = (v == 1) & (c.valid == 1) & ok[:, None]
    assert np.abs(dx[both] - c.dx[both]).max() < 1e-4
    assert np.abs(dy[both] - c.dy[both]).max() < 1e-4


def _smooth_field(nx, ny, seed):
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:ny, 0:nx]
    fx = (2.5 * np.sin(xx / 3.0 + rng.random()) + 0.3 * yy).astype(np.float32).ravel()
    fy = (-1.5 * np.cos(yy / 2.5 + rng.random()) + 0.2 * xx).astype(np.float32).ravel()
    return fx, fy


@pytest.mark.parametrize("ws,sp", [(32, 16), (64, 32), (32, 8)])
def test_deformation(cuda, ws, sp):
    s = P.synth_params(200, 150, ppp=0.05, seed=41)
    f1, f2 = P.synth_pair(s)
    p = c0_params(N=200, Ny=150, ws=ws, sp=sp, Npass1=2)
    op = O.params_from(p)
    _, g = O.geometry(op)
    fx, fy = _smooth_field(g.Nx_vec[0], g.Ny_vec[0], 1)
    with P.Engine(p) as e:
        e.set_images(f1, f2)
        e.prep()
        e.set_field(0, fx, fy, np.ones_like(fx, np.uint8))
        e.pass_grid1(1)
        got = e.deformed(0)
    want, oob = O.deform(f2, op, g, 0, fx, fy)
    assert oob == 0
    # the engine's FP32 bilinear sums contract into FMAs (as the reference's nvcc build
    # does); the oracle rounds every product: a few ulp of the sample position times the
    # image gradient (up to ~250 grey levels / px)
    d = np.abs(got - want)
    assert d.max() < 1e-2 and d.mean() < 1e-4


def test_upsampling(cuda):
    p = P.default_params(Nx=640, Ny=480, Npass1=1, Npass2=1)
    op = O.params_from(p)
    _, g = O.geometry(op)
    fx, fy = _smooth_field(g.Nx_vec[0], g.Ny_vec[0], 2)
    with P.Engine(p) as e:
        e.set_field(0, fx, fy, np.ones_like(fx, np.uint8))
        e.upsample()
        _, _, gx, gy, _ = e.field(3)
    wx, wy = O.upsample(op, g, fx, fy)
    assert np.abs(gx - wx).max() < 1e-5 and np.abs(gy - wy).max() < 1e-5


@pytest.mark.parametrize("wm,npm,wsm,nps_s,minn", [(5, 2, 3, 1, 5), (3, 1, 5, 2, 3), (7, 3, 3, 0, 8), (5, 0, 3, 1, 5),
                                                  (4, 2, 2, 1, 4)])
def test_validation_grid1_bitexact(cuda, wm, npm, wsm, nps_s, minn):
    """MedianFilter_Smoothing_p1 always fills holes (X/xcorr2d_multi_grid.cu:1514)."""
    nx, ny, nps = 37, 29, 4
    rng = np.random.default_rng(7 + wm + npm)
    base_x, base_y = _smooth_field(nx, ny, 3)
    dx = (base_x[:, None] + rng.normal(0, 0.2, (nx * ny, nps))).astype(np.float32)
    dy = (base_y[:, None] + rng.normal(0, 0.2, (nx * ny, nps))).astype(np.float32)
    out = rng.random((nx * ny, nps)) < 0.15
    dx[out] += rng.normal(0, 8, out.sum()).astype(np.float32)
    dy[out] -= rng.normal(0, 8, out.sum()).astype(np.float32)
    valid = (rng.random((nx * ny, nps)) > 0.1).astype(np.uint8)
    valid[200:260, :] = 0  # a hole that needs several fill iterations
    dx[valid == 0] = 0
    dy[valid == 0] = 0
    p = P.default_params(Nx=nx * 16 + 8, Ny=ny * 16 + 8, ws_x1=32, ws_y1=32, spacing_x1=16, spacing_y1=16,
                         Npass1=1, Npass2=0, wx1_median=wm, wy1_median=wm, wx1_smooth=wsm, wy1_smooth=wsm)
    with P.Engine(p) as e:
        assert e.geom["Nx_vec"][0] == nx and e.geom["Ny_vec"][0] == ny
        e.set_candidates(0, dx, dy, valid)
        e.validate_grid1(npm, minn, 2.0, 2.0, nps_s)
        _, _, gx, gy, gv = e.field(1)
    wx, wy, wv, iters = O.validate(dx, dy, valid, nx, ny, nps, wm, wm, wsm, wsm, npm, minn, 2.0, nps_s, 1)
    assert iters >= 2
    assert np.array_equal(gv, wv)
    assert np.array_equal(gx, wx) and np.array_equal(gy, wy)


@pytest.mark.parametrize("fill,smooth", [(0, 0), (1, 1), (0, 2)])
def test_validation_grid2_fill_switch(cuda, fill, smooth):
    nx, ny, nps = 41, 23, 4
    rng = np.random.default_rng(11 + fill)
    bx, by = _smooth_field(nx, ny, 4)
    dx = (bx[:, None] + rng.normal(0, 0.3, (nx * ny, nps))).astype(np.float32)
    dy = (by[:, None] + rng.normal(0, 0.3, (nx * ny, nps))).astype(np.float32)
    valid = (rng.random((nx * ny, nps)) > 0.2).astype(np.uint8)
    p = P.default_params(Nx=640, Ny=384, Npass1=1, Npass2=1, ws_x2=32, ws_y2=32, spacing_x2=16, spacing_y2=16)
    with P.Engine(p) as e:
        nx2, ny2 = e.geom["Nx_vec"][1], e.geom["Ny_vec"][1]
        nt = nx2 * ny2
        dx2 = np.resize(dx, (nt, nps))
        dy2 = np.resize(dy, (nt, nps))
        v2 = np.resize(valid, (nt, nps))
        e.set_candidates(1, dx2, dy2, v2)
        e.validate_grid2(2, 5, 2.0, 3.0, smooth, fill)
        _, _, gx, gy, gv = e.field(3)
    wx, wy, wv, _ = O.validate(dx2, dy2, v2, nx2, ny2, nps, 5, 5, 3, 3, 2, 5, 3.0, smooth, fill)
    assert np.array_equal(gv, wv)
    assert np.array_equal(gx, wx) and np.array_equal(gy, wy)
