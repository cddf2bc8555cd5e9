"""Large frames: 16384 x 12288 pixels (201 M pixels a frame, 0.8 GB for each FP32 deformed frame),
where every offset of the far corner of the frames and of the window grid is large.

  far-corner windows    the correlation planes of the last windows of the grid (and of a block
                        in the middle) within 2e-6 of the window peak of the FP64 oracle's planes
                        of the same pixels; peak counts, indices, values and validity bit-exact
                        against the oracle's peak search on the engine's planes
  whole multigrid pair  MHE, 64 -> 32 px, 2 + 3 passes: the filtered field against the
                        generator's known displacement (a size-independent property): at least
                        99 % valid vectors, interior RMS error under 0.06 px
"""
import numpy as np
import pytest

import piv_b200 as P
from oracle import oracle as O

pytestmark = pytest.mark.gpu

NX, NY = 16384, 12288


def _device_pair(s):
    import torch

    d1 = torch.empty((s.Ny, s.Nx), dtype=torch.uint8, device="cuda")
    d2 = torch.empty_like(d1)
    scratch = torch.empty(2 * s.Nx * s.Ny, dtype=torch.float32, device="cuda")
    P.synth_pair_device(s, d1, d2, scratch)
    torch.cuda.synchronize()
    del scratch
    return d1, d2


def _window(img, geom, w, ws, sp):
    """Window w of grid 1 from the frame, zero outside it (the padded frame's margins)."""
    nxv = geom["Nx_vec"][0]
    iy, ix = divmod(int(w), nxv)
    x0, y0 = ix * sp - geom["Nx_left"][0], iy * sp - geom["Ny_left"][0]
    out = np.zeros((ws, ws), np.float64)
    ya, yb = max(y0, 0), min(y0 + ws, img.shape[0])
    xa, xb = max(x0, 0), min(x0 + ws, img.shape[1])
    if ya < yb and xa < xb:
        out[ya - y0:yb - y0, xa - x0:xb - x0] = img[ya:yb, xa:xb]
    return out


def test_far_corner_windows_against_fp64(cuda):
    import torch

    s = P.synth_params(NX, NY, ppp=0.04, sigma=0.6, field=P.PIV_FIELD_FOURIER, a=150.0, b=900.0, c=4.0, seed=7)
    d1, d2 = _device_pair(s)
    f1, f2 = d1.cpu().numpy(), d2.cpu().numpy()
    ws, sp = 64, 32
    p = P.default_params(Nx=NX, Ny=NY, if_mhe=0, ws_x1=ws, ws_y1=ws, spacing_x1=sp, spacing_y1=sp, Npass1=1,
                         Npass2=0, max_dispx_win_percent1=0.25, max_dispy_win_percent1=0.25)
    with P.Engine(p) as e:
        e.set_device_images(d1.data_ptr(), d2.data_ptr())
        e.prep()
        e.pass_grid1(0)
        e.synchronize()
        geom = dict(e.geom)
        nt = geom["Nt_vec"][0]
        cnt, idx, val = e.peaks(0)
        _, _, dx, dy, v = e.field(0)
        op = O.params_from(p)
        for first in (nt - 40, nt // 2 - 20):
            n = 40
            planes = e.cc_planes(0, first, n)
            worst = 0.0
            for k in range(n):
                want = O.xcorr_plane(_window(f1, geom, first + k, ws, sp), _window(f2, geom, first + k, ws, sp))
                worst = max(worst, float(np.abs(planes[k] - want).max() / max(want.max(), 1.0)))
            assert worst <= 2e-6, f"windows {first}..{first + n}: {worst:.2e} of the window peak"
            # the oracle's peak search on the same planes (a sub-geometry of these n windows)
            _, og = O.geometry(op)
            og.Nt_vec[0] = n
            z = np.zeros(n, np.float32)
            c = O.peaks_from_planes(planes, op, og, 0, z, z)
            ok = c.flags == 0
            sl = slice(first, first + n)
            assert ok.mean() > 0.8
            assert np.array_equal(cnt[sl], c.count)
            assert np.array_equal(idx[sl][ok], c.peak_index[ok]) and np.array_equal(val[sl][ok], c.peak_value[ok])
            assert np.array_equal(v[sl][ok], c.valid[ok])
    del d1, d2
    torch.cuda.empty_cache()


def test_whole_pair_accuracy(cuda):
    import torch

    s = P.synth_params(NX, NY, ppp=0.04, sigma=0.6, field=P.PIV_FIELD_VORTEX, a=10.0, b=1500.0, c=0.002, seed=5)
    d1, d2 = _device_pair(s)
    p = P.default_params(Nx=NX, Ny=NY, if_mhe=1, mhe_ws=40, mhe_thresh=0.91, ws_x1=64, ws_y1=64, spacing_x1=32,
                         spacing_y1=32, Npass1=2, ws_x2=32, ws_y2=32, spacing_x2=16, spacing_y2=16, Npass2=3,
                         insert_threshold_p1=2.0, insert_threshold_p2=2.0)
    with P.Engine(p) as e:
        e.set_device_images(d1.data_ptr(), d2.data_ptr())
        e.run_pair()
        e.synchronize()
        x, y, dx, dy, v = e.field(3)
        assert x.size == e.geom["Nt_vec"][1] > 700000
    assert np.isfinite(dx).all() and np.isfinite(dy).all()
    u, w = P.synth_field(s, x, y)
    ok = v == 1
    inner = ok & (x > 32) & (x < NX - 32) & (y > 32) & (y < NY - 32)
    rms = float(np.sqrt(np.mean((dx - u)[inner] ** 2 + (dy - w)[inner] ** 2)))
    print(f"\n{NX}x{NY}: {x.size} vectors, valid {ok.mean():.4%}, interior RMS {rms:.4f} px")
    assert ok.mean() >= 0.99
    assert rms <= 0.06
    del d1, d2
    torch.cuda.empty_cache()
