"""The tensor-core correlation kernel for non-square windows (48x24, 24x48; csrc/xcorr_tc_rect.cuh)
against the FP64 oracle and the FP32 kernels.

  correlation planes        split-BF16 and split-FP16 DFT products vs the FP64 FFT: 2e-5 of
                            the window peak (undeformed pass), and vs the FP32 kernel on the
                            deformed pass
  peak search               the oracle's on the engine's own planes: counts, indices, values and
                            validity bit-exact (oracle-flagged windows excluded), displacements
                            within the FP32-log fit bound
  against the FP32 kernel   peak indices exact outside near ties, displacements within the fit
                            tolerance of the planes' difference
Single products (BF16, FP16) are reported by the precision sweep, not held here.
"""
import numpy as np
import pytest

import piv_b200 as P
from oracle import oracle as O
from parity_util import fit_tolerance, near_ties

pytestmark = pytest.mark.gpu

SHAPES = [(48, 24), (24, 48)]
PATHS = [("split-bf16", P.PIV_XCORR_TC_SPLIT), ("split-fp16", P.PIV_XCORR_TC_SPLIT_F16)]


def _params(wx, wy, Nx=432, Ny=360):
    return P.default_params(Nx=Nx, Ny=Ny, ws_x1=wx, ws_y1=wy, spacing_x1=wx // 2, spacing_y1=wy // 2, Npass1=2,
                            Npass2=0, max_dispx_win_percent1=0.25, max_dispy_win_percent1=0.25)


def _frames(Nx, Ny, seed):
    return P.synth_pair(P.synth_params(Nx, Ny, ppp=0.05, field=P.PIV_FIELD_FOURIER, a=150.0, b=900.0, c=4.0,
                                       seed=seed))


def _windows(img, geom, wx, wy):
    Ny, Nx = img.shape
    nxv, nyv = geom["Nx_vec"][0], geom["Ny_vec"][0]
    xl, yl = geom["Nx_left"][0], geom["Ny_left"][0]
    pad = max(wx, wy) + max(xl, yl) + 4
    big = np.zeros((Ny + 2 * pad, Nx + 2 * pad), np.float64)
    big[pad:pad + Ny, pad:pad + Nx] = img
    out = np.empty((nyv * nxv, wy, wx))
    for iy in range(nyv):
        for ix in range(nxv):
            y0, x0 = iy * (wy // 2) - yl + pad, ix * (wx // 2) - xl + pad
            out[iy * nxv + ix] = big[y0:y0 + wy, x0:x0 + wx]
    return out


def _run(p, f1, f2, path, field=None):
    with P.Engine(p) as e:
        if path != P.PIV_XCORR_SIMT:
            e.set_xcorr_path(0, path)
        e.set_images(f1, f2)
        e.prep()
        nt = e.geom["Nt_vec"][0]
        out = []
        for j in (0, 1):
            if j == 1:
                e.set_field(0, field[0], field[1], np.ones(nt, np.uint8))
            e.pass_grid1(j)
            e.synchronize()
            out.append((e.cc_planes(0, 0, nt), e.peaks(0), e.field(0)))
        return out, dict(e.geom)


@pytest.mark.parametrize("wx,wy", SHAPES, ids=[f"{x}x{y}" for x, y in SHAPES])
@pytest.mark.parametrize("name,path", PATHS, ids=[n for n, _ in PATHS])
def test_rect_tc_against_fp64_and_fp32(cuda, wx, wy, name, path):
    p = _params(wx, wy)
    f1, f2 = _frames(p.Nx, p.Ny, seed=11 + wx)
    g = P.geometry(p)
    yy, xx = np.mgrid[0:g["Ny_vec"][0], 0:g["Nx_vec"][0]]
    field = ((1.5 * np.sin(xx / 3.0) + 0.05 * yy).astype(np.float32).ravel(),
             (-1.0 * np.cos(yy / 2.5)).astype(np.float32).ravel())
    (tc0, tc1), geom = _run(p, f1, f2, path, field)
    (s0, s1), _ = _run(p, f1, f2, P.PIV_XCORR_SIMT, field)
    nt = geom["Nt_vec"][0]
    # undeformed pass: planes against the FP64 FFT
    planes, (cnt, idx, val), (_, _, dx, dy, v) = tc0
    w1, w2 = _windows(f1, geom, wx, wy), _windows(f2, geom, wx, wy)
    worst = 0.0
    for w in range(0, nt, max(1, nt // 40)):
        want = O.xcorr_plane(w1[w], w2[w])
        worst = max(worst, float(np.abs(planes[w] - want).max() / max(want.max(), 1.0)))
    print(f"\n{name} tc {wx}x{wy}: plane error {worst:.2e} of the window peak")
    assert worst <= 2e-5
    # the oracle's peak search on these planes
    op = O.params_from(p)
    _, og = O.geometry(op)
    z = np.zeros(nt, np.float32)
    c = O.peaks_from_planes(planes, op, og, 0, z, z)
    ok = c.flags == 0
    assert ok.mean() > 0.8
    assert np.array_equal(cnt, c.count) and np.array_equal(idx[ok], c.peak_index[ok])
    assert np.array_equal(val[ok], c.peak_value[ok]) and np.array_equal(v[ok], c.valid[ok])
    both = (v == 1) & (c.valid == 1) & ok[:, None]
    tx, ty = fit_tolerance(planes, idx, wx, rel_cc=0.0, base=1e-5, safety=2.0)
    assert (np.abs(dx - c.dx)[both] <= tx[both]).all() and (np.abs(dy - c.dy)[both] <= ty[both]).all()
    # both passes against the FP32 kernel
    for (pa, (ca, ia, _), (_, _, dxa, dya, va)), (pb, (cb, ib, _), (_, _, dxb, dyb, vb)) in ((s0, tc0), (s1, tc1)):
        peak = np.maximum(pa.reshape(nt, -1).max(1), 1e-30)
        err = float((np.abs(pa - pb).reshape(nt, -1).max(1) / peak).max())
        assert err <= 2e-5, err
        tie_top, _ = near_ties(pa, geom["border_x"][0], geom["border_y"][0], p.Npeak_save, rel=1e-4)
        assert np.array_equal(ia[~tie_top], ib[~tie_top])
        same = (ia == ib) & (va == 1) & (vb == 1) & ~tie_top[:, None]
        tx, ty = fit_tolerance(pa, ia, wx, rel_cc=2e-5)
        assert (np.abs(dxa - dxb)[same] <= tx[same]).all() and (np.abs(dya - dyb)[same] <= ty[same]).all()
