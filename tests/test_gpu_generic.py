"""Every window shape and peak count the reference's parameter file allows.

The reference accepts ws_x, ws_y multiples of 4 from 4 to 1024 and any Npeak_save
(X/xcorr2d_multi_grid.cu:896-920; cuFFT plans any size).  Shapes without a fused
register-FFT instance (8..64 px) and Npeak_save > 8 run on the generic-size kernel
(csrc/xcorr_generic.cu): mixed radix 4/2/3/5/7 plus any prime (44 = 4*11, 148 = 4*37),
planes above 20,480 points in a global workspace (256x256, 148x148).  Checked against:
  - the FP64 oracle: correlation planes within 3e-6 of the window peak;
  - the oracle's peak search on the engine's own planes: counts, peak indices, values and
    validity bit-exact (windows the oracle flags for exact value ties or slot overflow
    excluded), displacements within the propagated FP32-log bound of the fit (1e-5 px plus
    twice the numerator's rounding over the denominator: flat peaks amplify it);
  - the fused kernels (PIV_XCORR_GENERIC=1 forces the generic kernel): planes within 2e-6
    of the peak, peak indices exact outside near ties, displacements within the fit bound
    for planes that agree to 2e-6;
  - the reference engine itself (oracle/_ref): peak indices exact outside slot overflow and
    near ties, validity exact where the fit reads no value within the plane error of zero,
    raw displacements within the fit tolerance, on a pass staged with the reference's own
    predictor.
"""
import numpy as np
import pytest

import piv_b200 as P
from oracle import oracle as O
from oracle import ref as R
from parity_util import fit_tolerance, fit_undetermined, near_ties

pytestmark = pytest.mark.gpu

# (ws_x, ws_y, spacing_x, spacing_y, image Nx, Ny)
SHAPES = [(40, 40, 20, 20, 320, 240), (20, 28, 10, 14, 200, 168), (44, 44, 22, 22, 264, 220),
          (96, 96, 48, 48, 480, 384), (128, 64, 64, 32, 512, 320), (128, 128, 64, 64, 512, 448),
          (36, 60, 18, 30, 288, 300), (148, 148, 74, 74, 520, 444), (256, 256, 128, 128, 768, 640)]


def _params(wx, wy, sx, sy, Nx, Ny, nps=4, npass=1, **kw):
    return P.default_params(Nx=Nx, Ny=Ny, ws_x1=wx, ws_y1=wy, spacing_x1=sx, spacing_y1=sy, Npass1=npass, Npass2=0,
                            Npeak_save=nps, max_dispx_win_percent1=0.25, max_dispy_win_percent1=0.25,
                            insert_threshold_p1=2.0, **kw)


def _frames(Nx, Ny, seed):
    return P.synth_pair(P.synth_params(Nx, Ny, ppp=0.04, field=P.PIV_FIELD_FOURIER, a=150.0, b=900.0, c=5.0,
                                       seed=seed))


def _windows(img, geom, wsx, wsy, spx, spy):
    Ny, Nx = img.shape
    nxv, nyv = geom["Nx_vec"][0], geom["Ny_vec"][0]
    xl, yl = geom["Nx_left"][0], geom["Ny_left"][0]
    pad = max(wsx, wsy) + max(xl, yl) + 4
    big = np.zeros((Ny + 2 * pad, Nx + 2 * pad), np.float64)
    big[pad:pad + Ny, pad:pad + Nx] = img
    out = np.empty((nyv * nxv, wsy, wsx))
    for iy in range(nyv):
        for ix in range(nxv):
            y0, x0 = iy * spy - yl + pad, ix * spx - xl + pad
            out[iy * nxv + ix] = big[y0:y0 + wsy, x0:x0 + wsx]
    return out


@pytest.mark.parametrize("shape", SHAPES, ids=[f"{s[0]}x{s[1]}" for s in SHAPES])
@pytest.mark.parametrize("nps", [4, 10])
def test_generic_planes_and_peaks_vs_oracle(cuda, shape, nps):
    wx, wy, sx, sy, Nx, Ny = shape
    f1, f2 = _frames(Nx, Ny, seed=wx * 7 + wy)
    p = _params(wx, wy, sx, sy, Nx, Ny, nps=nps)
    with P.Engine(p) as e:
        assert e.xcorr_config(0)[:2] == (1, 256), "expected the generic-size kernel"
        e.set_images(f1, f2)
        e.prep()
        e.pass_grid1(0)
        e.synchronize()
        nt = e.geom["Nt_vec"][0]
        planes = e.cc_planes(0, 0, nt)
        _, _, dx, dy, v = e.field(0)
        cnt, idx, val = e.peaks(0)
        geom = e.geom
    w1 = _windows(f1, geom, wx, wy, sx, sy)
    w2 = _windows(f2, geom, wx, wy, sx, sy)
    for w in range(0, nt, max(1, nt // 12)):
        want = O.xcorr_plane(w1[w], w2[w])
        assert np.abs(planes[w] - want).max() <= 3e-6 * max(want.max(), 1.0), f"window {w}"
    op = O.params_from(p)
    _, g = O.geometry(op)
    z = np.zeros(nt, np.float32)
    c = O.peaks_from_planes(planes, op, g, 0, z, z)
    ok = c.flags == 0
    assert ok.mean() > 0.8
    assert np.array_equal(cnt, c.count)
    assert np.array_equal(idx[ok], c.peak_index[ok])
    assert np.array_equal(val[ok], c.peak_value[ok])
    assert np.array_equal(v[ok], c.valid[ok])
    both = (v == 1) & (c.valid == 1) & ok[:, None]
    assert both[:, 0].mean() > 0.5
    # same planes, FP32 log numerator against the oracle's FP64 fit
    tx, ty = fit_tolerance(planes, idx, wx, rel_cc=0.0, base=1e-5, safety=2.0)
    assert (np.abs(dx - c.dx)[both] <= tx[both]).all() and (np.abs(dy - c.dy)[both] <= ty[both]).all()


@pytest.mark.parametrize("wx,wy", [(32, 32), (64, 64), (48, 24), (16, 16)])
def test_generic_matches_fused_kernels(cuda, monkeypatch, wx, wy):
    Nx, Ny = 448, 352
    f1, f2 = _frames(Nx, Ny, seed=41 + wx)
    p = _params(wx, wy, wx // 2, wy // 2, Nx, Ny, npass=2)
    g = P.geometry(p)
    yy, xx = np.mgrid[0:g["Ny_vec"][0], 0:g["Nx_vec"][0]]
    sfx = (2.0 * np.sin(xx / 4.0) + 0.1 * yy).astype(np.float32).ravel()
    sfy = (-1.5 * np.cos(yy / 3.0)).astype(np.float32).ravel()
    out = {}
    for forced in ("0", "1"):
        monkeypatch.setenv("PIV_XCORR_GENERIC", forced)
        with P.Engine(p) as e:
            assert (e.xcorr_config(0)[:2] == (1, 256)) == (forced == "1")
            e.set_images(f1, f2)
            e.prep()
            nt = e.geom["Nt_vec"][0]
            res = []
            for j in (0, 1):  # undeformed, then deformed by the same field on both sides
                if j == 1:
                    e.set_field(0, sfx, sfy, np.ones(nt, np.uint8))
                e.pass_grid1(j)
                e.synchronize()
                res.append((e.cc_planes(0, 0, nt), e.peaks(0), e.field(0)))
            out[forced] = res
    for j in (0, 1):
        (pa, (ca, ia, _), (_, _, dxa, dya, vva)), (pb, (cb, ib, _), (_, _, dxb, dyb, vvb)) = out["0"][j], out["1"][j]
        peak = np.maximum(pa.reshape(len(pa), -1).max(1), 1e-30)
        err = np.abs(pa - pb).reshape(len(pa), -1).max(1) / peak
        assert err.max() <= 2e-6, (j, err.max())
        tie_top, tie_cnt = near_ties(pa, g["border_x"][0], g["border_y"][0], p.Npeak_save)
        ok = ~tie_top
        assert np.array_equal(ia[ok], ib[ok]), j
        assert np.array_equal(ca[~tie_cnt], cb[~tie_cnt]), j
        both = (vva == 1) & (vvb == 1) & (ia == ib) & ok[:, None]
        tx, ty = fit_tolerance(pa, ia, wx, rel_cc=2e-6, base=1e-5, safety=2.0)
        assert (np.abs(dxa - dxb)[both] <= tx[both]).all() and (np.abs(dya - dyb)[both] <= ty[both]).all(), j


@pytest.mark.parametrize("wx,wy,nps", [(40, 40, 10), (128, 128, 4), (44, 20, 6), (32, 32, 12)])
def test_generic_against_reference(cuda, wx, wy, nps):
    if not R.available():
        pytest.skip("oracle/_ref/libref_xcorr2d.so was not built (make -C oracle ref)")
    Nx, Ny = 832, 704
    f1, f2 = _frames(Nx, Ny, seed=77 + wx + nps)
    p = _params(wx, wy, wx // 2, wy // 2, Nx, Ny, nps=nps, npass=2, if_mhe=1)
    g = P.geometry(p)
    nt = g["Nt_vec"][0]
    with R.RefEngine(p) as r:
        rec = r.run_pair_recording(f1, f2, nt, g["Nt_vec"][1])
        rc, ri, rv = r.peaks(0, nt)
        rdx, rdy, rvalid = r.raw(0, nt)
        rpl = r.cc(0, 0, nt, wx, wy)
    with P.Engine(p) as e:
        e.set_images(f1, f2)
        e.prep()
        e.pass_grid1(0)
        e.validate_grid1()
        e.set_field(0, rec["p1x"], rec["p1y"], np.ones(nt, np.uint8))  # the reference's own predictor
        e.pass_grid1(1)
        e.synchronize()
        planes = e.cc_planes(0, 0, nt)
        cnt, idx, val = e.peaks(0)
        _, _, dx, dy, v = e.field(0)
    err = np.abs(planes - rpl).reshape(nt, -1).max(1) / rpl.reshape(nt, -1).max(1)
    assert err.max() <= 1e-6, f"plane error {err.max():.2e} of the peak"
    tie_top, _ = near_ties(planes, g["border_x"][0], g["border_y"][0], nps)
    overflow = (cnt > g["Npeak"][0]) | (rc > g["Npeak"][0])
    ok = ~tie_top & ~overflow
    print(f"\n{wx}x{wy} Npeak_save {nps}: {nt} windows, overflow {overflow.mean():.2%}, near ties "
          f"{tie_top.mean():.2%}")
    assert ok.mean() > 0.5
    assert np.array_equal(idx[ok], ri[ok])
    same = (idx == ri) & ok[:, None] & ~fit_undetermined(planes, idx, wx)
    for w, q in zip(*np.nonzero(same & (v != rvalid))):
        li = idx[w, q]
        fl = planes[w].ravel()
        nb = [fl[li + o] if 0 <= li + o < fl.size else None for o in (-1, 1, -wx, wx)]
        print(f"  window {w} peak {q} idx {li}: engine valid {v[w, q]} dx {dx[w, q]} dy {dy[w, q]} val {val[w, q]}; "
              f"reference valid {rvalid[w, q]} dx {rdx[w, q]} dy {rdy[w, q]} val {rv[w, q]}; neighbours {nb}")
    assert np.array_equal(v[same], rvalid[same])
    both = same & (v == 1)
    tx, ty = fit_tolerance(planes, idx, wx)
    assert (np.abs(dx - rdx)[both] <= tx[both]).all() and (np.abs(dy - rdy)[both] <= ty[both]).all()
