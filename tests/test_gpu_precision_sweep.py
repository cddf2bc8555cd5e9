"""Precision sweep of the correlation paths on the 6600x4400 workload's images.

The 6600x4400 pair (0.04 particles/px, Lamb-Oseen vortex of 10 px and 600 px core plus
0.002 shear, seed 1) goes through MHE on the engine; the sweep then runs one undeformed
pass over the central 1536x1024 crop (the vortex core and its shear) for the window shapes
16x16, 32x32, 48x24 and 64x64 at 50 % overlap, on every correlation path that covers the
shape:
  fp32 simt         register FFTs in FP32 (the fused kernels)
  fp32 generic      the generic-size kernel (shared-memory FFTs in FP32)
  split-bf16 tc     DFT products on tcgen05, BF16 hi + lo operands, FP32 accumulation
  bf16 tc           one BF16 product (about 8 significant bits per operand)
  split-fp16 tc     FP16 hi + lo operands (about 22 bits)
  fp16 tc           one FP16 product (11 bits)
Against the FP64 oracle (its own FFT and fit on the same windows) it reports the plane
error (of the window peak), the peak-index mismatch rate (all windows, and outside windows
the oracle flags or whose top maxima are near ties), and the main-peak displacement error
(max and RMS, px) where both sides find the same peak.  The FP32 and split paths hold the
parity bar: no index mismatch outside near ties, every main peak within the fit tolerance
of its plane error (1e-3 px plus the FP32 fit's propagated error: 16x16 windows against
this 10 px vortex leave many peaks flat, where the fit is ill-conditioned on every path;
the fraction within 1e-3 px is reported).  Run with -s to print the table.
"""
import numpy as np
import pytest

import piv_b200 as P
from oracle import oracle as O
from parity_util import fit_tolerance, near_ties

pytestmark = pytest.mark.gpu

NX, NY = 6600, 4400
CROP = (slice(1688, 2712), slice(2532, 4068))  # rows, cols: 1024 x 1536 around the vortex core
SHAPES = [(16, 16), (32, 32), (48, 24), (64, 64)]
PATHS = [("fp32 simt", P.PIV_XCORR_SIMT, False), ("fp32 generic", P.PIV_XCORR_SIMT, True),
         ("split-bf16 tc", P.PIV_XCORR_TC_SPLIT, False), ("bf16 tc", P.PIV_XCORR_TC_BF16, False),
         ("split-fp16 tc", P.PIV_XCORR_TC_SPLIT_F16, False), ("fp16 tc", P.PIV_XCORR_TC_F16, False)]
SPLIT_PLANE_REL = 2e-5  # plane error bound of the FP32 and split paths (of the window peak)


@pytest.fixture(scope="module")
def frames(cuda):
    p = P.default_params(Nx=NX, Ny=NY, if_mhe=1, mhe_ws=40, mhe_thresh=0.91, Npass1=1, Npass2=0)
    f1, f2 = P.synth_pair(P.synth_params(NX, NY, ppp=0.04, sigma=0.6, field=P.PIV_FIELD_VORTEX, a=10.0, b=600.0,
                                         c=0.002, seed=1))
    with P.Engine(p) as e:
        e.set_images(f1, f2)
        e.prep()
        m1, m2 = e.frames()
    return np.ascontiguousarray(m1[CROP]), np.ascontiguousarray(m2[CROP])


def _params(wx, wy):
    Ny, Nx = CROP[0].stop - CROP[0].start, CROP[1].stop - CROP[1].start
    return P.default_params(Nx=Nx, Ny=Ny, ws_x1=wx, ws_y1=wy, spacing_x1=wx // 2, spacing_y1=wy // 2, Npass1=1,
                            Npass2=0, max_dispx_win_percent1=0.25, max_dispy_win_percent1=0.25,
                            insert_threshold_p1=2.0)


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


def _run(p, f1, f2, path, generic, monkeypatch):
    monkeypatch.setenv("PIV_XCORR_GENERIC", "1" if generic else "0")
    with P.Engine(p) as e:
        if path != P.PIV_XCORR_SIMT:
            e.set_xcorr_path(0, path)
        e.set_images(f1, f2)
        e.prep()
        e.pass_grid1(0)
        e.synchronize()
        nt = e.geom["Nt_vec"][0]
        return e.cc_planes(0, 0, nt), e.peaks(0), e.field(0), dict(e.geom)


@pytest.mark.parametrize("wx,wy", SHAPES, ids=[f"{x}x{y}" for x, y in SHAPES])
def test_precision_sweep(frames, monkeypatch, wx, wy):
    f1, f2 = frames
    p = _params(wx, wy)
    op = O.params_from(p)
    _, og = O.geometry(op)
    nt = og.Nt_vec[0]
    z = np.zeros(nt, np.float32)
    ref = O.correlate_grid(f1, f2, None, op, og, 0, z, z)  # FP64 planes and fit
    rows = []
    for name, path, generic in PATHS:
        tc = path != P.PIV_XCORR_SIMT
        if tc and not ((wx == wy and wx in (16, 32, 64)) or (wx, wy) in ((48, 24), (24, 48))):
            rows.append((name, None))
            continue
        planes, (cnt, idx, val), (_, _, dx, dy, v), geom = _run(p, f1, f2, path, generic, monkeypatch)
        w1 = _windows(f1, geom, wx, wy)
        w2 = _windows(f2, geom, wx, wy)
        perr = 0.0
        for w in range(0, nt, max(1, nt // 50)):
            want = O.xcorr_plane(w1[w], w2[w])
            perr = max(perr, float(np.abs(planes[w] - want).max() / max(want.max(), 1.0)))
        tie_top, _ = near_ties(planes, geom["border_x"][0], geom["border_y"][0], p.Npeak_save, rel=max(1e-5, 4 * perr))
        clean = ~tie_top & (ref.flags == 0)
        mism = np.any(idx != ref.peak_index, axis=1)
        for w in np.nonzero(mism & clean)[0][:3]:
            print(f"\n  {name} window {w}: engine count {cnt[w]} idx {idx[w]} val {val[w]}; oracle count "
                  f"{ref.count[w]} idx {ref.peak_index[w]} val {ref.peak_value[w]} flags {ref.flags[w]}")
        main = (idx[:, 0] == ref.peak_index[:, 0]) & (v[:, 0] == 1) & (ref.valid[:, 0] == 1)
        d = np.maximum(np.abs(dx[:, 0] - ref.dx[:, 0]), np.abs(dy[:, 0] - ref.dy[:, 0]))
        # per-window plane error: the sampled maximum, with a margin of 4 for the windows not sampled
        tx, ty = fit_tolerance(planes, idx, wx, rel_cc=max(4 * perr, 1e-6))
        in_tol = (np.abs(dx - ref.dx)[:, 0] <= tx[:, 0]) & (np.abs(dy - ref.dy)[:, 0] <= ty[:, 0])
        for w in np.nonzero(main & clean & ~in_tol)[0][:3]:
            li = idx[w, 0]
            fl = planes[w].ravel()
            print(f"\n  {name} window {w}: idx {li} engine dx {dx[w, 0]} dy {dy[w, 0]} oracle dx {ref.dx[w, 0]} dy "
                  f"{ref.dy[w, 0]} tol {tx[w, 0]:.3g} {ty[w, 0]:.3g} plane {[fl[li + o] for o in (-wx, -1, 0, 1, wx)]}")
        rows.append((name, dict(plane=perr, mism_all=float(mism.mean()), mism_clean=float(mism[clean].mean()),
                                clean=float(clean.mean()), dmax=float(d[main].max()),
                                drms=float(np.sqrt(np.mean(d[main] ** 2))), within=float(np.mean(d[main] < 1e-3)),
                                in_tol=bool(in_tol[main & clean].all()))))
    print(f"\n{wx}x{wy} ({nt} windows): path, plane error, index mismatch all / outside near ties, "
          f"main-peak |d| max / RMS px, fraction within 1e-3 px")
    for name, r in rows:
        if r is None:
            print(f"  {name:14s} (no tensor-core kernel for this shape)")
            continue
        print(f"  {name:14s} {r['plane']:9.2e}  {r['mism_all']:8.4%} / {r['mism_clean']:8.4%}  "
              f"{r['dmax']:9.2e} / {r['drms']:9.2e}  {r['within']:8.4%}")
    for name, r in rows:
        if r is None:
            continue
        if name in ("fp32 simt", "fp32 generic", "split-bf16 tc", "split-fp16 tc"):
            assert r["plane"] <= SPLIT_PLANE_REL, (name, r)
            assert r["mism_clean"] == 0.0, (name, r)
            assert r["in_tol"], (name, r)
        else:
            assert r["plane"] < 0.05, (name, r)
