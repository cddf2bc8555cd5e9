"""Windows whose frame-1 or frame-2 content is all zero (dark regions, zero padding at the
image edge, a masked area).

The reference transforms the two windows separately (cufftExecC2C on each,
X/xcorr2d_multi_grid.cu:1334-1341), so an all-zero window gives a spectrum of exact zeros
and a correlation plane of exact zeros: find_local_max_2d (:585) keeps no candidate (it
needs cc > 0), the count is 0 and every saved peak is invalid.  The engine transforms
f1 + i*f2 together; these tests check that it detects such windows and reproduces the
reference's result exactly, on every correlation path, and that their neighbours are
unaffected.
"""
import numpy as np
import pytest

import piv_b200 as P
from oracle import oracle as O
from oracle import ref as R
from parity_util import near_ties

pytestmark = pytest.mark.gpu

NX, NY = 512, 384


def _frames():
    f1, f2 = P.synth_pair(P.synth_params(NX, NY, ppp=0.05, field=P.PIV_FIELD_UNIFORM, a=2.3, b=-1.4, seed=61))
    f1 = f1.copy()
    f2 = f2.copy()
    f1[40:200, 60:230] = 0     # frame 1 dark
    f2[180:330, 300:470] = 0   # frame 2 dark
    f1[300:384, 0:120] = 0     # both dark
    f2[300:384, 0:120] = 0
    return f1, f2


def _params(ws):
    return P.default_params(Nx=NX, Ny=NY, ws_x1=ws, ws_y1=ws, spacing_x1=ws // 2, spacing_y1=ws // 2, Npass1=1,
                            Npass2=0, max_dispx_win_percent1=0.25, max_dispy_win_percent1=0.25)


def _dead_windows(f1, f2, geom, ws):
    nxv, nyv = geom["Nx_vec"][0], geom["Ny_vec"][0]
    xl, yl = geom["Nx_left"][0], geom["Ny_left"][0]
    pad = ws + max(xl, yl) + 4
    out = np.zeros(nxv * nyv, bool)
    for f in (f1, f2):
        big = np.zeros((NY + 2 * pad, NX + 2 * pad), np.uint8)
        big[pad:pad + NY, pad:pad + NX] = f
        for iy in range(nyv):
            for ix in range(nxv):
                y0, x0 = iy * (ws // 2) - yl + pad, ix * (ws // 2) - xl + pad
                out[iy * nxv + ix] |= not big[y0:y0 + ws, x0:x0 + ws].any()
    return out


PATHS = [("fused", None, P.PIV_XCORR_SIMT, "0"), ("fused variant 2", "2,0", P.PIV_XCORR_SIMT, "0"),
         ("generic", None, P.PIV_XCORR_SIMT, "1"), ("split-bf16 tc", None, P.PIV_XCORR_TC_SPLIT, "0"),
         ("split-fp16 tc", None, P.PIV_XCORR_TC_SPLIT_F16, "0")]


@pytest.mark.parametrize("ws", [16, 32, 64])
@pytest.mark.parametrize("name,variant,path,generic", PATHS, ids=[p[0] for p in PATHS])
def test_all_zero_windows_match_the_reference_rule(cuda, monkeypatch, ws, name, variant, path, generic):
    f1, f2 = _frames()
    p = _params(ws)
    if variant:
        monkeypatch.setenv("PIV_XCORR_VARIANT", variant)
    monkeypatch.setenv("PIV_XCORR_GENERIC", generic)
    with P.Engine(p) as e:
        if path != P.PIV_XCORR_SIMT:
            e.set_xcorr_path(0, path)
        e.set_images(f1, f2)
        e.prep()
        e.pass_grid1(0)
        e.synchronize()
        nt = e.geom["Nt_vec"][0]
        planes = e.cc_planes(0, 0, nt)
        cnt, idx, val = e.peaks(0)
        _, _, dx, dy, v = e.field(0)
        geom = dict(e.geom)
    dead = _dead_windows(f1, f2, geom, ws)
    assert dead.sum() >= 6, "the frames were meant to hold all-zero windows"
    assert (planes[dead] == 0).all()
    assert (cnt[dead] == 0).all() and (idx[dead] == -1).all() and (val[dead] == 0).all()
    assert (v[dead] == 0).all() and (dx[dead] == 0).all() and (dy[dead] == 0).all()
    # the rest against the FP64 oracle on the engine's own planes
    op = O.params_from(p)
    _, g = O.geometry(op)
    z = np.zeros(nt, np.float32)
    ref = O.correlate_grid(f1, f2, None, op, g, 0, z, z)
    assert (ref.count[dead] == 0).all()
    tie_top, tie_cnt = near_ties(planes, geom["border_x"][0], geom["border_y"][0], p.Npeak_save,
                                 rel=1e-5 if path == P.PIV_XCORR_SIMT else 1e-4)
    ok = ~tie_top & (ref.flags == 0)
    assert np.array_equal(idx[ok], ref.peak_index[ok])
    assert np.array_equal(cnt[~tie_cnt & (ref.flags == 0)], ref.count[~tie_cnt & (ref.flags == 0)])


def test_all_zero_windows_against_the_reference(cuda):
    if not R.available():
        pytest.skip("oracle/_ref/libref_xcorr2d.so was not built (make -C oracle ref)")
    f1, f2 = _frames()
    p = _params(32)
    g = P.geometry(p)
    nt = g["Nt_vec"][0]
    with R.RefEngine(p) as r:
        r.run_pair(f1, f2)
        rc, ri, rv = r.peaks(0, nt)
        _, _, rvalid = r.raw(0, nt)
    with P.Engine(p) as e:
        e.set_images(f1, f2)
        e.run_pair()
        cnt, idx, val = e.peaks(0)
        _, _, _, _, v = e.field(0)
    dead = _dead_windows(f1, f2, g, 32)
    assert (rc[dead] == 0).all() and (cnt[dead] == 0).all()
    assert np.array_equal(idx[dead], ri[dead]) and np.array_equal(v[dead], rvalid[dead])
