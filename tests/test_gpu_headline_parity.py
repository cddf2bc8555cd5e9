"""Parity with the reference engine itself at the 6600x4400 multigrid workload.

The reference (xcorr2d_multi + mhe_gpu, compiled for sm_100a from its own sources by
`make -C oracle ref`, oracle/_ref/) and the engine run the same seeded pair: 6600x4400,
MHE 40 px / 0.91, grid 1 64x64 windows at 32 px for 2 passes, grid 2 32x32 at 16 px for 3
passes (X/main.cpp:288-326 drives the reference; X/xcorr2d_multi_grid.cu:1620-1764 is its
grid-2 pass).

Where the reference is not reproducible, by anyone: find_local_max_2d
(X/xcorr2d_multi_grid.cu:585) stores a window's local maxima in Npeak = ws_x*ws_y/16 slots
at min(atomicAdd(count), Npeak - 1), so in a window with more maxima than slots the late
ones overwrite the last slot in the order the atomics land, and the reference can lose its
own main peak.  With MHE on, 12-15 % of this workload's windows overflow; the reference
then disagrees with itself from run to run (measured on a B200: 96 % of its raw peak lists
and 89-92 % of its filtered vectors within 1e-3 px repeat).  The engine takes the top
Npeak_save of ALL maxima, deterministically.

Checks:
  - MHE frames: bit-exact;
  - the last pass of each grid, staged with the reference's own predictor and deformation
    field (the filtered field that pass starts from): correlation planes within 1e-6 of the
    window peak; peak indices bit-exact in every window that neither overflows (either
    engine's count > Npeak) nor holds a near tie of its top Npeak_save+1 maxima (1e-5 relative);
    candidate counts bit-exact outside windows with a 4-neighbour comparison within 2e-6 of
    the peak; raw displacements within the fit tolerance (1e-3 px plus the reference's FP32
    log error); main peaks within 1e-3 px;
  - validation on identical candidates, in both directions: the engine's median test, fill
    and smoothing on the reference's candidates, and the reference's on the engine's,
    give exactly the other's validity flags and replacement choices (the median-only
    output is bit-exact; smoothed values agree to 1e-5 px, the reference sums in atomic
    order);
  - end to end (no staging): the engine's filtered fields agree with a reference run at
    least as well as two reference runs agree with each other.
Run with -s to print the fractions.
"""
import numpy as np
import pytest

import piv_b200 as P
from oracle import ref as R
from parity_util import fit_tolerance, fit_undetermined, near_ties

pytestmark = pytest.mark.gpu

NX, NY = 6600, 4400


def _params():
    return P.default_params(Nx=NX, Ny=NY, if_mhe=1, mhe_ws=40, mhe_thresh=0.91, ws_x1=64, ws_y1=64, spacing_x1=32,
                            spacing_y1=32, Npass1=2, ws_x2=32, ws_y2=32, spacing_x2=16, spacing_y2=16, Npass2=3,
                            Nsec_cc=1, insert_threshold_p1=2.0, insert_threshold_p2=2.0)


@pytest.fixture(scope="module")
def run(cuda):
    if not R.available():
        pytest.skip("oracle/_ref/libref_xcorr2d.so was not built (make -C oracle ref)")
    p = _params()
    f1, f2 = P.synth_pair(P.synth_params(NX, NY, ppp=0.04, sigma=0.6, field=P.PIV_FIELD_VORTEX, a=10.0, b=600.0,
                                         c=0.002, seed=1))
    g = P.geometry(p)
    nt = g["Nt_vec"]
    # grid 1 from a reference run without grid 2 (its correlation buffer then still holds
    # grid 1's planes); the reference is not reproducible from run to run (slot overflow), so
    # the planes, candidates and the predictor the engine is staged with come from one run
    p1 = _params()
    p1.Npass2 = 0
    ref = {}
    with R.RefEngine(p1) as r1:
        ref["pred1"] = r1.run_pair_recording(f1, f2, nt[0], nt[1])
        ref["planes0"] = r1.cc(0, 0, nt[0], p.ws_x1, p.ws_y1)
        ref["raw0"] = r1.raw(0, nt[0])
        ref["peaks0"] = r1.peaks(0, nt[0])
        ref["filt0"] = r1.filtered(0, nt[0])
    r = R.RefEngine(p)
    ref["mhe"] = (r.mhe(f1), r.mhe(f2))
    r.run_pair(f1, f2)
    ref["again"] = [r.filtered(k, nt[k]) for k in (0, 1)]  # a second full run, for self-agreement
    ref["pred"] = r.run_pair_recording(f1, f2, nt[0], nt[1])
    ref["e2e"] = [r.filtered(k, nt[k]) for k in (0, 1)]
    ref["planes1"] = r.cc(1, 0, nt[1], p.ws_x2, p.ws_y2)
    ref["raw1"] = r.raw(1, nt[1])
    ref["peaks1"] = r.peaks(1, nt[1])
    ref["filt1"] = r.filtered(1, nt[1])
    r.median_only()  # X/main.cpp:363
    ref["median1"] = r.filtered(1, nt[1])

    # the engine, staged: each grid's last pass starts from the reference's filtered field
    e = P.Engine(p)
    e.set_images(f1, f2)
    e.prep()
    for j in range(p.Npass1):
        if j == p.Npass1 - 1:
            e.set_field(0, ref["pred1"]["p1x"], ref["pred1"]["p1y"], np.ones(nt[0], np.uint8))
        e.pass_grid1(j)
        e.validate_grid1()
    e.upsample()
    for j in range(p.Npass2):
        if j == p.Npass2 - 1:
            e.set_field(1, ref["pred"]["p2x"], ref["pred"]["p2y"], np.ones(nt[1], np.uint8))
        e.pass_grid2()
        e.validate_grid2(iffill=1)
    e.synchronize()
    yield p, g, f1, f2, r, ref, e
    e.close()
    r.close()


def test_mhe_frames_bitexact(run):
    p, g, f1, f2, r, ref, e = run
    m1, m2 = e.frames()
    assert np.array_equal(m1, ref["mhe"][0]) and np.array_equal(m2, ref["mhe"][1])


@pytest.mark.parametrize("k", [0, 1])
def test_last_pass_peaks_and_candidates(run, k):
    p, g, f1, f2, r, ref, e = run
    nt, wsx = g["Nt_vec"][k], (p.ws_x1, p.ws_x2)[k]
    planes = e.cc_planes(k, 0, nt)
    rpl = ref[f"planes{k}"]
    err = np.abs(planes - rpl).reshape(nt, -1).max(1) / rpl.reshape(nt, -1).max(1)
    assert err.max() <= 1e-6, f"grid {k + 1}: plane error {err.max():.2e} of the peak"
    tie_top, _ = near_ties(planes, g["border_x"][k], g["border_y"][k], p.Npeak_save, rel=1e-5)
    _, tie_cnt = near_ties(planes, g["border_x"][k], g["border_y"][k], p.Npeak_save, rel=2e-6)
    cnt, idx, val = e.peaks(k)
    rc, ri, rv = ref[f"peaks{k}"]
    _, _, dx, dy, v = e.field(2 * k)
    rdx, rdy, rvalid = ref[f"raw{k}"]
    # overflow in either engine's count (the two counts differ only where a 4-neighbour
    # comparison is a near tie, which can move a window across the slot limit)
    overflow = (cnt > g["Npeak"][k]) | (rc > g["Npeak"][k])
    ok = ~tie_top & ~overflow
    differ = (idx != ri).any(1)
    print(f"\ngrid {k + 1}: {nt} windows; plane error max {err.max():.2e} of the peak; slot overflow in the "
          f"reference {overflow.mean():.3%}; near-tie top-{p.Npeak_save + 1} {tie_top.mean():.3%}; "
          f"compared {ok.mean():.3%}; peak lists differing: {differ[overflow].sum()} overflow, "
          f"{differ[tie_top & ~overflow].sum()} near-tie, {differ[ok].sum()} other")
    for w in np.nonzero(differ & ok)[0][:5]:
        print(f"  window {w}: engine count {cnt[w]} idx {idx[w]} val {val[w]}; reference count {rc[w]} idx {ri[w]} "
              f"val {rv[w]}")
    assert ok.mean() > 0.8
    assert np.array_equal(idx[ok], ri[ok]), f"grid {k + 1}: {differ[ok].sum()} windows differ"
    okc = ~tie_cnt
    print(f"grid {k + 1}: counts compared in {okc.mean():.3%} of windows")
    assert np.array_equal(cnt[okc], rc[okc])
    same = (idx == ri) & ok[:, None] & ~fit_undetermined(planes, idx, wsx)
    assert np.array_equal(v[same], rvalid[same])
    both = same & (v == 1)
    tx, ty = fit_tolerance(planes, idx, wsx)
    del planes
    ex, ey = np.abs(dx - rdx), np.abs(dy - rdy)
    assert (ex[both] <= tx[both]).all() and (ey[both] <= ty[both]).all()
    d0 = np.maximum(ex, ey)[:, 0][both[:, 0]]
    print(f"grid {k + 1}: main peaks within 1e-3 px of the reference: {(d0 < 1e-3).mean():.5%}, "
          f"median |d| {np.median(d0):.2e}, max {d0.max():.2e} px")
    assert (d0 < 1e-3).mean() >= 0.999
    assert np.abs(val[same] - rv[same]).max() <= 1e-5 * np.abs(val).max()


def _engine_validates(e, p, k, dx, dy, valid, smooth=True, fill=1):
    e.set_candidates(k, dx, dy, valid)
    if k == 0:
        e.validate_grid1()
    elif smooth:
        e.validate_grid2(iffill=fill)
    else:
        e.validate_grid2(p.Npass2_median, p.minNneigh_p2, p.residual_threshold_p2, p.insert_threshold_p2, 0, 0)
    return e.field(2 * k + 1)[2:]


@pytest.mark.parametrize("k", [0, 1])
def test_engine_validation_of_reference_candidates(run, k):
    p, g, f1, f2, r, ref, e = run
    fx, fy, fv = _engine_validates(e, p, k, *ref[f"raw{k}"])
    rx, ry, rv = ref[f"filt{k}"]
    assert np.array_equal(fv, rv), f"grid {k + 1}: {(fv != rv).sum()} validity flags differ"
    d = np.maximum(np.abs(fx - rx), np.abs(fy - ry))
    assert d.max() <= 1e-5, f"grid {k + 1}: {d.max()}"
    if k == 1:
        mx, my, mv = _engine_validates(e, p, k, *ref["raw1"], smooth=False)
        assert np.array_equal(mv, ref["median1"][2])
        assert np.array_equal(mx, ref["median1"][0]) and np.array_equal(my, ref["median1"][1])


def test_reference_validation_of_engine_candidates(run):
    p, g, f1, f2, r, ref, e = run
    # the engine's own last-pass grid-2 candidates (staged run), re-validated by both engines
    e.set_field(1, ref["pred"]["p2x"], ref["pred"]["p2y"], np.ones(g["Nt_vec"][1], np.uint8))
    e.pass_grid2()
    e.synchronize()
    _, _, cdx, cdy, cv = e.field(2)
    r.set_raw(1, cdx, cdy, cv)
    r.validate(1, p.Npass2_median, p.minNneigh_p2, p.residual_threshold_p2, p.insert_threshold_p2, 0, 0)
    rx, ry, rv = r.filtered(1, g["Nt_vec"][1])
    mx, my, mv = _engine_validates(e, p, 1, cdx, cdy, cv, smooth=False)
    assert np.array_equal(mv, rv) and np.array_equal(mx, rx) and np.array_equal(my, ry)
    r.set_raw(1, cdx, cdy, cv)
    r.validate(1, p.Npass2_median, p.minNneigh_p2, p.residual_threshold_p2, p.insert_threshold_p2,
               p.Npass2_smooth, 1)
    rx, ry, rv = r.filtered(1, g["Nt_vec"][1])
    fx, fy, fv = _engine_validates(e, p, 1, cdx, cdy, cv)
    assert np.array_equal(fv, rv)
    assert np.maximum(np.abs(fx - rx), np.abs(fy - ry)).max() <= 1e-5


def test_end_to_end_fields(run):
    """The whole pair through piv_run_pair (no staging) against the reference's run, held to
    the reference's agreement with its own second run on the same input."""
    p, g, f1, f2, r, ref, e = run
    with P.Engine(p) as full:
        full.set_images(f1, f2)
        full.run_pair()
        full.synchronize()
        for k in (0, 1):
            _, _, fx, fy, fv = full.field(2 * k + 1)
            rx, ry, rv = ref["e2e"][k]
            ax, ay, av = ref["again"][k]
            d = np.maximum(np.abs(fx - rx), np.abs(fy - ry))
            dr = np.maximum(np.abs(ax - rx), np.abs(ay - ry))
            print(f"\nend to end, grid {k + 1}: engine vs reference: validity equal {np.mean(fv == rv):.4%}, "
                  f"within 1e-3 px {np.mean(d < 1e-3):.4%}, max {d.max():.3e} px; reference vs itself: "
                  f"validity equal {np.mean(av == rv):.4%}, within 1e-3 px {np.mean(dr < 1e-3):.4%}, "
                  f"max {dr.max():.3e} px")
            assert np.mean(fv == rv) >= min(np.mean(av == rv), 0.999) - 1e-3
            assert np.mean(d < 1e-3) >= np.mean(dr < 1e-3) - 0.02
            assert d.max() <= max(2 * dr.max(), 0.05)
