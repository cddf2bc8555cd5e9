"""The CUDA engine against the reference's own outputs (tests/golden/, recorded from the
reference engine compiled for sm_100a; see tests/golden/make_golden.py).

Tolerances (FP32 on both sides, different FFT algorithms):
  MHE frames                   bit-exact
  top-N peak indices           bit-exact, except windows whose top Nps+1 candidate values
                               lie within 1e-5 (relative) of each other
  candidate counts             bit-exact, except windows holding a 4-neighbour comparison
                               within 1e-5 of the window peak (the local-maximum test flips)
  raw displacements            1e-3 px where the peak index agrees
  filtered / median-only field validity and 1e-3 px on >= 99.5 % of vectors
  correlation planes           1e-5 of the window peak
  deformed frame               1e-3 grey levels
Near-tie windows are found from the engine's own correlation planes (piv_debug_cc_planes).
"""
import ast
from pathlib import Path

import numpy as np
import pytest

import piv_b200 as P

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden"


def load(name):
    f = GOLD / f"golden_{name}.npz"
    if not f.exists():
        pytest.skip(f"{f.name} missing")
    return np.load(f)


def near_ties(planes, bx, by, nps, rel=1e-5):
    """(tie_topN, tie_count) masks per window from shifted planes [n][wsy][wsx]."""
    n, wsy, wsx = planes.shape
    c = planes[:, by:wsy - by, bx:wsx - bx]
    l = planes[:, by:wsy - by, bx - 1:wsx - bx - 1]
    r = planes[:, by:wsy - by, bx + 1:wsx - bx + 1]
    u = planes[:, by - 1:wsy - by - 1, bx:wsx - bx]
    d = planes[:, by + 1:wsy - by + 1, bx:wsx - bx]
    peak = planes.reshape(n, -1).max(1)[:, None, None]
    tol = rel * np.maximum(peak, 1e-30)
    cand = (c > 0) & (c >= l) & (c >= r) & (c >= u) & (c >= d)
    close = np.zeros_like(cand)
    for nb in (l, r, u, d):
        close |= np.abs(c - nb) <= tol
    tie_count = close.reshape(n, -1).any(1)
    tie_top = np.zeros(n, bool)
    for w in range(n):
        v = np.sort(c[w][cand[w]])[::-1][:nps + 1]
        if v.size > 1 and (np.abs(np.diff(v)) <= rel * v[0]).any():
            tie_top[w] = True
    return tie_top, tie_count | tie_top


def fit_tolerance(planes, idx, wsx, rel_cc=1e-5):
    """Per-candidate bound on |engine - reference| for the 3-point Gaussian fit.

    delta = num / (2 den), num = ln f- - ln f+, den = ln f- + ln f+ - 2 ln f0.  Two FP32
    FFTs of different algorithms agree to an ABSOLUTE error of about rel_cc times the
    window's largest correlation value (the planes test asserts it), so a value c carries
    a log error of rel_cc * max / c -- large for weak secondary peaks.  The reference also
    forms den in FP32 (each logf within 1 ulp, then two roundings); the engine in FP64.
    Propagating: |d delta| <= (|delta| * e_den + e_num / 2) / |den| with
    e_num = e(f-) + e(f+) + 2^-23 (|ln f-| + |ln f+|),
    e_den = e(f-) + e(f+) + 2 e(f0) + 2^-22 (|ln f-| + |ln f+| + 2 |ln f0|).
    Strong, well-conditioned peaks get ~1e-3 px."""
    n, wsy, _ = planes.shape
    tols = []
    for axis in (1, wsx):
        t = np.full(idx.shape, 1e-3)
        for w in range(n):
            flat = planes[w].ravel()
            cmax = float(flat.max())
            for q in range(idx.shape[1]):
                li = idx[w, q]
                if li < 0 or li - axis < 0 or li + axis >= flat.size:
                    continue
                c0, c1, c2 = (float(flat[li - axis]), float(flat[li]), float(flat[li + axis]))
                if min(c0, c1, c2) <= 0:
                    t[w, q] = np.inf
                    continue
                f0, f1, f2 = np.log(c0), np.log(c1), np.log(c2)
                den = f0 + f2 - 2 * f1
                e0, e1, e2 = (rel_cc * cmax / c0, rel_cc * cmax / c1, rel_cc * cmax / c2)
                e_num = e0 + e2 + 2.0 ** -23 * (abs(f0) + abs(f2))
                e_den = e0 + e2 + 2 * e1 + 2.0 ** -22 * (abs(f0) + abs(f2) + 2 * abs(f1))
                if abs(den) <= e_den:
                    t[w, q] = np.inf  # the denominator's sign is not determined at this precision
                    continue
                delta = (f0 - f2) / den / 2
                t[w, q] = 1e-3 + (abs(delta) * e_den + e_num / 2) / (abs(den) - e_den)
        tols.append(t)
    return tols


def staged_run(e, p, z):
    """X/main.cpp:288-326 through the stage entry points; before each grid's last pass
    the reference's own filtered field (its predictor and deformation field) is put in
    place, so that the last pass of every grid sees the reference's inputs."""
    e.prep()
    for j in range(p.Npass1):
        if j == p.Npass1 - 1 and j > 0 and "pred0_dx" in z.files:
            e.set_field(0, z["pred0_dx"], z["pred0_dy"], np.ones(z["pred0_dx"].size, np.uint8))
        e.pass_grid1(j)
        e.validate_grid1()
    if p.Npass2 > 0:
        e.upsample()
        for j in range(p.Npass2):
            if j == p.Npass2 - 1 and "pred1_dx" in z.files:
                e.set_field(1, z["pred1_dx"], z["pred1_dy"], np.ones(z["pred1_dx"].size, np.uint8))
            e.pass_grid2()
            e.validate_grid2(iffill=1)
    e.synchronize()


@pytest.fixture(scope="module", params=["c0", "multigrid", "nonsquare"])
def run(request, cuda):
    z = load(request.param)
    sk = ast.literal_eval(str(z["synth"][0]))
    pk = ast.literal_eval(str(z["params"][0]))
    f1, f2 = P.synth_pair(P.synth_params(**sk))
    p = P.default_params(**pk)
    e = P.Engine(p)
    e.set_images(f1, f2)
    staged_run(e, p, z)
    yield request.param, z, p, e
    e.close()


@pytest.fixture(scope="module", params=["c0", "multigrid", "nonsquare"])
def full_run(request, cuda):
    """The whole pair through piv_run_pair (no injected state)."""
    z = load(request.param)
    sk = ast.literal_eval(str(z["synth"][0]))
    pk = ast.literal_eval(str(z["params"][0]))
    f1, f2 = P.synth_pair(P.synth_params(**sk))
    p = P.default_params(**pk)
    e = P.Engine(p)
    e.set_images(f1, f2)
    e.run_pair()
    e.synchronize()
    yield request.param, z, p, e
    e.close()


def test_mhe_frames_bitexact(run):
    name, z, p, e = run
    if not p.if_mhe:
        pytest.skip("MHE off in this case")
    g1, g2 = e.frames()
    assert np.array_equal(g1, z["f1_mhe"]) and np.array_equal(g2, z["f2_mhe"])


def test_peaks_and_candidates(run):
    name, z, p, e = run
    for k in ([0, 1] if p.Npass2 > 0 else [0]):
        nt = e.geom["Nt_vec"][k]
        planes = e.cc_planes(k, 0, nt)
        tie_top, tie_cnt = near_ties(planes, e.geom["border_x"][k], e.geom["border_y"][k], p.Npeak_save)
        cnt, idx, val = e.peaks(k)
        _, _, dx, dy, v = e.field(2 * k)
        ok = ~tie_top
        assert ok.mean() > 0.9
        assert np.array_equal(idx[ok], z[f"peaks{k}_index"][ok]), f"{name} grid {k}"
        okc = ~tie_cnt
        assert np.array_equal(cnt[okc], z[f"peaks{k}_count"][okc]), f"{name} grid {k}"
        same = (idx == z[f"peaks{k}_index"]) & ok[:, None]
        assert np.array_equal(v[same], z[f"raw{k}_valid"][same])
        both = same & (v == 1)
        tx, ty = fit_tolerance(planes, idx, p.ws_x2 if k else p.ws_x1)
        assert (np.abs(dx - z[f"raw{k}_dx"])[both] <= tx[both]).all()
        assert (np.abs(dy - z[f"raw{k}_dy"])[both] <= ty[both]).all()
        # the main peak of each window: within 1e-3 px almost everywhere
        b0 = both[:, 0]
        d0 = np.maximum(np.abs(dx - z[f"raw{k}_dx"]), np.abs(dy - z[f"raw{k}_dy"]))[:, 0]
        assert (d0[b0] < 1e-3).mean() >= 0.999
        assert np.abs(val[same] - z[f"peaks{k}_value"][same]).max() <= 1e-5 * np.abs(val).max()


def test_filtered_fields(full_run):
    """End to end (no staging).  Validation itself is exact on identical candidates
    (test_validation_of_reference_candidates); the 0.5 % left here is the flags and vectors
    that follow candidates differing upstream at FP32 rounding (each grid's passes feed the
    next through the filtered field), near the median test's thresholds."""
    name, z, p, e = full_run
    for k in ([0, 1] if p.Npass2 > 0 else [0]):
        _, _, fx, fy, fv = e.field(2 * k + 1)
        assert (fv == z[f"filt{k}_valid"]).mean() >= 0.995
        d = np.maximum(np.abs(fx - z[f"filt{k}_dx"]), np.abs(fy - z[f"filt{k}_dy"]))
        assert (d < 1e-3).mean() >= 0.995, f"{name} grid {k}: {np.sort(d)[-5:]}"


def test_median_only_field(full_run):
    name, z, p, e = full_run
    if p.Npass2 == 0:
        pytest.skip("single grid")
    # X/main.cpp:363: median test only, no smoothing, no fill
    e.validate_grid2(p.Npass2_median, p.minNneigh_p2, p.residual_threshold_p2, p.insert_threshold_p2, 0, 0)
    _, _, mx, my, mv = e.field(3)
    assert (mv == z["median2_valid"]).mean() >= 0.995
    d = np.maximum(np.abs(mx - z["median2_dx"]), np.abs(my - z["median2_dy"]))
    assert (d < 1e-3).mean() >= 0.995


def test_planes_and_deformation(run):
    name, z, p, e = run
    last = 1 if p.Npass2 > 0 else 0
    n = z["cc_last"].shape[0]
    got = e.cc_planes(last, 0, n)
    for w in range(n):
        assert np.abs(got[w] - z["cc_last"][w]).max() <= 1e-5 * z["cc_last"][w].max()
    if p.Npass2 > 0:
        # the two engines deform with filtered fields that differ by ~1e-5 px (FP32 FFTs of
        # different algorithms upstream); times image gradients of up to ~250 grey levels/px
        d = np.abs(e.deformed(1)[::16] - z["deformed1_rows"])
        assert d.max() < 2e-2 and d.mean() < 2e-4


def test_reference_style_driver_matches_run_pair(cuda):
    """The xcorr2d_multi mirror driven in X/main.cpp order gives the run_pair results."""
    z = load("multigrid")
    sk = ast.literal_eval(str(z["synth"][0]))
    pk = dict(ast.literal_eval(str(z["params"][0])))
    pk["if_mhe"] = 0
    f1, f2 = P.synth_pair(P.synth_params(**sk))
    p = P.default_params(**pk)
    x = P.xcorr2d_multi()
    assert x.init(p.Nx, p.Ny, p.Nsec_cc, p.ws_x1, p.ws_y1, p.spacing_x1, p.spacing_y1, p.Npass1, p.ws_x2, p.ws_y2,
                  p.spacing_x2, p.spacing_y2, p.Npass2, p.wx1_median, p.wy1_median, p.wx2_median, p.wy2_median,
                  p.wx1_smooth, p.wy1_smooth, p.wx2_smooth, p.wy2_smooth, p.Npeak_save, p.max_dispx_win_percent1,
                  p.max_dispy_win_percent1, p.max_dispx_win_percent2, p.max_dispy_win_percent2, p.dispx_lim1,
                  p.dispx_lim2, p.dispy_lim1, p.dispy_lim2)
    x.h_img1_org[:] = f1
    x.h_img2_org[:] = f2
    x.prep_img_data()
    for j in range(x.Npass1):
        if j > 0:
            x.extend_filtered_vecfield_p1()
        assert x.Calc_cc_map_p1(j)
        assert x.MedianFilter_Smoothing_p1(p.Npass1_median, p.minNneigh_p1, p.residual_threshold_p1,
                                           p.insert_threshold_p1, p.Npass1_smooth)
    x.extend_filtered_vecfield_p1()
    assert x.Upsampling_vector_field()
    for j in range(x.Npass2):
        x.extend_filtered_vecfield_p2()
        assert x.Calc_cc_map_p2()
        assert x.MedianFilter_Smoothing_p2(p.Npass2_median, p.minNneigh_p2, p.residual_threshold_p2,
                                           p.insert_threshold_p2, p.Npass2_smooth, 1)
    _, _, ax, ay, av = x._e.field(3)
    x.freemem()
    with P.Engine(p) as e:
        e.set_images(f1, f2)
        e.run_pair()
        _, _, bx, by, bv = e.field(3)
    assert np.array_equal(av, bv) and np.array_equal(ax, bx) and np.array_equal(ay, by)


@pytest.mark.parametrize("name", ["c0", "multigrid", "nonsquare"])
def test_validation_of_reference_candidates(cuda, name):
    """Validation alone, on the reference's own last-pass candidates of each grid: the median
    test, hole fill and smoothing (X/xcorr2d_multi_grid.cu:174-443, 1480-1545) give exactly the
    reference's validity flags and replacement choices, and the smoothed values to 1e-5 px (the
    reference sums them in atomic order).  So every end-to-end difference in the filtered
    fields comes from candidates that differ upstream, not from the validation."""
    z = load(name)
    sk = ast.literal_eval(str(z["synth"][0]))
    pk = ast.literal_eval(str(z["params"][0]))
    f1, f2 = P.synth_pair(P.synth_params(**sk))
    p = P.default_params(**pk)
    with P.Engine(p) as e:
        e.set_images(f1, f2)
        e.prep()
        for k in ([0, 1] if p.Npass2 > 0 else [0]):
            e.set_candidates(k, z[f"raw{k}_dx"], z[f"raw{k}_dy"], z[f"raw{k}_valid"])
            if k == 0:
                e.validate_grid1()
            else:
                e.validate_grid2(iffill=1)
            _, _, fx, fy, fv = e.field(2 * k + 1)
            assert np.array_equal(fv, z[f"filt{k}_valid"]), f"{name} grid {k}: {(fv != z[f'filt{k}_valid']).sum()}"
            d = np.maximum(np.abs(fx - z[f"filt{k}_dx"]), np.abs(fy - z[f"filt{k}_dy"]))
            assert d.max() <= 1e-5, f"{name} grid {k}: {d.max()}"
        if p.Npass2 > 0:
            # X/main.cpp:363: the median test alone, bit-exact
            e.set_candidates(1, z["raw1_dx"], z["raw1_dy"], z["raw1_valid"])
            e.validate_grid2(p.Npass2_median, p.minNneigh_p2, p.residual_threshold_p2, p.insert_threshold_p2, 0, 0)
            _, _, mx, my, mv = e.field(3)
            assert np.array_equal(mv, z["median2_valid"])
            assert np.array_equal(mx, z["median2_dx"]) and np.array_equal(my, z["median2_dy"])
