"""Pins the CPU oracle to the reference's own outputs (CPU only).

tests/golden/golden_*.npz were recorded by tests/golden/make_golden.py from the reference
engine itself (xcorr2d_multi + mhe_gpu compiled for sm_100a from the reference sources,
driven in main.cpp order) on seeded synthetic inputs.  The oracle must reproduce them:
  MHE                        bit-exact
  peak indices (top-N)       bit-exact in every window (these fixtures hold no exact ties)
  candidate counts           bit-exact except windows whose 4-neighbour comparisons are
                             within FP32 rounding (oracle planes are FP64, the reference's
                             cuFFT planes FP32): at least 95 % of windows
  displacements (raw)        within 1e-3 px for the first peak; 99 % of all candidates
  filtered fields            validity bit-exact, displacement within 1e-3 px
  correlation planes         within 1e-5 of each window's peak value
Oracle FFT itself: against the exact direct correlation sum and numpy.
"""
import ast
from pathlib import Path

import numpy as np
import pytest

import piv_b200 as P
from oracle import oracle as O

GOLD = Path(__file__).resolve().parent / "golden"
CASES = ["c0", "multigrid", "nonsquare"]


def load(name):
    f = GOLD / f"golden_{name}.npz"
    if not f.exists():
        pytest.skip(f"{f.name} missing")
    return np.load(f)


def case_inputs(z):
    sk = ast.literal_eval(str(z["synth"][0]))
    pk = ast.literal_eval(str(z["params"][0]))
    f1, f2 = P.synth_pair(P.synth_params(**sk))
    return f1, f2, P.default_params(**pk)


@pytest.fixture(scope="module", params=CASES)
def oracle_case(request):
    z = load(request.param)
    f1, f2, p = case_inputs(z)
    if p.if_mhe:
        f1 = O.mhe(f1, p.mhe_ws, p.mhe_thresh)
        f2 = O.mhe(f2, p.mhe_ws, p.mhe_thresh)
    return request.param, z, p, f1, f2, O.run_pair(f1, f2, p)


@pytest.mark.parametrize("name", ["mhe_640x480", "mhe_333x251", "mhe_300x200_16"])
def test_oracle_mhe_matches_reference(name):
    z = load(name)
    s = ast.literal_eval(str(z["synth"][0]))
    f1, _ = P.synth_pair(P.synth_params(**s))
    assert np.array_equal(O.mhe(f1, int(z["ws"]), float(z["thresh"])), z["out"])


def test_oracle_mhe_frames_of_multigrid_case():
    z = load("multigrid")
    f1, f2, p = case_inputs(z)
    assert np.array_equal(O.mhe(f1, p.mhe_ws, p.mhe_thresh), z["f1_mhe"])
    assert np.array_equal(O.mhe(f2, p.mhe_ws, p.mhe_thresh), z["f2_mhe"])


def test_oracle_candidates_match_reference(oracle_case):
    name, z, p, _, _, r = oracle_case
    for k in ([0, 1] if p.Npass2 > 0 else [0]):
        c = r["raw"][k]
        assert (c.flags == 0).all()
        assert np.array_equal(c.peak_index, z[f"peaks{k}_index"]), f"{name} grid {k}"
        assert (c.count == z[f"peaks{k}_count"]).mean() >= 0.95
        v = (c.valid == 1) & (z[f"raw{k}_valid"] == 1)
        assert np.array_equal(c.valid, z[f"raw{k}_valid"])
        d = np.maximum(np.abs(c.dx - z[f"raw{k}_dx"]), np.abs(c.dy - z[f"raw{k}_dy"]))[v]
        assert (d < 1e-3).mean() >= 0.99
        first = v[:, 0]
        d0 = np.maximum(np.abs(c.dx[:, 0] - z[f"raw{k}_dx"][:, 0]), np.abs(c.dy[:, 0] - z[f"raw{k}_dy"][:, 0]))
        assert d0[first].max() < 1e-3


def test_oracle_filtered_fields_match_reference(oracle_case):
    name, z, p, _, _, r = oracle_case
    for k in ([0, 1] if p.Npass2 > 0 else [0]):
        fx, fy, fv = r["filt"][k]
        assert np.array_equal(fv, z[f"filt{k}_valid"])
        assert np.abs(fx - z[f"filt{k}_dx"]).max() < 1e-3 and np.abs(fy - z[f"filt{k}_dy"]).max() < 1e-3
    if p.Npass2 > 0:
        mx, my, mv = r["median_only"]
        assert np.array_equal(mv, z["median2_valid"])
        assert np.abs(mx - z["median2_dx"]).max() < 1e-3 and np.abs(my - z["median2_dy"]).max() < 1e-3


def test_oracle_planes_match_reference_c0():
    z = load("c0")
    f1, f2, p = case_inputs(z)
    g = P.geometry(p)
    xl, yl, sp, ws = g["Nx_left"][0], g["Ny_left"][0], p.spacing_x1, p.ws_x1
    pad = 64
    a = np.pad(f1.astype(np.float64), pad)
    b = np.pad(f2.astype(np.float64), pad)
    nxv = g["Nx_vec"][0]
    for w in range(z["cc_last"].shape[0]):
        iy, ix = divmod(w, nxv)
        y0, x0 = iy * sp - yl + pad, ix * sp - xl + pad
        cc = O.xcorr_plane(a[y0:y0 + ws, x0:x0 + ws], b[y0:y0 + ws, x0:x0 + ws])
        assert np.abs(cc - z["cc_last"][w]).max() <= 1e-5 * cc.max()


@pytest.mark.parametrize("wsx,wsy", [(8, 8), (12, 12), (16, 16), (24, 24), (32, 32), (48, 24), (20, 28), (64, 64)])
def test_oracle_fft_against_direct_sum_and_numpy(wsx, wsy):
    rng = np.random.default_rng(wsx * 100 + wsy)
    w1 = rng.integers(0, 256, (wsy, wsx)).astype(np.float64)
    w2 = rng.integers(0, 256, (wsy, wsx)).astype(np.float64)
    fft = O.xcorr_plane(w1, w2)
    direct = O.xcorr_plane(w1, w2, direct=True)
    ref = np.fft.fftshift(np.abs(np.fft.ifft2(np.conj(np.fft.fft2(w1)) * np.fft.fft2(w2))))
    assert np.abs(fft - direct).max() <= 1e-12 * direct.max()
    assert np.abs(fft - ref).max() <= 1e-12 * direct.max()
