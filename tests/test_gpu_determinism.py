"""A pair's results do not depend on how its windows are launched.

The reference splits each pass's windows into Nsec_cc sections of Neach windows
(X/xcorr2d_multi_grid.cu:805-829, the section loop :1308-1441) only to bound the memory of
its FFT buffers; each window's correlation is computed alone, so the split never changes a
result.  Here the fused kernel shares one inverse transform between windows 2m and 2m + 1
and runs in several tile variants (windows per CTA, threads per CTA) that an autotuner
picks by timing.  These tests hold the engine to the reference's property, bit for bit:
  - every tile variant of every instantiated window shape (PIV_XCORR_VARIANT), with top-4
    and top-8 peak lists, gives identical candidates, peak taps and fields;
  - Nsec_cc = 1, 2, 3, 5, 7 (odd window counts per section) give identical results;
  - a batch whose groups are forced to other variants than the engines run alone
    (PIV_BATCH_VARIANT, PIV_AUTOTUNE=off) reproduces the pairs run alone;
  - a batch member set to the tensor-core path runs that path, as it would alone.
"""
import numpy as np
import pytest

import piv_b200 as P

pytestmark = pytest.mark.gpu

SHAPES = [(8, 8), (12, 12), (16, 16), (24, 24), (32, 32), (48, 48), (64, 64), (48, 24), (24, 48), (32, 16),
          (16, 32), (64, 32), (32, 64)]


def _frames(Nx, Ny, seed, c=4.0):
    s = P.synth_params(Nx, Ny, ppp=0.05, field=P.PIV_FIELD_FOURIER, a=150.0, b=1200.0, c=c, seed=seed)
    return P.synth_pair(s)


def _outputs(e, grids):
    out = []
    for k in grids:
        out.append(e.field(2 * k))         # raw candidates [Nt][Nps]
        out.append(e.field(2 * k + 1))     # filtered field
        out.append(e.peaks(k))             # counts, peak indices, values
    return out


def _assert_same(a, b, what):
    for i, (u, v) in enumerate(zip(a, b)):
        for j, (x, y) in enumerate(zip(u, v)):
            assert np.array_equal(x, y), f"{what}: output {i}.{j} differs"


def _run(p, f1, f2):
    with P.Engine(p) as e:
        e.set_images(f1, f2)
        e.run_pair()
        e.synchronize()
        return _outputs(e, [k for k, n in enumerate((p.Npass1, p.Npass2)) if n > 0]), e.xcorr_config(0)


@pytest.mark.parametrize("shape", SHAPES, ids=[f"{x}x{y}" for x, y in SHAPES])
@pytest.mark.parametrize("nps", [4, 6])
def test_every_tile_variant_gives_the_same_bits(cuda, monkeypatch, shape, nps):
    wx, wy = shape
    Nx, Ny = 416, 328
    f1, f2 = _frames(Nx, Ny, seed=700 + wx + wy)
    # grid 1 = the shape under test, two passes (undeformed, then deformed)
    p = P.default_params(Nx=Nx, Ny=Ny, ws_x1=wx, ws_y1=wy, spacing_x1=wx // 2, spacing_y1=wy // 2, Npass1=2,
                         Npass2=0, Npeak_save=nps, insert_threshold_p1=2.0, max_dispx_win_percent1=0.25,
                         max_dispy_win_percent1=0.25)
    ref = None
    seen = set()
    for v in range(8):
        monkeypatch.setenv("PIV_XCORR_VARIANT", f"{v},0")
        try:
            got, cfg = _run(p, f1, f2)
        except P.PivError as err:
            assert err.status == P.PIV_ERR_ARG and v > 0, err  # past the shape's last variant
            break
        seen.add(cfg[:2])
        if ref is None:
            ref = got
        else:
            _assert_same(got, ref, f"{wx}x{wy} variant {v} (windows/CTA, threads) = {cfg[:2]}")
    assert len(seen) >= 2, f"{wx}x{wy}: fewer than two variants exercised"


@pytest.mark.parametrize("tuned", ["on", "off"])
def test_nsec_cc_sections_give_the_same_bits(cuda, monkeypatch, tuned):
    monkeypatch.setenv("PIV_AUTOTUNE", tuned)
    Nx, Ny = 536, 408
    f1, f2 = _frames(Nx, Ny, seed=811, c=6.0)
    base = dict(Nx=Nx, Ny=Ny, if_mhe=1, ws_x1=64, ws_y1=64, spacing_x1=32, spacing_y1=32, Npass1=2, ws_x2=32,
                ws_y2=32, spacing_x2=16, spacing_y2=16, Npass2=2, insert_threshold_p1=2.0, insert_threshold_p2=2.0)
    ref = None
    odd = 0
    for nsec in (1, 2, 3, 5, 7):
        p = P.default_params(Nsec_cc=nsec, **base)
        g = P.geometry(p)
        odd += sum(n % 2 for n in g["Neach"])
        got, _ = _run(p, f1, f2)
        if ref is None:
            ref = got
        else:
            _assert_same(got, ref, f"Nsec_cc={nsec} (Neach {g['Neach']}, Nlast {g['Nlast']})")
    assert odd >= 2, "no section with an odd window count was exercised"


PAIRS = [(640, 480, 16, 0.75, 1), (520, 400, 24, 0.5, 0), (1024, 768, 32, 0.5, 1), (800, 600, 64, 0.75, 1),
         (600, 440, 48, 0.5, 0)]


def _pair_params(Nx, Ny, ws2, overlap, mhe):
    ws1 = min(2 * ws2, 64)
    sp = lambda ws: int(round(ws * (1 - overlap)))
    return P.default_params(Nx=Nx, Ny=Ny, if_mhe=mhe, mhe_ws=40, mhe_thresh=0.91, ws_x1=ws1, ws_y1=ws1,
                            spacing_x1=sp(ws1), spacing_y1=sp(ws1), Npass1=2, ws_x2=ws2, ws_y2=ws2,
                            spacing_x2=sp(ws2), spacing_y2=sp(ws2), Npass2=2, insert_threshold_p1=2.0,
                            insert_threshold_p2=2.0)


def _alone(params, frames, paths=None):
    out = []
    for i, (p, (f1, f2)) in enumerate(zip(params, frames)):
        with P.Engine(p) as e:
            if paths and paths[i]:
                e.set_xcorr_path(1, paths[i])
            e.set_images(f1, f2)
            e.run_pair()
            out.append([e.field(s) for s in range(4)])
    return out


def _batch(params, frames, paths=None, reps=2):
    got = []
    with P.Batch(params) as b:
        for i, (e, (f1, f2)) in enumerate(zip(b.engines, frames)):
            if paths and paths[i]:
                e.set_xcorr_path(1, paths[i])
            e.set_images(f1, f2)
        for _ in range(reps):
            b.run()
            b.synchronize()
            got.append([[e.field(s) for s in range(4)] for e in b.engines])
        groups = b.groups()
    return got, groups


@pytest.mark.parametrize("alone_variant,batch_variant", [("last", "0"), ("0", "1"), ("tuned", "tuned")])
def test_batch_matches_alone_whatever_the_variants(cuda, monkeypatch, alone_variant, batch_variant):
    params = [_pair_params(*q) for q in PAIRS]
    frames = [_frames(q[0], q[1], seed=900 + k) for k, q in enumerate(PAIRS)]
    if alone_variant == "last":
        monkeypatch.setenv("PIV_XCORR_VARIANT", "3,3")  # every shape used here has at least 4 variants
    elif alone_variant == "0":
        monkeypatch.setenv("PIV_AUTOTUNE", "off")
    want = _alone(params, frames)
    monkeypatch.delenv("PIV_XCORR_VARIANT", raising=False)
    monkeypatch.delenv("PIV_AUTOTUNE", raising=False)
    if batch_variant != "tuned":
        monkeypatch.setenv("PIV_BATCH_VARIANT", batch_variant)
    got, groups = _batch(params, frames)
    if batch_variant != "tuned":
        assert all(g["variant"] == int(batch_variant) % 2 for g in groups)
    for rep, fields in enumerate(got):
        for i in range(len(PAIRS)):
            for s in range(4):
                for u, v in zip(fields[i][s], want[i][s]):
                    assert np.array_equal(u, v), (alone_variant, batch_variant, rep, i, s)


def test_batch_runs_a_members_tensor_core_path(cuda):
    params = [_pair_params(*q) for q in PAIRS[:3]]
    frames = [_frames(q[0], q[1], seed=950 + k) for k, q in enumerate(PAIRS[:3])]
    paths = [0, 0, P.PIV_XCORR_TC_SPLIT]  # the 32x32 pair's grid 2 on split-BF16 tcgen05
    want = _alone(params, frames, paths)
    simt = _alone(params[2:], frames[2:])
    got, groups = _batch(params, frames, paths)
    # the tensor-core pair is in no SIMT group of grid 2
    assert sum(g["pairs"] for g in groups if g["grid"] == 1) == 2
    for fields in got:
        for i in range(3):
            for s in range(4):
                for u, v in zip(fields[i][s], want[i][s]):
                    assert np.array_equal(u, v), (i, s)
    # and its result is the tensor-core one, not the SIMT one
    assert not all(np.array_equal(u, v) for u, v in zip(got[-1][2][2], simt[0][2]))


BLOCK_32 = 5  # index of the 2x2-block form among the 32x32 variants (after the row-major ones)


@pytest.mark.parametrize("Nx,Ny,sp,nsec", [(432, 344, 8, 1), (432, 344, 8, 7), (448, 352, 32, 1), (448, 352, 32, 3),
                                           (432, 344, 16, 1), (416, 328, 16, 5)],
                         ids=["75pc-rows-odd", "75pc-7-sections", "no-overlap", "no-overlap-3-sections",
                              "odd-row-fallback", "50pc-5-sections"])
def test_block_form_gives_the_same_bits(cuda, monkeypatch, Nx, Ny, sp, nsec):
    """The 2x2-block form (two window rows per CTA sharing their overlapping pixel rows)
    against the row-major 4 x 128 form: window grids with an odd number of rows (a partial
    last block row), 75 %, 50 % and no overlap, sections starting inside a block row, an odd
    row of windows (the form falls back to the row-major launch), and a plane dump starting
    at an odd window."""
    f1, f2 = _frames(Nx, Ny, seed=900 + sp + nsec)
    p = P.default_params(Nx=Nx, Ny=Ny, ws_x1=32, ws_y1=32, spacing_x1=sp, spacing_y1=sp, Npass1=2, Npass2=0,
                         Nsec_cc=nsec, insert_threshold_p1=2.0, max_dispx_win_percent1=0.25,
                         max_dispy_win_percent1=0.25)
    res = []
    for v in (1, BLOCK_32):
        monkeypatch.setenv("PIV_XCORR_VARIANT", f"{v},0")
        with P.Engine(p) as e:
            e.set_images(f1, f2)
            e.run_pair()
            e.synchronize()
            assert e.xcorr_config(0)[:2] == (4, 128)
            nt = e.geom["Nt_vec"][0]
            res.append((_outputs(e, [0]), e.cc_planes(0, 37, min(300, nt - 40))))
    _assert_same(res[1][0], res[0][0], f"{Nx}x{Ny} sp {sp} Nsec {nsec}: block form")
    assert np.array_equal(res[1][1], res[0][1]), "plane dump differs"
