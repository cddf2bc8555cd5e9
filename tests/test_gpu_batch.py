"""Batches of uneven pairs (piv_batch_*): mixed image sizes, window shapes and overlaps in
one graph with one persistent correlation launch per pass and window shape.  Every
pair's fields must be bit-identical to the same pair run alone (piv_run_pair): the batch
kernel runs the same correlation body on the same inputs."""
import numpy as np
import pytest

import piv_b200 as P

pytestmark = pytest.mark.gpu

# (Nx, Ny, ws2, overlap, mhe): grid 1 uses min(2*ws2, 64) at the same overlap
PAIRS = [(640, 480, 16, 0.75, 1), (520, 400, 24, 0.5, 0), (1024, 768, 32, 0.5, 1), (800, 600, 64, 0.75, 1),
         (640, 480, 32, 0.75, 0), (700, 500, 16, 0.5, 1)]


def pair_params(Nx, Ny, ws2, overlap, mhe):
    ws1 = min(2 * ws2, 64)
    sp = lambda ws: int(round(ws * (1 - overlap)))
    return P.default_params(Nx=Nx, Ny=Ny, if_mhe=mhe, mhe_ws=40, mhe_thresh=0.91, ws_x1=ws1, ws_y1=ws1,
                            spacing_x1=sp(ws1), spacing_y1=sp(ws1), Npass1=2, ws_x2=ws2, ws_y2=ws2,
                            spacing_x2=sp(ws2), spacing_y2=sp(ws2), Npass2=3, insert_threshold_p1=2.0,
                            insert_threshold_p2=2.0)


def _frames(k, Nx, Ny):
    s = P.synth_params(Nx, Ny, ppp=0.05, field=P.PIV_FIELD_FOURIER, a=200.0, b=2000.0, c=6.0 + k, seed=300 + k)
    return P.synth_pair(s)


def test_batch_matches_pairs_run_alone(cuda):
    params = [pair_params(*q) for q in PAIRS]
    frames = [_frames(k, q[0], q[1]) for k, q in enumerate(PAIRS)]
    want = []
    for p, (f1, f2) in zip(params, frames):
        with P.Engine(p) as e:
            e.set_images(f1, f2)
            e.run_pair()
            want.append([e.field(s) for s in range(4)])
    with P.Batch(params) as b:
        groups = b.groups()
        shapes = {(g["wsx"], g["grid"]) for g in groups}
        assert {(16, 1), (24, 1), (32, 1), (64, 1), (32, 0), (48, 0), (64, 0)} <= shapes
        assert sum(g["pairs"] for g in groups if g["grid"] == 1) == len(PAIRS)
        for e, (f1, f2) in zip(b.engines, frames):
            e.set_images(f1, f2)
        for rep in range(2):  # the first run tunes and runs eagerly, the second replays the graph
            b.run()
            b.synchronize()
            for i, e in enumerate(b.engines):
                for s in range(4):
                    got = e.field(s)
                    for u, v in zip(got, want[i][s]):
                        assert np.array_equal(u, v), (rep, i, s)


def test_batch_device_frames_and_regraph(cuda):
    import torch

    params = [pair_params(*q) for q in PAIRS[:3]]
    frames = [_frames(10 + k, q[0], q[1]) for k, q in enumerate(PAIRS[:3])]
    with P.Batch(params) as b:
        dev = []
        for e, (f1, f2) in zip(b.engines, frames):
            d1, d2 = torch.from_numpy(f1).cuda(), torch.from_numpy(f2).cuda()
            dev.append((d1, d2))
            torch.cuda.synchronize()
            e.set_device_images(d1.data_ptr(), d2.data_ptr())
        b.run()
        b.synchronize()
        got = [e.field(3) for e in b.engines]
        # host frames now: the batch graph is captured again for the new inputs
        for e, (f1, f2) in zip(b.engines, frames):
            e.set_images(f1, f2)
        b.run()
        b.synchronize()
        for i, e in enumerate(b.engines):
            for u, v in zip(e.field(3), got[i]):
                assert np.array_equal(u, v)


def test_batch_rejects_mixed_pass_counts(cuda):
    a = pair_params(*PAIRS[0])
    c = pair_params(*PAIRS[1])
    c.Npass2 = 2
    with pytest.raises(P.PivError):
        P.Batch([a, c])


def test_batch_group_over_96_pairs_single_grid(cuda):
    """100 pairs of one window shape form one group, which takes two launches (96 + 4 pairs
    per launch parameter); grid 1 only (Npass2 = 0).  Every pair matches its run alone."""
    n = 100
    p = P.default_params(Nx=160, Ny=128, if_mhe=0, ws_x1=32, ws_y1=32, spacing_x1=16, spacing_y1=16, Npass1=2,
                         ws_x2=32, ws_y2=32, spacing_x2=16, spacing_y2=16, Npass2=0)
    frames = []
    for k in range(n):
        s = P.synth_params(160, 128, ppp=0.05, field=P.PIV_FIELD_UNIFORM, a=1.0 + 0.02 * k, b=-0.5, seed=900 + k)
        frames.append(P.synth_pair(s))
    with P.Batch([p] * n) as b:
        groups = b.groups()
        assert [g["pairs"] for g in groups] == [n, n]  # grid 1: the undeformed and the deformed pass
        for e, (f1, f2) in zip(b.engines, frames):
            e.set_images(f1, f2)
        b.run()
        b.synchronize()
        got = [b.engines[i].field(1) for i in (0, 95, 96, 99)]
    for i, g in zip((0, 95, 96, 99), got):
        with P.Engine(p) as e:
            e.set_images(*frames[i])
            e.run_pair()
            for u, v in zip(g, e.field(1)):
                assert np.array_equal(u, v), i
