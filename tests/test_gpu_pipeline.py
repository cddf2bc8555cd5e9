"""Pipelined input (piv_queue_images): the upload of pair k+1 on the engine's copy stream
overlaps the computation of pair k, through two device input slots.  Every pair must
give exactly the fields of the one-pair-at-a-time path (piv_set_images + piv_run_pair):
same kernels, same inputs, so bit-identical.  Also: the slot reuse across more pairs than
slots, both input paths (MHE on and off), and the out-of-order call refused."""
import numpy as np
import pytest

import piv_b200 as P

pytestmark = pytest.mark.gpu


def _pairs(n, Nx, Ny):
    out = []
    for k in range(n):
        s = P.synth_params(Nx, Ny, ppp=0.05, field=P.PIV_FIELD_VORTEX, a=4.0 + k, b=90.0, c=0.001 * k, seed=70 + k)
        out.append(P.synth_pair(s))
    return out


def _params(Nx, Ny, mhe):
    return P.default_params(Nx=Nx, Ny=Ny, if_mhe=mhe, mhe_ws=40, mhe_thresh=0.91, ws_x1=64, ws_y1=64,
                            spacing_x1=32, spacing_y1=32, Npass1=2, ws_x2=32, ws_y2=32, spacing_x2=16,
                            spacing_y2=16, Npass2=2)


@pytest.mark.parametrize("mhe", [1, 0])
def test_queued_pairs_match_one_at_a_time(cuda, mhe):
    import torch

    Nx, Ny = 480, 400
    pairs = _pairs(5, Nx, Ny)
    p = _params(Nx, Ny, mhe)
    want = []
    with P.Engine(p) as e:
        for f1, f2 in pairs:
            e.set_images(f1, f2)
            e.run_pair()
            want.append([e.field(k) for k in range(4)])
    # pinned host copies, one per pair, as a streaming caller would hold them
    pinned = [(torch.from_numpy(f1).pin_memory(), torch.from_numpy(f2).pin_memory()) for f1, f2 in pairs]
    with P.Engine(p) as e:
        e.queue_images(*pinned[0])
        for k in range(len(pairs)):
            e.run_pair()
            if k + 1 < len(pairs):
                e.queue_images(*pinned[k + 1])
            got = [e.field(s) for s in range(4)]
            for s in range(4):
                for a, b in zip(got[s], want[k][s]):
                    assert np.array_equal(a, b), f"pair {k} selection {s}"


def test_queue_twice_is_refused_and_set_images_discards(cuda):
    Nx, Ny = 320, 256
    (f1, f2), (g1, g2) = _pairs(2, Nx, Ny)
    p = _params(Nx, Ny, 0)
    with P.Engine(p) as e:
        e.queue_images(f1, f2)
        with pytest.raises(P.PivError) as ex:
            e.queue_images(g1, g2)
        assert ex.value.status == P.PIV_ERR_STATE
        # an explicit input discards the queued pair
        e.set_images(g1, g2)
        e.run_pair()
        got = e.field(3)
        e.queue_images(g1, g2)
        e.run_pair()
        again = e.field(3)
        for a, b in zip(got, again):
            assert np.array_equal(a, b)


def test_async_readback_pipeline(cuda):
    """Queued uploads and asynchronous readbacks together: every pair's field matches the
    one-at-a-time path bit for bit although the next pair is always queued, and its
    readback enqueued, before the previous pair's results are collected; at most two
    readbacks may be pending, and a stale ticket is refused."""
    import torch

    Nx, Ny = 480, 400
    pairs = _pairs(4, Nx, Ny)
    p = _params(Nx, Ny, 1)
    want = []
    with P.Engine(p) as e:
        for f1, f2 in pairs:
            e.set_images(f1, f2)
            e.run_pair()
            want.append((e.field(3), e.field(2)))
    pinned = [(torch.from_numpy(f1).pin_memory(), torch.from_numpy(f2).pin_memory()) for f1, f2 in pairs]
    with P.Engine(p) as e:
        got = []
        e.queue_images(*pinned[0])
        prev = None
        for k in range(len(pairs)):
            e.run_pair()
            tk = e.field_async(3)
            if k + 1 < len(pairs):
                e.queue_images(*pinned[k + 1])
            if prev is not None:
                got.append(e.field_wait(prev))
            prev = tk
        got.append(e.field_wait(prev))
        with pytest.raises(P.PivError):
            e.field_wait(prev)  # already collected
        # both slots in use: a third pending readback is refused until one is collected
        ta, tb = e.field_async(3), e.field_async(2)
        with pytest.raises(P.PivError) as ex:
            e.field_async(0)
        assert ex.value.status == P.PIV_ERR_STATE
        raw2 = e.field_wait(tb)
        last3 = e.field_wait(ta)
    for k in range(len(pairs)):
        for a, b in zip(got[k], want[k][0]):
            assert np.array_equal(a, b), f"pair {k}"
    for a, b in zip(last3, want[-1][0]):
        assert np.array_equal(a, b)
    for a, b in zip(raw2, want[-1][1]):
        assert np.array_equal(a, b)
