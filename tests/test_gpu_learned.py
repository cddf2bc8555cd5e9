"""The learned grid-1 predictor's kernels against the NumPy oracle (oracle/learned.py):
the device synthetic generator against the host one, the features (box average + cost
volume), the network's forward pass, loss and full parameter gradient, one Adam step,
and the learned pair with its judge and fallback."""
import numpy as np
import pytest

import piv_b200 as P
from oracle import learned as L

pytestmark = pytest.mark.gpu


def test_device_synth_matches_host(cuda):
    import torch

    for field, (a, b, c) in ((P.PIV_FIELD_FOURIER, (200.0, 2000.0, 12.0)), (P.PIV_FIELD_VORTEX, (8.0, 150.0, 0.002))):
        s = P.synth_params(333, 251, ppp=0.06, sigma=0.6, field=field, a=a, b=b, c=c, seed=11)
        h1, h2 = P.synth_pair(s)
        d1 = torch.empty(251 * 333, dtype=torch.uint8, device="cuda")
        d2 = torch.empty_like(d1)
        scratch = torch.empty(2 * 251 * 333, dtype=torch.float32, device="cuda")
        P.synth_pair_device(s, d1, d2, scratch)
        torch.cuda.synchronize()
        g1 = d1.cpu().numpy().reshape(251, 333)
        g2 = d2.cpu().numpy().reshape(251, 333)
        for h, g in ((h1, g1), (h2, g2)):
            diff = np.abs(h.astype(int) - g.astype(int))
            assert diff.max() <= 1
            assert (diff > 0).mean() < 1e-3  # rounding ties of the float accumulation only


def test_features_match_oracle(cuda):
    import torch

    Nx, Ny = 520, 392
    s = P.synth_params(Nx, Ny, ppp=0.05, field=P.PIV_FIELD_VORTEX, a=6.0, b=120.0, c=0.001, seed=5)
    f1, f2 = P.synth_pair(s)
    p = P.default_params(Nx=Nx, Ny=Ny, if_mhe=0, ws_x1=64, ws_y1=64, spacing_x1=32, spacing_y1=32, Npass1=2,
                         ws_x2=32, ws_y2=32, spacing_x2=16, spacing_y2=16, Npass2=1)
    with P.Engine(p) as e, P.PredictorNet(seed=1) as net:
        e.set_images(f1, f2)
        e.prep()
        g = e.geom
        H, W = g["Ny_vec"][0], g["Nx_vec"][0]
        out = torch.empty(81 * H * W, dtype=torch.float32, device="cuda")
        e.features(net, out)
        e.synchronize()
        got = out.cpu().numpy().reshape(81, H, W)
    want = L.features(f1, f2, W, H, 32, 32, g["Nx_left"][0], g["Ny_left"][0], 64, 64)
    assert np.abs(got - want).max() < 2e-5
    # every interior vector's strongest shift is the true displacement rounded to the
    # downsampled grid (|u| <= 6 px = 1.5 downsampled px)
    k = want.reshape(81, -1).argmax(axis=0)
    assert (np.abs(k // 9 - 4) <= 2).all() and (np.abs(k % 9 - 4) <= 2).all()


@pytest.mark.parametrize("ws,sp", [(32, 16), (48, 24)])
def test_features_other_window_sizes(cuda, ws, sp):
    """The cost volume's generic window width (ws/4 = 8 and 12 downsampled px) against the
    oracle."""
    import torch

    Nx, Ny = 400, 336
    s = P.synth_params(Nx, Ny, ppp=0.05, field=P.PIV_FIELD_VORTEX, a=4.0, b=100.0, c=0.0, seed=6)
    f1, f2 = P.synth_pair(s)
    p = P.default_params(Nx=Nx, Ny=Ny, if_mhe=0, ws_x1=ws, ws_y1=ws, spacing_x1=sp, spacing_y1=sp, Npass1=1,
                         ws_x2=32, ws_y2=32, spacing_x2=16, spacing_y2=16, Npass2=0)
    with P.Engine(p) as e, P.PredictorNet(seed=1) as net:
        e.set_images(f1, f2)
        e.prep()
        g = e.geom
        H, W = g["Ny_vec"][0], g["Nx_vec"][0]
        out = torch.empty(81 * H * W, dtype=torch.float32, device="cuda")
        e.features(net, out)
        e.synchronize()
        got = out.cpu().numpy().reshape(81, H, W)
    want = L.features(f1, f2, W, H, sp, sp, g["Nx_left"][0], g["Ny_left"][0], ws, ws)
    assert np.abs(got - want).max() < 2e-5


def _batch(seed, N, H, W):
    rng = np.random.default_rng(seed)
    x = rng.normal(0, 0.5, (N, 81, H, W)).astype(np.float32)
    label = rng.normal(0, 1, (N, 2, H, W)).astype(np.float32)
    mask = (rng.random((N, H, W)) > 0.15).astype(np.float32)
    return x, label, mask


@pytest.mark.parametrize("shape", [(2, 9, 11), (1, 16, 16), (3, 5, 6)])
def test_forward_loss_and_gradient_match_oracle(cuda, shape):
    import torch

    N, H, W = shape
    x, label, mask = _batch(7 + H, N, H, W)
    with P.PredictorNet(seed=3) as net:
        params = net.params()
        # nonzero biases so their gradients and the bias path are exercised
        _, P_ = L.layout()
        rng = np.random.default_rng(1)
        for (w_off, b_off, cout, cin) in L.layout()[0]:
            params[b_off: b_off + cout] = rng.normal(0, 0.05, cout)
        net.set_params(params)
        dx = torch.from_numpy(x).cuda()
        dl = torch.from_numpy(label).cuda()
        dm = torch.from_numpy(mask).cuda()
        out = torch.empty((N, 2, H, W), dtype=torch.float32, device="cuda")
        net.forward(dx, N, H, W, out)
        net.synchronize()
        loss = net.loss_grad(dx, dl, dm, N, H, W)
        grad = net.grads()
        got_out = out.cpu().numpy()
    want_loss, want_grad, want_out = L.loss_and_grad(params.astype(np.float64), x.astype(np.float64),
                                                    label.astype(np.float64), mask.astype(np.float64))
    assert np.abs(got_out - want_out).max() <= 1e-4 * (1 + np.abs(want_out).max())
    assert abs(loss - want_loss) <= 1e-5 * (1 + abs(want_loss))
    lay, _ = L.layout()
    for i, (w_off, b_off, cout, cin) in enumerate(lay):
        for lo, hi in ((w_off, b_off), (b_off, b_off + cout)):
            g, w = grad[lo:hi], want_grad[lo:hi]
            err = np.linalg.norm(g - w) / max(np.linalg.norm(w), 1e-12)
            assert err < 2e-4, (i, lo == b_off, err)


def test_tensor_core_forward_matches_oracle_and_simt(cuda, monkeypatch):
    """At 130 x 132 the wide stride-1 layers (0, 1 and 11 with 32 output channels, 3 and 10
    with 64, the last two through upsampling and concatenation) run on the tcgen05
    convolution, with partial tiles at both edges: its forward output, the loss and the
    gradients match the oracle, and its output matches the SIMT kernels'."""
    import torch

    N, H, W = 1, 130, 132
    x, label, mask = _batch(21, N, H, W)
    dx = torch.from_numpy(x).cuda()
    dl = torch.from_numpy(label).cuda()
    dm = torch.from_numpy(mask).cuda()
    outs = {}
    for tc in ("1", "0"):
        monkeypatch.setenv("PIV_NET_TC", tc)
        with P.PredictorNet(seed=6) as net:
            params = net.params()
            rng = np.random.default_rng(2)
            for (w_off, b_off, cout, cin) in L.layout()[0]:
                params[b_off: b_off + cout] = rng.normal(0, 0.05, cout)
            net.set_params(params)
            out = torch.empty((N, 2, H, W), dtype=torch.float32, device="cuda")
            net.forward(dx, N, H, W, out)
            net.synchronize()
            outs[tc] = out.cpu().numpy()
            if tc == "1":
                loss = net.loss_grad(dx, dl, dm, N, H, W)
                grad = net.grads()
    want_loss, want_grad, want_out = L.loss_and_grad(params.astype(np.float64), x.astype(np.float64),
                                                    label.astype(np.float64), mask.astype(np.float64))
    scale = 1 + np.abs(want_out).max()
    assert np.abs(outs["1"] - want_out).max() <= 1e-4 * scale
    assert np.abs(outs["1"] - outs["0"]).max() <= 1e-4 * scale
    assert abs(loss - want_loss) <= 1e-5 * (1 + abs(want_loss))
    # the backward kernels read the tensor-core forward's activations (split-BF16 operands,
    # about 1e-5 relative): the few pre-activations within that of zero take the other side
    # of the LeakyReLU kink, which moves the 17k-pixel gradient sums of the layers computed
    # on the tensor cores by up to about 1e-3 relative (SIMT forward: 1e-6, the bar above)
    for i, (w_off, b_off, cout, cin) in enumerate(L.layout()[0]):
        for lo, hi in ((w_off, b_off), (b_off, b_off + cout)):
            g, w = grad[lo:hi], want_grad[lo:hi]
            err = np.linalg.norm(g - w) / max(np.linalg.norm(w), 1e-12)
            assert err < 3e-3, (i, lo == b_off, err)


def test_adam_step(cuda):
    import torch

    N, H, W = 2, 8, 8
    x, label, mask = _batch(3, N, H, W)
    with P.PredictorNet(seed=9) as net:
        p0 = net.params()
        dx = torch.from_numpy(x).cuda()
        dl = torch.from_numpy(label).cuda()
        dm = torch.from_numpy(mask).cuda()
        l0 = net.loss_grad(dx, dl, dm, N, H, W)
        g = net.grads()
        lr = 1e-3
        net.adam_step(lr)
        net.synchronize()
        p1 = net.params()
        # first step: m_hat = g, v_hat = g^2, so p1 = p0 - lr * g / (|g| + 1e-8)
        want = p0 - lr * g / (np.abs(g) + 1e-8)
        assert np.abs(p1 - want).max() <= 1e-6 + 1e-6 * np.abs(p0).max()
        for _ in range(20):
            net.loss_grad(dx, dl, dm, N, H, W)
            net.adam_step(lr)
        l1 = net.loss_grad(dx, dl, dm, N, H, W)
    assert l1 < 0.9 * l0


def test_save_load_round_trip(cuda, tmp_path):
    with P.PredictorNet(seed=4) as a, P.PredictorNet(seed=5) as b:
        assert not np.array_equal(a.params(), b.params())
        a.save(tmp_path / "w.bin")
        b.load(tmp_path / "w.bin")
        assert np.array_equal(a.params(), b.params())
        (tmp_path / "bad.bin").write_bytes(b"PIVNET01" + (3).to_bytes(8, "little"))
        with pytest.raises(P.PivError):
            b.load(tmp_path / "bad.bin")


def test_learned_pair_judge_and_fallback(cuda):
    Nx, Ny = 640, 512
    s = P.synth_params(Nx, Ny, ppp=0.05, field=P.PIV_FIELD_VORTEX, a=5.0, b=150.0, c=0.001, seed=21)
    f1, f2 = P.synth_pair(s)
    p = P.default_params(Nx=Nx, Ny=Ny, if_mhe=1, mhe_ws=40, mhe_thresh=0.91, ws_x1=64, ws_y1=64, spacing_x1=32,
                         spacing_y1=32, Npass1=2, ws_x2=32, ws_y2=32, spacing_x2=16, spacing_y2=16, Npass2=3)
    with P.Engine(p) as e, P.PredictorNet(seed=2) as net:
        e.set_images(f1, f2)
        e.run_pair()
        plain = [e.field(k) for k in (2, 3)]
        # a judge that cannot pass: the pair falls back to the plain method, bit for bit
        r = e.run_pair_learned(net, max_reject_frac=-1.0, max_rms_px=0.0)
        assert r["fell_back"]
        for a, b in zip([e.field(k) for k in (2, 3)], plain):
            for u, v in zip(a, b):
                assert np.array_equal(u, v)
        # a judge that always passes: the learned form's own grid-2 field
        r = e.run_pair_learned(net, max_reject_frac=2.0, max_rms_px=1e9)
        assert not r["fell_back"]
        assert 0.0 <= r["reject_frac"] <= 1.0 and np.isfinite(r["rms_px"])
        e.synchronize()
        x, y, dx, dy, v = e.field(3)
        assert np.isfinite(dx).all() and np.isfinite(dy).all()


WEIGHTS = P.LIB_PATH.parent.parent / "weights" / "predictor.bin"


def _rms(a, b, mask=None):
    d2 = (a[0] - b[0]) ** 2 + (a[1] - b[1]) ** 2
    if mask is not None:
        d2 = d2[mask]
    return float(np.sqrt(d2.mean()))


def test_trained_predictor_gain(cuda):
    """The committed predictor on a held-out pair (not in its training set: other size,
    seed and field): its grid-1 field is far closer to the truth than the zero predictor
    the plain method starts from and close to the plain method's own converged grid-1
    field; the learned pair passes the judge and ends as accurate as the plain pair."""
    import torch

    assert WEIGHTS.exists(), "train_predictor.py writes the weights"
    Nx, Ny = 2048, 1536
    s = P.synth_params(Nx, Ny, ppp=0.04, field=P.PIV_FIELD_VORTEX, a=9.0, b=500.0, c=0.002, seed=424242)
    f1, f2 = P.synth_pair(s)
    p = P.default_params(Nx=Nx, Ny=Ny, if_mhe=1, mhe_ws=40, mhe_thresh=0.91, ws_x1=64, ws_y1=64, spacing_x1=32,
                         spacing_y1=32, Npass1=2, ws_x2=32, ws_y2=32, spacing_x2=16, spacing_y2=16, Npass2=3,
                         insert_threshold_p1=2.0, insert_threshold_p2=2.0)
    with P.Engine(p) as e, P.PredictorNet(weights=WEIGHTS) as net:
        e.set_images(f1, f2)
        e.run_pair()
        x1, y1, px, py, _ = e.field(1)
        x2, y2, dx, dy, v2 = e.field(3)
        H, W = e.geom["Ny_vec"][0], e.geom["Nx_vec"][0]
        cv = torch.empty(81 * H * W, dtype=torch.float32, device="cuda")
        out = torch.empty(2 * H * W, dtype=torch.float32, device="cuda")
        e.features(net, cv)
        e.synchronize()
        net.forward(cv, 1, H, W, out)
        net.synchronize()
        pred = out.cpu().numpy().reshape(2, -1) * 4.0
        truth1 = P.synth_field(s, x1, y1)
        err_pred = _rms(pred, truth1)
        err_zero = _rms(np.zeros_like(pred), truth1)
        err_plain1 = _rms((px, py), truth1)
        print(f"grid 1 vs truth: predictor {err_pred:.3f} px, zero {err_zero:.3f} px, plain {err_plain1:.3f} px")
        assert err_pred < 0.1 * err_zero
        assert err_pred < 0.5
        truth2 = P.synth_field(s, x2, y2)
        acc_plain = _rms((dx, dy), truth2, v2 == 1)
        r = e.run_pair_learned(net)
        x2l, y2l, dxl, dyl, v2l = e.field(3)
        acc_learned = _rms((dxl, dyl), truth2, v2l == 1)
        print(f"grid 2 vs truth: plain {acc_plain:.4f} px, learned {acc_learned:.4f} px, judge {r}")
        assert not r["fell_back"]
        assert acc_learned <= acc_plain + 0.01


def test_learned_pair_tensor_core_layers(cuda, monkeypatch):
    """At 4096 x 2160 the grid-1 vector grid (127 x 67) is large enough for the predictor's
    level-0 convolutions to run on the tensor cores inside the learned pair's graph: the
    pair passes the judge with them on and off, and the final grid-2 fields agree to a
    small fraction of a pixel (the split-BF16 activations move the prediction by ~1e-5
    relative; the grid-2 passes then converge on the same peaks)."""
    assert WEIGHTS.exists()
    Nx, Ny = 4096, 2160
    s = P.synth_params(Nx, Ny, ppp=0.04, field=P.PIV_FIELD_FOURIER, a=300.0, b=2000.0, c=8.0, seed=777)
    f1, f2 = P.synth_pair(s)
    p = P.default_params(Nx=Nx, Ny=Ny, if_mhe=1, mhe_ws=40, mhe_thresh=0.91, ws_x1=64, ws_y1=64, spacing_x1=32,
                         spacing_y1=32, Npass1=2, ws_x2=32, ws_y2=32, spacing_x2=16, spacing_y2=16, Npass2=3,
                         insert_threshold_p1=2.0, insert_threshold_p2=2.0)
    fields = {}
    for tc in ("1", "0"):
        monkeypatch.setenv("PIV_NET_TC", tc)
        with P.Engine(p) as e, P.PredictorNet(weights=WEIGHTS) as net:
            assert e.geom["Ny_vec"][0] * e.geom["Nx_vec"][0] >= 4096
            e.set_images(f1, f2)
            r = e.run_pair_learned(net)
            assert not r["fell_back"], r
            fields[tc] = e.field(3)
    x, y, dx1, dy1, v1 = fields["1"]
    _, _, dx0, dy0, v0 = fields["0"]
    both = (v1 == 1) & (v0 == 1)
    assert both.mean() > 0.99
    d = np.hypot(dx1 - dx0, dy1 - dy0)[both]
    assert np.quantile(d, 0.999) < 0.01 and d.max() < 0.5
    u, w = P.synth_field(s, x, y)
    assert np.sqrt(np.mean(((dx1 - u) ** 2 + (dy1 - w) ** 2)[v1 == 1])) < 0.1
