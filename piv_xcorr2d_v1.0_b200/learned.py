"""Training and evaluation of the learned grid-1 predictor (host side of piv_net_*).

Training pairs come from the synthetic generator on the GPU (piv_synth_pair_device):
1024x1024 frames, 0.02-0.08 particles/px, displacement fields that are either a sum of
8 random Fourier modes (wavelengths 200-2000 px, at most 12 px) or a Lamb-Oseen vortex
(peak 2-12 px, core 150-1200 px) plus a shear of up to 0.008 px/px (4 px at the edges).  Each pair's label is the field the plain
method itself converges on: the engine's filtered grid-1 field after three grid-1 passes
(MHE 40 px / 0.91, 64x64 windows at 32 px); its input is the engine's cost volume of the
same prepared frames (piv_net_features).  The network trains on them with the hand-
written kernels (piv_net_loss_grad, piv_net_adam_step), Adam with a cosine learning
rate, random flips of the vector grid (mirroring the cost volume's shift axes and the
label's sign) as augmentation.  PyTorch is used for device buffers and batch gathering
only.
"""
from __future__ import annotations

import math
import time

import numpy as np

from . import (PIV_FIELD_FOURIER, PIV_FIELD_VORTEX, Engine, PredictorNet, default_params, synth_field,
               synth_pair_device, synth_params)

DOWN = 4
TRAIN_SIZE = 1024


def label_params(Nx=TRAIN_SIZE, Ny=TRAIN_SIZE, **kw):
    """Engine parameters of the label runs: the plain method's grid 1, converged."""
    base = dict(Nx=Nx, Ny=Ny, if_mhe=1, mhe_ws=40, mhe_thresh=0.91, ws_x1=64, ws_y1=64, spacing_x1=32,
                spacing_y1=32, Npass1=3, ws_x2=32, ws_y2=32, spacing_x2=16, spacing_y2=16, Npass2=0,
                insert_threshold_p1=2.0, insert_threshold_p2=2.0)
    base.update(kw)
    return default_params(**base)


def draw_pair(rng, size=TRAIN_SIZE, seed=0):
    """Synthetic parameters of one training pair."""
    ppp = rng.uniform(0.02, 0.08)
    if rng.random() < 0.7:
        return synth_params(size, size, ppp=ppp, field=PIV_FIELD_FOURIER, a=200.0, b=2000.0,
                            c=float(rng.uniform(2.0, 12.0)), seed=seed)
    return synth_params(size, size, ppp=ppp, field=PIV_FIELD_VORTEX, a=float(rng.uniform(2.0, 12.0)),
                        b=float(rng.uniform(150.0, 1200.0)), c=float(rng.uniform(-0.008, 0.008)), seed=seed)


def make_dataset(n_pairs, seed=1, size=TRAIN_SIZE, device="cuda", log=None):
    """Generates n_pairs labelled pairs on the GPU.  Returns a dict of device tensors:
    x [n][81][H][W], label [n][2][H][W] (downsampled px), mask [n][H][W] and truth
    [n][2][H][W] (the generator's field at the vector positions, downsampled px)."""
    import torch

    rng = np.random.default_rng(seed)
    p = label_params(size, size)
    net = PredictorNet(seed=1)  # only its feature scratch is used here
    e = Engine(p)
    g = e.geom
    H, W = g["Ny_vec"][0], g["Nx_vec"][0]
    x = torch.empty((n_pairs, 81, H, W), dtype=torch.float32, device=device)
    label = torch.empty((n_pairs, 2, H, W), dtype=torch.float32, device=device)
    mask = torch.empty((n_pairs, H, W), dtype=torch.float32, device=device)
    truth = torch.empty((n_pairs, 2, H, W), dtype=torch.float32, device=device)
    d1 = torch.empty(size * size, dtype=torch.uint8, device=device)
    d2 = torch.empty_like(d1)
    scratch = torch.empty(2 * size * size, dtype=torch.float32, device=device)
    torch.cuda.synchronize()
    e.set_device_images(d1.data_ptr(), d2.data_ptr())
    t0 = time.time()
    for k in range(n_pairs):
        s = draw_pair(rng, size, seed=seed * 1000003 + k)
        synth_pair_device(s, d1, d2, scratch, e.stream())
        e.run_pair()
        e.features(net, x[k])
        xs, ys, dx, dy, v = e.field(1)  # synchronises the engine stream
        lab = np.stack([dx, dy]).reshape(2, H, W) / DOWN
        u, w = synth_field(s, xs, ys)
        tru = np.stack([u, w]).reshape(2, H, W) / DOWN
        label[k].copy_(torch.from_numpy(lab))
        mask[k].copy_(torch.from_numpy((v == 1).astype(np.float32).reshape(H, W)))
        truth[k].copy_(torch.from_numpy(tru))
        if log and (k + 1) % 2000 == 0:
            log(f"  {k + 1} pairs, {time.time() - t0:.1f} s")
    torch.cuda.synchronize()
    e.close()
    net.close()
    return {"x": x, "label": label, "mask": mask, "truth": truth, "H": H, "W": W}


def _flip(xb, lb, mb, fx, fy):
    """Mirror a batch on the vector grid: x-flip mirrors the shift axis dx and negates the
    label's x component; likewise for y."""
    import torch

    if fx:
        xb = xb.flip(3).view(xb.shape[0], 9, 9, xb.shape[2], xb.shape[3]).flip(2).reshape(xb.shape)
        lb = lb.flip(3)
        lb = torch.stack([-lb[:, 0], lb[:, 1]], 1)
        mb = mb.flip(2)
    if fy:
        xb = xb.flip(2).view(xb.shape[0], 9, 9, xb.shape[2], xb.shape[3]).flip(1).reshape(xb.shape)
        lb = lb.flip(2)
        lb = torch.stack([lb[:, 0], -lb[:, 1]], 1)
        mb = mb.flip(1)
    return xb.contiguous(), lb.contiguous(), mb.contiguous()


def evaluate(net: PredictorNet, data, idx, target="label", batch=64):
    """RMS vector error (image px) of the network on pairs idx against the labels or the
    truth, over masked vectors."""
    import torch

    H, W = data["H"], data["W"]
    se, cnt = 0.0, 0.0
    out = torch.empty((batch, 2, H, W), dtype=torch.float32, device=data["x"].device)
    for i in range(0, len(idx), batch):
        j = idx[i: i + batch]
        n = len(j)
        xb = data["x"][j].contiguous()
        net.forward(xb, n, H, W, out)
        net.synchronize()
        ref = data[target][j]
        m = data["mask"][j]
        d = (out[:n] - ref) * DOWN
        se += float(((d[:, 0] ** 2 + d[:, 1] ** 2) * m).sum())
        cnt += float(m.sum())
    return math.sqrt(se / max(cnt, 1.0))


def train(net: PredictorNet, data, epochs=30, batch=64, lr=1e-3, lr_min=1e-5, val_frac=0.05, seed=2, log=None):
    """Trains net in place; returns the history (per epoch: loss, val RMS vs label and truth)."""
    import torch

    n = data["x"].shape[0]
    H, W = data["H"], data["W"]
    rng = np.random.default_rng(seed)
    n_val = max(1, int(round(n * val_frac)))
    val = np.arange(n - n_val, n)
    tr = np.arange(n - n_val)
    steps = epochs * (len(tr) // batch)
    hist = []
    step = 0
    t0 = time.time()
    for ep in range(epochs):
        perm = rng.permutation(tr)
        tot = 0.0
        nb = len(tr) // batch
        for b in range(nb):
            j = torch.from_numpy(perm[b * batch: (b + 1) * batch]).to(data["x"].device)
            xb, lb, mb = data["x"][j], data["label"][j], data["mask"][j]
            xb, lb, mb = _flip(xb, lb, mb, bool(rng.integers(2)), bool(rng.integers(2)))
            torch.cuda.synchronize()
            loss = net.loss_grad(xb, lb, mb, batch, H, W)
            cur = lr_min + 0.5 * (lr - lr_min) * (1 + math.cos(math.pi * step / max(steps, 1)))
            net.adam_step(cur)
            tot += loss
            step += 1
        vl = evaluate(net, data, val, "label")
        vt = evaluate(net, data, val, "truth")
        hist.append({"epoch": ep + 1, "loss": tot / max(nb, 1), "val_rms_label_px": vl, "val_rms_truth_px": vt,
                     "seconds": time.time() - t0})
        if log:
            log(f"epoch {ep + 1}: loss {tot / max(nb, 1):.4f}  val RMS vs label {vl:.3f} px, vs truth {vt:.3f} px"
                f"  ({time.time() - t0:.0f} s)")
    return hist
