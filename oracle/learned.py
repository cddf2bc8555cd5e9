"""NumPy restatement of the learned grid-1 predictor (features, network, loss, gradients).

TEST INFRASTRUCTURE ONLY: the checker for the predictor's CUDA kernels
(piv_xcorr2d_v1.0_b200/csrc/learned.cu).  Only tests/ may use it.  The predictor has no
counterpart in the reference (it replaces the plain grid-1 passes that X/main.cpp:290-300
drives), so this file restates the design itself, in float64:

  features  4x4 box average of each frame (grey/255), global mean removed; at each grid-1
            vector (window centre ix*sp - Nx_left + ws/2, rounded to the nearest 4-px
            block boundary) a (ws/4)^2 window of frame 1 against frame 2 shifted by
            dx, dy in [-4, 4] (downsampled px), normalised by sqrt(E1 * E2) with E2 the
            frame-2 window energy at zero shift; outside the image the frames are 0.
  network   13 3x3 convolutions (padding 1) of the U-Net in LAYERS; weights rounded to
            BF16 (round to nearest even) exactly as the kernels read them.
  loss      Charbonnier, eps 0.01: mean over masked vectors of
            sum_c sqrt(e_c^2 + eps^2) - eps.
The analytic backward pass is checked against central finite differences by
tests/test_learned_oracle.py, which pins this restatement before it is used.
"""
from __future__ import annotations

import numpy as np

SLOPE = 0.1
RADIUS = 4
DOWN = 4
EPS = 0.01

# (a, ca, b, cb, up, cout, stride, act): layer i reads tensor a (upsampled x2 if up)
# concatenated with tensor b and writes tensor i + 1; tensor 0 is the cost volume
LAYERS = [
    (0, 81, -1, 0, 0, 32, 1, 1),
    (1, 32, -1, 0, 0, 32, 1, 1),
    (2, 32, -1, 0, 0, 64, 2, 1),
    (3, 64, -1, 0, 0, 64, 1, 1),
    (4, 64, -1, 0, 0, 96, 2, 1),
    (5, 96, -1, 0, 0, 96, 1, 1),
    (6, 96, -1, 0, 0, 128, 2, 1),
    (7, 128, -1, 0, 0, 128, 1, 1),
    (8, 128, 6, 96, 1, 96, 1, 1),
    (9, 96, -1, 0, 0, 96, 1, 1),
    (10, 96, 4, 64, 1, 64, 1, 1),
    (11, 64, 2, 32, 1, 32, 1, 1),
    (12, 32, -1, 0, 0, 2, 1, 0),
]


def layout():
    """[(w_off, b_off, cout, cin)] of the flat parameter vector (weights then biases)."""
    out, off = [], 0
    for (_, ca, _, cb, _, cout, _, _) in LAYERS:
        cin = ca + cb
        out.append((off, off + cout * cin * 9, cout, cin))
        off += cout * cin * 9 + cout
    return out, off


def bf16(x: np.ndarray) -> np.ndarray:
    """float32 -> nearest BF16 (ties to even), returned as float32."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


# ---------------------------------------------------------------- features

def down4(img: np.ndarray) -> np.ndarray:
    ny, nx = img.shape[0] // DOWN, img.shape[1] // DOWN
    a = img[: ny * DOWN, : nx * DOWN].astype(np.float64).reshape(ny, DOWN, nx, DOWN)
    return a.sum(axis=(1, 3)) / (16.0 * 255.0)


def features(img1, img2, Nx_vec, Ny_vec, sp_x, sp_y, Nx_left, Ny_left, ws_x, ws_y):
    d1, d2 = down4(img1), down4(img2)
    d1 = d1 - d1.mean()
    d2 = d2 - d2.mean()
    H4, W4 = d1.shape
    Wd, Hd, R = ws_x // DOWN, ws_y // DOWN, RADIUS
    S = 2 * R + 1
    out = np.zeros((S * S, Ny_vec, Nx_vec))

    def region(d, y0, x0, h, w):
        r = np.zeros((h, w))
        ys, xs = max(y0, 0), max(x0, 0)
        ye, xe = min(y0 + h, H4), min(x0 + w, W4)
        if ye > ys and xe > xs:
            r[ys - y0: ye - y0, xs - x0: xe - x0] = d[ys:ye, xs:xe]
        return r

    for iy in range(Ny_vec):
        for ix in range(Nx_vec):
            cx = ix * sp_x - Nx_left + ws_x // 2
            cy = iy * sp_y - Ny_left + ws_y // 2
            dcx, dcy = (cx + DOWN // 2) >> 2, (cy + DOWN // 2) >> 2
            x0, y0 = dcx - Wd // 2, dcy - Hd // 2
            w1 = region(d1, y0, x0, Hd, Wd)
            w2 = region(d2, y0 - R, x0 - R, Hd + 2 * R, Wd + 2 * R)
            e1 = (w1 * w1).sum()
            c2 = w2[R: R + Hd, R: R + Wd]
            e2 = (c2 * c2).sum()
            den = e1 * e2
            for dy in range(S):
                for dx in range(S):
                    acc = (w1 * w2[dy: dy + Hd, dx: dx + Wd]).sum()
                    out[dy * S + dx, iy, ix] = acc / np.sqrt(den) if den > 0 else 0.0
    return out


# ---------------------------------------------------------------- network

def _levels(H, W):
    hs, ws = [H], [W]
    for _ in range(3):
        hs.append((hs[-1] + 1) // 2)
        ws.append((ws[-1] + 1) // 2)
    return hs, ws


def _im2col(x, stride, Ho, Wo):
    """x [N][C][H][W] -> [N][C*9][Ho*Wo] for a 3x3 kernel, padding 1."""
    N, Cc, H, W = x.shape
    xp = np.zeros((N, Cc, H + 2, W + 2), x.dtype)
    xp[:, :, 1:-1, 1:-1] = x
    cols = np.empty((N, Cc, 9, Ho, Wo), x.dtype)
    for ky in range(3):
        for kx in range(3):
            cols[:, :, ky * 3 + kx] = xp[:, :, ky: ky + stride * (Ho - 1) + 1: stride,
                                         kx: kx + stride * (Wo - 1) + 1: stride]
    return cols.reshape(N, Cc * 9, Ho * Wo)


def _col2im(cols, shape, stride, Ho, Wo):
    N, Cc, H, W = shape
    cols = cols.reshape(N, Cc, 9, Ho, Wo)
    xp = np.zeros((N, Cc, H + 2, W + 2), cols.dtype)
    for ky in range(3):
        for kx in range(3):
            xp[:, :, ky: ky + stride * (Ho - 1) + 1: stride, kx: kx + stride * (Wo - 1) + 1: stride] += cols[:, :, ky * 3 + kx]
    return xp[:, :, 1:-1, 1:-1]


def _up(x, H, W):
    return np.repeat(np.repeat(x, 2, axis=2), 2, axis=3)[:, :, :H, :W]


def _weights(params, w_off, cout, cin, use_bf16):
    w = params[w_off: w_off + cout * cin * 9]
    w = bf16(w.astype(np.float32)) if use_bf16 else w
    return w.astype(np.float64).reshape(cout, cin * 9)


def _input_of(i, t, hs, ws):
    a, ca, b, cb, up, cout, stride, act = LAYERS[i]
    xa = t[a]
    if up:
        Hin, Win = t[b].shape[2], t[b].shape[3]
        xa = _up(xa, Hin, Win)
    return np.concatenate([xa, t[b]], axis=1) if b >= 0 else xa


def forward(params, x, use_bf16=True):
    """params: flat float32 vector; x: [N][81][H][W].  Returns the list of tensors."""
    lay, _ = layout()
    N, _, H, W = x.shape
    hs, ws = _levels(H, W)
    level = [0, 0, 0, 1, 1, 2, 2, 3, 3, 2, 2, 1, 0, 0]
    t = [x.astype(np.float64)]
    for i, (a, ca, b, cb, up, cout, stride, act) in enumerate(LAYERS):
        w_off, b_off, _, cin = lay[i]
        w = _weights(params, w_off, cout, cin, use_bf16)
        bias = params[b_off: b_off + cout].astype(np.float64)
        xin = _input_of(i, t, hs, ws)
        Ho, Wo = hs[level[i + 1]], ws[level[i + 1]]
        cols = _im2col(xin, stride, Ho, Wo)
        y = np.einsum("ok,nkp->nop", w, cols) + bias[None, :, None]
        y = y.reshape(N, cout, Ho, Wo)
        if act:
            y = np.where(y > 0, y, SLOPE * y)
        t.append(y)
    return t


def loss_and_grad(params, x, label, mask, use_bf16=True):
    """Charbonnier loss over masked vectors and its gradient w.r.t. the flat parameters."""
    lay, P = layout()
    t = forward(params, x, use_bf16)
    N, _, H, W = x.shape
    hs, ws = _levels(H, W)
    level = [0, 0, 0, 1, 1, 2, 2, 3, 3, 2, 2, 1, 0, 0]
    cnt = mask.sum()
    inv = 1.0 / cnt if cnt > 0 else 0.0
    e = t[-1] - label
    r = np.sqrt(e * e + EPS * EPS)
    m = mask[:, None] * inv
    loss = float((m * (r - EPS)).sum())
    g = [np.zeros_like(a) for a in t]
    g[-1] = m * e / r
    grad = np.zeros(P)
    for i in range(len(LAYERS) - 1, -1, -1):
        a, ca, b, cb, up, cout, stride, act = LAYERS[i]
        w_off, b_off, _, cin = lay[i]
        w = _weights(params, w_off, cout, cin, use_bf16)
        gy = g[i + 1]
        if act:
            gy = np.where(t[i + 1] > 0, gy, SLOPE * gy)
        Ho, Wo = gy.shape[2], gy.shape[3]
        xin = _input_of(i, t, hs, ws)
        cols = _im2col(xin, stride, Ho, Wo)
        gyf = gy.reshape(N, cout, Ho * Wo)
        grad[w_off: w_off + cout * cin * 9] = np.einsum("nop,nkp->ok", gyf, cols).ravel()
        grad[b_off: b_off + cout] = gyf.sum(axis=(0, 2))
        if i == 0:
            continue
        gcols = np.einsum("ok,nop->nkp", w, gyf)
        gin = _col2im(gcols, xin.shape, stride, Ho, Wo)
        ga = gin[:, :ca]
        if up:
            Hc, Wc = t[a].shape[2], t[a].shape[3]
            acc = np.zeros((N, ca, 2 * Hc, 2 * Wc))
            acc[:, :, : ga.shape[2], : ga.shape[3]] = ga
            ga = acc.reshape(N, ca, Hc, 2, Wc, 2).sum(axis=(3, 5))
        g[a] += ga
        if b >= 0:
            g[b] += gin[:, ca:]
    return loss, grad, t[-1]
