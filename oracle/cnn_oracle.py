"""FP64 numpy forward and backward of the orientation-proposer network.

TEST INFRASTRUCTURE ONLY: the checker for the CUDA network in
bsoft_b200/csrc/cnn.cu (layer layout, parameter order, loss and gradients);
nothing in the product imports it.  The network has no counterpart in the
reference, so this oracle is pinned by finite differences of its own loss
(tests/test_cnn_oracle.py) rather than by reference output.

Conventions shared with the CUDA code:
  activations NHWC; convolution 3x3, stride 2, padding 1, im2col column
  index (ky * 3 + kx) * cin + ci; weights W[cout][ky][kx][cin];
  parameters in the order conv1..conv6 (W, b), fc1 (W, b), fc2 (W, b);
  the network uses the weights rounded to BF16 (round to nearest even);
  input images normalised to zero mean and unit variance (population);
  head: b1 = a1/|a1|, b2 = (a2 - (b1.a2) b1)/|.|, b3 = b1 x b2,
  R = [b1 b2 b3] (columns), loss = mean |R - R*|^2 + lambda |t - t*|^2.
"""
from __future__ import annotations

import numpy as np

NOUT = 8


def bf16_round(w: np.ndarray) -> np.ndarray:
    """Round float32 values to the nearest BF16 (ties to even), as float64."""
    a = np.ascontiguousarray(w, dtype=np.float32).view(np.uint32).astype(np.uint64)
    lsb = (a >> 16) & 1
    r = ((a + 0x7FFF + lsb) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def layout(box: int, channels, hidden: int):
    """[(name, shape)] of the parameters in the library's order."""
    out = []
    cin, h = 1, box
    for l, c in enumerate(channels):
        out.append((f"conv{l + 1}.W", (c, 3, 3, cin)))
        out.append((f"conv{l + 1}.b", (c,)))
        cin, h = c, h // 2
    out.append(("fc1.W", (hidden, h * h * cin)))
    out.append(("fc1.b", (hidden,)))
    out.append(("fc2.W", (NOUT, hidden)))
    out.append(("fc2.b", (NOUT,)))
    return out


def unpack(flat: np.ndarray, box: int, channels, hidden: int):
    params, off = [], 0
    for _, shape in layout(box, channels, hidden):
        n = int(np.prod(shape))
        params.append(flat[off:off + n].reshape(shape))
        off += n
    assert off == flat.size
    return params


def _im2col(x):
    B, H, W, C = x.shape
    Ho, Wo = H // 2, W // 2
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (0, 0)))
    cols = [xp[:, ky:ky + 2 * Ho:2, kx:kx + 2 * Wo:2, :] for ky in range(3) for kx in range(3)]
    return np.stack(cols, axis=3).reshape(B * Ho * Wo, 9 * C), (B, Ho, Wo)


def _col2im(gcol, shape_in):
    B, H, W, C = shape_in
    Ho, Wo = H // 2, W // 2
    g = gcol.reshape(B, Ho, Wo, 9, C)
    gxp = np.zeros((B, H + 2, W + 2, C))
    for ky in range(3):
        for kx in range(3):
            gxp[:, ky:ky + 2 * Ho:2, kx:kx + 2 * Wo:2, :] += g[:, :, :, ky * 3 + kx, :]
    return gxp[:, 1:H + 1, 1:W + 1, :]


def normalise(images: np.ndarray) -> np.ndarray:
    x = np.asarray(images, dtype=np.float64)
    B = x.shape[0]
    f = x.reshape(B, -1)
    mean = f.mean(axis=1)
    var = (f * f).mean(axis=1) - mean * mean
    inv = np.where(var > 1e-30, 1.0 / np.sqrt(np.maximum(var, 1e-300)), 1.0)
    return ((f - mean[:, None]) * inv[:, None]).reshape(x.shape)


def _head(o, tgt, lam):
    a1, a2, t = o[:, 0:3], o[:, 3:6], o[:, 6:8]
    n1 = np.linalg.norm(a1, axis=1, keepdims=True) + 1e-12
    b1 = a1 / n1
    d = (b1 * a2).sum(1, keepdims=True)
    u2 = a2 - d * b1
    n2 = np.linalg.norm(u2, axis=1, keepdims=True) + 1e-12
    b2 = u2 / n2
    b3 = np.cross(b1, b2)
    R = np.stack([b1, b2, b3], axis=2)                 # columns
    if tgt is None:
        return R, t, None, None
    Rt = tgt[:, :9].reshape(-1, 3, 3)
    tt = tgt[:, 9:11]
    B = o.shape[0]
    per = ((R - Rt) ** 2).sum((1, 2)) + lam * ((t - tt) ** 2).sum(1)
    gR = 2 * (R - Rt)
    gb1, gb2, gb3 = gR[:, :, 0], gR[:, :, 1], gR[:, :, 2]
    gb1 = gb1 + np.cross(b2, gb3)
    gb2 = gb2 + np.cross(gb3, b1)
    gu2 = (gb2 - (gb2 * b2).sum(1, keepdims=True) * b2) / n2
    gu2b1 = (gu2 * b1).sum(1, keepdims=True)
    ga2 = gu2 - gu2b1 * b1
    gb1 = gb1 - d * gu2 - a2 * gu2b1
    ga1 = (gb1 - (gb1 * b1).sum(1, keepdims=True) * b1) / n1
    go = np.concatenate([ga1, ga2, 2 * lam * (t - tt)], axis=1) / B
    return R, t, per.mean(), go


def forward_backward(flat_params, images, targets=None, box=None, channels=None, hidden=None, lam=0.05,
                     rounded=True):
    """Returns (R (B,3,3), t (B,2), loss, grads flat) in FP64; grads are
    with respect to the weights the network uses: the BF16 rounding of the
    given ones (rounded=False uses them as they are, for finite
    differences of the oracle itself)."""
    w = bf16_round(flat_params) if rounded else np.asarray(flat_params, dtype=np.float64)
    params = unpack(w, box, channels, hidden)
    nconv = len(channels)
    x = normalise(images)[..., None]
    acts, cols, shapes = [x], [], []
    for l in range(nconv):
        W, b = params[2 * l], params[2 * l + 1]
        col, (B, Ho, Wo) = _im2col(acts[-1])
        y = col @ W.reshape(W.shape[0], -1).T + b
        y = np.maximum(y, 0.0)
        cols.append(col)
        shapes.append(acts[-1].shape)
        acts.append(y.reshape(B, Ho, Wo, -1))
    W1, b1, W2, b2 = params[2 * nconv:]
    a6 = acts[-1].reshape(acts[-1].shape[0], -1)
    h = np.maximum(a6 @ W1.T + b1, 0.0)
    o = h @ W2.T + b2
    tgt = None if targets is None else np.asarray(targets, dtype=np.float64)
    R, t, loss, go = _head(o, tgt, lam)
    if tgt is None:
        return R, t, None, None
    grads = [None] * len(params)
    grads[2 * nconv + 2] = go.T @ h
    grads[2 * nconv + 3] = go.sum(0)
    gh = (go @ W2) * (h > 0)
    grads[2 * nconv] = gh.T @ a6
    grads[2 * nconv + 1] = gh.sum(0)
    ga = (gh @ W1).reshape(acts[-1].shape)
    for l in range(nconv - 1, -1, -1):
        W = params[2 * l]
        gy = (ga * (acts[l + 1] > 0)).reshape(-1, W.shape[0])
        grads[2 * l] = (gy.T @ cols[l]).reshape(W.shape)
        grads[2 * l + 1] = gy.sum(0)
        if l > 0:
            ga = _col2im(gy @ W.reshape(W.shape[0], -1), shapes[l])
    flat = np.concatenate([g.reshape(-1) for g in grads])
    return R, t, loss, flat
