"""CPU oracle of the learned entry/stop MLP: float64 forward and backward.

TEST INFRASTRUCTURE ONLY (the checker of the GPU training kernels in
2020_song_ex_b200/csrc/song_learn.cu).  The network and packed parameter
layout are the library's: 24 inputs, two ReLU layers of 64, `out` outputs;
params = [W1 (64x24), b1 (64), W2 (64x64), b2 (64), W3 (out x 64), b3 (out)].
The loss is the batch mean of sample_weight * loss_b with
  loss_kind 0: binary cross-entropy with logits (out = 1, y in [0, 1]),
  loss_kind 1: softmax cross-entropy (y = class index).
"""
from __future__ import annotations

import numpy as np

FEAT, HID = 24, 64


def n_params(out: int) -> int:
    return HID * FEAT + HID + HID * HID + HID + out * HID + out


def unpack(p: np.ndarray, out: int):
    p = np.asarray(p, dtype=np.float64)
    o = 0
    W1 = p[o:o + HID * FEAT].reshape(HID, FEAT); o += HID * FEAT
    b1 = p[o:o + HID]; o += HID
    W2 = p[o:o + HID * HID].reshape(HID, HID); o += HID * HID
    b2 = p[o:o + HID]; o += HID
    W3 = p[o:o + out * HID].reshape(out, HID); o += out * HID
    b3 = p[o:o + out]; o += out
    assert o == p.size
    return W1, b1, W2, b2, W3, b3


def forward(p, out, x):
    W1, b1, W2, b2, W3, b3 = unpack(p, out)
    x = np.asarray(x, dtype=np.float64)
    a1 = x @ W1.T + b1
    h1 = np.maximum(a1, 0)
    a2 = h1 @ W2.T + b2
    h2 = np.maximum(a2, 0)
    z = h2 @ W3.T + b3
    return z, (x, a1, h1, a2, h2)


def loss_and_grad(p, out, loss_kind, x, y, w=None):
    """Mean weighted loss and its gradient w.r.t. the packed parameters."""
    W1, b1, W2, b2, W3, b3 = unpack(p, out)
    z, (x, a1, h1, a2, h2) = forward(p, out, x)
    B = x.shape[0]
    w = np.ones(B) if w is None else np.asarray(w, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    if loss_kind == 0:
        zz = z[:, 0]
        loss = np.maximum(zz, 0) - zz * y + np.log1p(np.exp(-np.abs(zz)))
        dz = ((1 / (1 + np.exp(-zz)) - y) * w / B)[:, None]
    else:
        zm = z.max(axis=1, keepdims=True)
        e = np.exp(z - zm)
        sm = e / e.sum(axis=1, keepdims=True)
        yi = y.astype(np.int64)
        loss = np.log(e.sum(axis=1)) + zm[:, 0] - z[np.arange(B), yi]
        oh = np.zeros_like(sm)
        oh[np.arange(B), yi] = 1
        dz = (sm - oh) * w[:, None] / B
    gW3 = dz.T @ h2
    gb3 = dz.sum(0)
    d2 = (dz @ W3) * (a2 > 0)
    gW2 = d2.T @ h1
    gb2 = d2.sum(0)
    d1 = (d2 @ W2) * (a1 > 0)
    gW1 = d1.T @ x
    gb1 = d1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return float((loss * w).mean()), g
