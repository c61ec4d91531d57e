"""CPU oracle of the subtree-proposal network (test infrastructure only: the
tests and nothing else import it; the product path never does).

The reference has no learned component, so there is no reference code to pin
this against. It restates, in numpy, exactly the computation the CUDA path
performs, with the same BF16 rounding points:

  X   = bf16(features)                               (rays x 192, cols >= 144 zero)
  H_l = bf16(relu(H_{l-1} W_l^T + b_l)),  l = 1..3    (FP32 math)
  L   = H_3 W_4^T + b_4                               (FP32)
  G   = bf16((softmax(L) - onehot(label)) / B)
  dW_4 = G^T H_3,  db_4 = sum_rows G
  D_3 = bf16((G W_4) * [H_3 > 0]),  dW_3 = D_3^T H_2,  db_3 = sum_rows D_3
  D_2 = bf16((D_3 W_3) * [H_2 > 0]), dW_2 = D_2^T H_1,  db_2 = sum_rows D_2
  D_1 = bf16((D_2 W_2) * [H_1 > 0]), dW_1 = D_1^T X,    db_1 = sum_rows D_1

Products of BF16 values are exact in float64, so this oracle accumulates in
float64 and rounds once; the GPU accumulates in FP32 in another order, so the
two agree to a tolerance (stated in the tests), not bit for bit. With
`rounding=False` every BF16 rounding is skipped and the math is float64
throughout, which is what the finite-difference self-check of the backward
formulas uses.
"""
from __future__ import annotations

import numpy as np

FEATURES = 144
FEATURES_PAD = 192
FREQS = 12


def bf16(x) -> np.ndarray:
    """Round float32 values to the nearest BF16 (ties to even), kept as float32."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return (r & 0xFFFFFFFF).astype(np.uint32).view(np.float32)


def bf16_bits_to_f32(bits) -> np.ndarray:
    return (np.asarray(bits, dtype=np.uint16).astype(np.uint32) << 16).view(np.float32)


def features(orig: np.ndarray, dirs: np.ndarray, box, rounding: bool = True) -> np.ndarray:
    """(R, 192) features: u = ((o - c) * 2 / (hi - lo), d / |d|), then
    sin / cos(pi 2^j u_i) interleaved per input, j < 12."""
    o = np.asarray(orig, np.float32)[:, :3]
    d = np.asarray(dirs, np.float32)[:, :3]
    lo = np.asarray(box[:3], np.float32)
    hi = np.asarray(box[3:6], np.float32)
    c = np.float32(0.5) * (lo + hi)
    s = np.float32(2.0) / (hi - lo)
    uo = (o - c) * s
    ln = np.sqrt((d.astype(np.float64) ** 2).sum(1)).astype(np.float32)
    ud = np.where(ln[:, None] > 0, d / np.where(ln > 0, ln, 1)[:, None], 0).astype(np.float32)
    u = np.concatenate([uo, ud], 1).astype(np.float64)  # (R, 6)
    R = u.shape[0]
    f = np.zeros((R, FEATURES_PAD), np.float64)
    for i in range(6):
        for j in range(FREQS):
            a = np.pi * (2.0 ** j) * u[:, i]
            f[:, 24 * i + 2 * j] = np.sin(a)
            f[:, 24 * i + 2 * j + 1] = np.cos(a)
    f32 = f.astype(np.float32)
    return bf16(f32) if rounding else f


def _round(x, rounding):
    return bf16(x.astype(np.float32)) if rounding else x


def forward(X, W, b, rounding: bool = True):
    """Hidden activations [H1, H2, H3] and logits L."""
    H = []
    h = X.astype(np.float64)
    for l in range(3):
        z = h @ W[l].astype(np.float64).T + b[l].astype(np.float64)
        h = _round(np.maximum(z, 0.0), rounding).astype(np.float64)
        H.append(h)
    L = h @ W[3].astype(np.float64).T + b[3].astype(np.float64)
    if rounding:
        L = L.astype(np.float32).astype(np.float64)
    return H, L


def loss_and_grad_logits(L, labels, rounding: bool = True):
    B = L.shape[0]
    m = L.max(1, keepdims=True)
    e = np.exp(L - m)
    s = e.sum(1, keepdims=True)
    p = e / s
    loss = float(np.mean(np.log(s[:, 0]) + m[:, 0] - L[np.arange(B), labels]))
    g = p.copy()
    g[np.arange(B), labels] -= 1.0
    g /= B
    return loss, _round(g, rounding).astype(np.float64)


def backward(X, W, H, G, rounding: bool = True):
    """Weight and bias gradients (dW_1..4, db_1..4) from the logit gradient G."""
    acts = [X.astype(np.float64)] + H
    dW = [None] * 4
    db = [None] * 4
    D = G
    for l in range(3, -1, -1):
        dW[l] = D.T @ acts[l]
        db[l] = D.sum(0)
        if l > 0:
            Dn = (D @ W[l].astype(np.float64)) * (acts[l] > 0)
            D = _round(Dn, rounding).astype(np.float64)
    return dW, db


def train_grads(X, W, b, labels, rounding: bool = True):
    H, L = forward(X, W, b, rounding)
    loss, G = loss_and_grad_logits(L, labels, rounding)
    dW, db = backward(X, W, H, G, rounding)
    return loss, dW, db


def loss_only(X, W, b, labels):
    _, L = forward(X, W, b, rounding=False)
    loss, _ = loss_and_grad_logits(L, labels, rounding=False)
    return loss
