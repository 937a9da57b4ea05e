"""CPU restatement of the learned stop predictor (test infrastructure).

Restates, in numpy float32 with the same operation order, the product's MLP
kernels (parex_b200/csrc/pxr_mlp.cuh, pxr_mlp.cu): bf16 rounding of layer
inputs and gradient operands, float accumulation in input order, per-block
sample-order gradient sums, block-order reduction, the Adam step.  Forward,
gradient and Adam results are therefore expected bit for bit.  Also restates
the per-cluster features (in float64: compared with a tolerance, since the
product evaluates log10f/log2f) and a float64 gradient of the same network
without bf16 rounding, for a finite-difference check of the backward
formulas.  No reference counterpart: the reference has no learned part.
"""
from __future__ import annotations

import numpy as np

F_IN = 16
HIDDEN = 32
OFF_W1 = 0
OFF_B1 = OFF_W1 + HIDDEN * F_IN
OFF_W2 = OFF_B1 + HIDDEN
OFF_B2 = OFF_W2 + HIDDEN * HIDDEN
OFF_W3 = OFF_B2 + HIDDEN
OFF_B3 = OFF_W3 + HIDDEN
PARAMS = OFF_B3 + 1
BLOCK = 64
f32 = np.float32


def bf16(x) -> np.ndarray:
    """Round float32 values to bf16 (nearest even), returned as float32."""
    a = np.ascontiguousarray(x, dtype=f32)
    b = a.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(f32).reshape(a.shape)


def bf16_bits(x) -> np.ndarray:
    return (bf16(x).view(np.uint32) >> 16).astype(np.uint16)


def from_bits(w_bits) -> np.ndarray:
    return (np.asarray(w_bits, dtype=np.uint32) << 16).view(f32)


def _unpack(w):
    W1 = w[OFF_W1:OFF_B1].reshape(HIDDEN, F_IN)
    b1 = w[OFF_B1:OFF_W2]
    W2 = w[OFF_W2:OFF_B2].reshape(HIDDEN, HIDDEN)
    b2 = w[OFF_B2:OFF_W3]
    W3 = w[OFF_W3:OFF_B3]
    b3 = w[OFF_B3]
    return W1, b1, W2, b2, W3, b3


def forward(w_bits, norm, X):
    """y and the intermediates, as mlp_forward computes them."""
    w = from_bits(w_bits)
    W1, b1, W2, b2, W3, b3 = _unpack(w)
    X = np.asarray(X, dtype=f32)
    norm = np.asarray(norm, dtype=f32)
    n = X.shape[0]
    z = bf16((X - norm[None, :F_IN]) * norm[None, F_IN:])
    a1 = np.repeat(b1[None, :], n, axis=0)
    for i in range(F_IN):
        a1 = a1 + W1[None, :, i] * z[:, i:i + 1]
    h1 = bf16(np.maximum(a1, f32(0)))
    a2 = np.repeat(b2[None, :], n, axis=0)
    for i in range(HIDDEN):
        a2 = a2 + W2[None, :, i] * h1[:, i:i + 1]
    h2 = bf16(np.maximum(a2, f32(0)))
    y = np.full(n, b3, dtype=f32)
    for i in range(HIDDEN):
        y = y + W3[i] * h2[:, i]
    return y, dict(z=z, a1=a1, h1=h1, a2=a2, h2=h2)


def gradient(w_bits, norm, X, T, delta: float, over: float):
    """(mean gradient [PARAMS], mean loss) in the product's summation order."""
    w = from_bits(w_bits)
    W1, b1, W2, b2, W3, b3 = _unpack(w)
    y, act = forward(w_bits, norm, X)
    T = np.asarray(T, dtype=f32)
    delta, over = f32(delta), f32(over)
    e = y - T
    ae = np.abs(e)
    wt = np.where(e > 0, over, f32(1))
    quad = ae <= delta
    loss = wt * np.where(quad, (f32(0.5) * e) * e, delta * (ae - f32(0.5) * delta))
    g = wt * np.where(quad, e, np.copysign(delta, e))
    gb = bf16(g)
    d2 = bf16(np.where(act["a2"] > 0, W3[None, :] * gb[:, None], f32(0)))
    dh = np.zeros_like(d2)
    for o in range(HIDDEN):
        dh = dh + W2[None, o, :] * d2[:, o:o + 1]
    d1 = bf16(np.where(act["a1"] > 0, dh, f32(0)))
    z, h1, h2 = act["z"], act["h1"], act["h2"]
    n = X.shape[0]
    total = np.zeros(PARAMS + 1, dtype=f32)
    for b0 in range(0, n, BLOCK):
        acc = np.zeros(PARAMS + 1, dtype=f32)
        for s in range(b0, min(b0 + BLOCK, n)):
            part = np.empty(PARAMS + 1, dtype=f32)
            part[OFF_W1:OFF_B1] = (d1[s][:, None] * z[s][None, :]).ravel()
            part[OFF_B1:OFF_W2] = d1[s]
            part[OFF_W2:OFF_B2] = (d2[s][:, None] * h1[s][None, :]).ravel()
            part[OFF_B2:OFF_W3] = d2[s]
            part[OFF_W3:OFF_B3] = gb[s] * h2[s]
            part[OFF_B3] = gb[s]
            part[PARAMS] = loss[s]
            acc = acc + part
        total = total + acc
    mean = total / f32(n)
    return mean[:PARAMS], mean[PARAMS]


def adam_step(master, m, v, grad, step: int, lr: float, beta1: float, beta2: float, eps: float):
    """(master, m, v, weight bits) after one Adam step, as k_mlp_adam."""
    b1, b2 = f32(beta1), f32(beta2)
    c1 = f32(1.0 - float(b1) ** step)
    c2 = f32(1.0 - float(b2) ** step)
    g = np.asarray(grad, dtype=f32)
    mp = b1 * m + (f32(1) - b1) * g
    vp = b2 * v + (f32(1) - b2) * (g * g)
    mh = mp / c1
    vh = vp / c2
    x = master - (f32(lr) * mh) / (np.sqrt(vh) + f32(eps))
    return x.astype(f32), mp.astype(f32), vp.astype(f32), bf16_bits(x)


def gradient_f64(w, norm, X, T, delta: float, over: float):
    """Mean loss and gradient of the same network in float64 without bf16
    rounding (for the finite-difference check of the backward formulas)."""
    w = np.asarray(w, dtype=np.float64)
    W1, b1, W2, b2, W3, b3 = _unpack(w)
    X = np.asarray(X, dtype=np.float64)
    norm = np.asarray(norm, dtype=np.float64)
    z = (X - norm[:F_IN]) * norm[F_IN:]
    a1 = z @ W1.T + b1
    h1 = np.maximum(a1, 0)
    a2 = h1 @ W2.T + b2
    h2 = np.maximum(a2, 0)
    y = h2 @ W3 + b3
    e = y - np.asarray(T, dtype=np.float64)
    ae = np.abs(e)
    wt = np.where(e > 0, over, 1.0)
    quad = ae <= delta
    loss = wt * np.where(quad, 0.5 * e * e, delta * (ae - 0.5 * delta))
    g = wt * np.where(quad, e, np.copysign(delta, e))
    n = X.shape[0]
    d2 = (a2 > 0) * (g[:, None] * W3[None, :])
    d1 = (a1 > 0) * (d2 @ W2)
    grad = np.zeros(PARAMS)
    grad[OFF_W1:OFF_B1] = (d1.T @ z).ravel() / n
    grad[OFF_B1:OFF_W2] = d1.sum(0) / n
    grad[OFF_W2:OFF_B2] = (d2.T @ h1).ravel() / n
    grad[OFF_B2:OFF_W3] = d2.sum(0) / n
    grad[OFF_W3:OFF_B3] = (g[:, None] * h2).sum(0) / n
    grad[OFF_B3] = g.sum() / n
    return loss.mean(), grad


def features(rec, rw: float, sc: float) -> np.ndarray:
    """Features of pxr_cluster_record rows (cluster_features), in float64."""
    s = rec["size"].astype(np.float64)
    vol = rec["volume"].astype(np.float64)
    pot = rec["potential"].astype(np.float64)
    sp = rec["sparsity"].astype(np.float64)
    has = rec["has_prev"].astype(bool)
    dr = np.where(has, rec["round"].astype(np.float64) - rec["prev_round"].astype(np.float64), 0.0)
    fdr = np.maximum(dr, 1.0)
    lp = np.log10(np.maximum(pot, 1e-12) / rw)
    spc = np.minimum(sp, 2.0)
    decay = np.where(has, (lp - np.log10(np.maximum(rec["prev_potential"].astype(np.float64), 1e-12) / rw)) / fdr, 0.0)
    slope = np.where(has, (spc - np.minimum(rec["prev_sparsity"].astype(np.float64), 2.0)) / fdr, 0.0)
    f = np.zeros((rec.shape[0], F_IN))
    f[:, 0] = np.log2(s)
    f[:, 1] = np.log2(vol + 1.0)
    f[:, 2] = vol / s / 8.0
    f[:, 3] = lp
    f[:, 4] = decay
    f[:, 5] = spc
    f[:, 6] = slope
    f[:, 7] = spc - sc
    f[:, 8] = np.log2(1.0 + rec["age"].astype(np.float64))
    f[:, 9] = has
    f[:, 10] = np.where(has, np.minimum(fdr, 64.0) / 8.0, 0.0)
    f[:, 11] = np.log2(1.0 + rec["round"].astype(np.float64)) / 8.0
    with np.errstate(divide="ignore", invalid="ignore"):
        f[:, 12] = np.where(has & (decay < -1e-3), np.minimum(np.maximum(lp, 0.0) / -decay, 64.0) / 16.0, 4.0)
        f[:, 13] = np.where(has & (slope < -1e-3), np.minimum(np.maximum(spc - sc, 0.0) / -slope, 64.0) / 16.0, 4.0)
    return f


def skip_from_prediction(y, safety: float, max_skip: int) -> np.ndarray:
    y = np.asarray(y, dtype=np.float64)
    r = np.floor(safety * (np.exp2(np.minimum(y, 16.0)) - 1.0))
    r = np.where(y > 0, r, 0.0)
    return np.clip(r, 0, max_skip).astype(np.int64)
