"""TEST INFRASTRUCTURE -- a NumPy (float64) restatement of the surrogate
network's forward pass, loss and gradients, for checking the tensor-core
training kernels (merlict_development_kit_b200/csrc/surrogate.cu).

The restatement rounds to BF16 exactly where the device kernels store BF16
tile images (the encoded inputs, layer outputs, the output gradient, the
hidden-layer gradients) and keeps everything else in float64, so that the only
differences to the device are the FP32 accumulation order and the device's
exp/log.  Only tests/ use it.
"""
from __future__ import annotations

import numpy as np

K = 8        # mixture components
D = 4        # mixture dimensions
LOG_SQRT_2PI = 0.91893853320467274


def bf16(x: np.ndarray) -> np.ndarray:
    """Round to the nearest BF16 (ties to even), via float32."""
    f = np.asarray(x, dtype=np.float32)
    b = f.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


OCTAVES = 12
ENCODED = 128


def encode(x) -> np.ndarray:
    """The fixed input encoding: the 5 inputs, then sin(pi 2^l x_j) and
    cos(pi 2^l x_j) for j = 0..4, l = 0..11 (feature 5 + 2 (12 j + l) + c),
    zero padding to 128; the inputs are the FP32 values the device reads."""
    x = np.asarray(x, dtype=np.float32).astype(np.float64)[:, :5]
    e = np.zeros((x.shape[0], ENCODED))
    e[:, :5] = x
    for j in range(5):
        for l in range(OCTAVES):
            a = np.pi * (2.0 ** l) * x[:, j]
            e[:, 5 + 2 * (OCTAVES * j + l)] = np.sin(a)
            e[:, 5 + 2 * (OCTAVES * j + l) + 1] = np.cos(a)
    return e


def unpack(params: np.ndarray) -> list:
    """[(W [out][in], b [out])] of the five layers."""
    shapes = ((ENCODED, 256), (256, 256), (256, 256), (256, 256), (256, 73))
    out, o = [], 0
    p = np.asarray(params, dtype=np.float64)
    for fin, fout in shapes:
        W = p[o:o + fin * fout].reshape(fout, fin)
        o += fin * fout
        b = p[o:o + fout]
        o += fout
        out.append((W, b))
    assert o == p.size
    return out


def forward(params, x):
    """Outputs [n][73] and the intermediates of the backward pass."""
    L = unpack(params)
    x = bf16(encode(x))
    z = [x @ bf16(L[0][0]).T + L[0][1]]
    h = [bf16(silu(z[0]))]
    for l in (1, 2, 3):
        z.append(h[-1] @ bf16(L[l][0]).T + L[l][1])
        h.append(bf16(silu(z[-1])))
    y = h[-1] @ bf16(L[4][0]).T + L[4][1]
    return y, (x, z, h)


def loss_and_grad_outputs(y, t, reached):
    """Batch-mean loss and its gradient with respect to the outputs
    (log-sigmas clamped to [-9, 3], zero gradient outside)."""
    n = y.shape[0]
    loss = np.zeros(n)
    dy = np.zeros_like(y)
    l = y[:, 0]
    sig = 1.0 / (1.0 + np.exp(-l))
    loss += np.maximum(l, 0.0) + np.log1p(np.exp(-np.abs(l))) - reached * l
    dy[:, 0] = sig - reached
    a = y[:, 1:1 + 9 * K:9]                                  # [n][K]
    mu = np.stack([y[:, 2 + 9 * k:6 + 9 * k] for k in range(K)], axis=1)    # [n][K][D]
    raw = np.stack([y[:, 6 + 9 * k:10 + 9 * k] for k in range(K)], axis=1)
    ls = np.clip(raw, -9.0, 3.0)
    log_pi = a - (a.max(axis=1, keepdims=True) +
                  np.log(np.exp(a - a.max(axis=1, keepdims=True)).sum(axis=1, keepdims=True)))
    u = (t[:, None, :] - mu) * np.exp(-ls)
    ell = log_pi + (-0.5 * u * u - ls - LOG_SQRT_2PI).sum(axis=2)
    m = ell.max(axis=1, keepdims=True)
    lse = m[:, 0] + np.log(np.exp(ell - m).sum(axis=1))
    gam = np.exp(ell - lse[:, None])
    r = reached.astype(bool)
    loss += np.where(r, -lse, 0.0)
    pi = np.exp(log_pi)
    da = pi - gam
    dmu = -gam[:, :, None] * u * np.exp(-ls)
    dls = np.where((raw >= -9.0) & (raw <= 3.0), gam[:, :, None] * (1.0 - u * u), 0.0)
    for k in range(K):
        dy[:, 1 + 9 * k] = np.where(r, da[:, k], 0.0)
        dy[:, 2 + 9 * k:6 + 9 * k] = np.where(r[:, None], dmu[:, k], 0.0)
        dy[:, 6 + 9 * k:10 + 9 * k] = np.where(r[:, None], dls[:, k], 0.0)
    return loss.mean(), dy / n


def gradients(params, x, t, reached):
    """(batch-mean loss, gradient of it in the flat parameter layout)."""
    L = unpack(params)
    y, (x, z, h) = forward(params, x)
    loss, dy = loss_and_grad_outputs(y, np.asarray(t, np.float64), np.asarray(reached, np.float64))
    g = []
    dyb = bf16(dy)
    dW = [None] * 5
    db = [None] * 5
    dW[4] = dyb.T @ h[3]
    db[4] = dy.sum(axis=0)
    dh = dyb @ bf16(L[4][0])
    for l in (3, 2, 1):
        dz = dh * dsilu(z[l])
        db[l] = dz.sum(axis=0)
        dzb = bf16(dz)
        dW[l] = dzb.T @ h[l - 1]
        dh = dzb @ bf16(L[l][0])
    dz0 = dh * dsilu(z[0])
    db[0] = dz0.sum(axis=0)
    dW[0] = bf16(dz0).T @ x
    for l in range(5):
        g.append(dW[l].reshape(-1))
        g.append(db[l])
    return loss, np.concatenate(g)
