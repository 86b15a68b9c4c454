"""CPU oracle of the learned correction network (test infrastructure only).

The reference has no learned component; the network is specified by the
project (8 conv layers 3x3, zero padding: 16->32, 6 x 32->32 with ReLU,
32->16 of which channel 0 is the residual; output = centre slice + mu_w *
residual; loss = mean(((pred - target) / mu_w)^2)). This module restates its
forward and backward passes in numpy float64, optionally rounding to BF16 at
exactly the points where the GPU kernels store BF16 (weights, activations,
the network input, the backpropagated gradients), so that the GPU's parameter
gradients can be checked element by element. With ``bf16=False`` it is plain
float64 backpropagation, which ``tests/test_cnn_oracle.py`` checks against
finite differences.

Parameter layout (shared with the library): per layer W[co][tap][ci]
(tap = 3*ky + kx) followed by b[co], layers concatenated.
"""
from __future__ import annotations

import numpy as np

CIN = (16, 32, 32, 32, 32, 32, 32, 32)
COUT = (32, 32, 32, 32, 32, 32, 32, 16)


def param_count() -> int:
    return sum(9 * ci * co + co for ci, co in zip(CIN, COUT))


def split(params: np.ndarray):
    """[(W [co][9][ci], b [co])] views of a flat parameter vector."""
    out, o = [], 0
    for ci, co in zip(CIN, COUT):
        w = params[o:o + 9 * ci * co].reshape(co, 9, ci)
        o += 9 * ci * co
        b = params[o:o + co]
        o += co
        out.append((w, b))
    assert o == params.size
    return out


def bf16(a) -> np.ndarray:
    """Round to BF16 (nearest, ties to even) and return as float64."""
    f = np.asarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def init_params(seed: int, zero_last: bool = True) -> np.ndarray:
    """He-normal weights (fan-in of the real input channels), zero biases;
    padded input channels of layer 1 and unused output channels of layer 8 are
    zero; the last layer starts at zero (the network starts as the identity)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(param_count(), dtype=np.float32)
    for l, (w, b) in enumerate(split(p)):
        ci_real = 5 if l == 0 else w.shape[2]
        co_real = 1 if l == 7 else w.shape[0]
        std = np.sqrt(2.0 / (9 * ci_real))
        if l == 7 and zero_last:
            continue
        w[:co_real, :, :ci_real] = rng.standard_normal((co_real, 9, ci_real)) * std
    return p


def conv(x: np.ndarray, w: np.ndarray) -> np.ndarray:
    """3x3 zero-padded convolution: x [B][H][W][ci], w [co][9][ci] -> [B][H][W][co]."""
    B, H, W, _ = x.shape
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (0, 0)))
    y = np.zeros((B, H, W, w.shape[0]))
    for tap in range(9):
        ky, kx = divmod(tap, 3)
        y += xp[:, ky:ky + H, kx:kx + W, :] @ w[:, tap, :].T
    return y


def conv_bwd_data(g: np.ndarray, w: np.ndarray) -> np.ndarray:
    """Gradient w.r.t. the conv input: g [B][H][W][co] -> [B][H][W][ci]."""
    B, H, W, _ = g.shape
    gp = np.pad(g, ((0, 0), (1, 1), (1, 1), (0, 0)))
    dx = np.zeros((B, H, W, w.shape[2]))
    for tap in range(9):
        ky, kx = divmod(tap, 3)
        dx += gp[:, 2 - ky:2 - ky + H, 2 - kx:2 - kx + W, :] @ w[:, tap, :]
    return dx


def conv_wgrad(x: np.ndarray, g: np.ndarray):
    """dW [co][9][ci] = sum_p g[p][co] x[p + tap][ci]; db [co] = sum_p g[p][co]."""
    B, H, W, ci = x.shape
    co = g.shape[3]
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (0, 0)))
    dw = np.zeros((co, 9, ci))
    g2 = g.reshape(-1, co)
    for tap in range(9):
        ky, kx = divmod(tap, 3)
        dw[:, tap, :] = g2.T @ xp[:, ky:ky + H, kx:kx + W, :].reshape(-1, ci)
    return dw, g2.sum(axis=0)


def forward(params, x, base, mu_w, bf16_mode=True):
    """Returns (pred [B][H][W], activations list, residual). x: [B][H][W][16]."""
    rnd = bf16 if bf16_mode else (lambda a: np.asarray(a, dtype=np.float64))
    layers = split(np.asarray(params, dtype=np.float32 if bf16_mode else np.float64))
    acts = [rnd(x)]
    for l in range(7):
        w, b = layers[l]
        acts.append(rnd(np.maximum(conv(acts[-1], rnd(w)) + b.astype(np.float64), 0.0)))
    w, b = layers[7]
    r = conv(acts[-1], rnd(w))[..., 0] + float(b[0])
    pred = np.asarray(base, dtype=np.float64) + mu_w * r
    return pred, acts, r


def loss_and_grads(params, x, base, target, mu_w, bf16_mode=True):
    """Loss and flat parameter gradient (float64), with the GPU's BF16 storage
    points when ``bf16_mode``."""
    rnd = bf16 if bf16_mode else (lambda a: np.asarray(a, dtype=np.float64))
    layers = split(np.asarray(params, dtype=np.float32 if bf16_mode else np.float64))
    pred, acts, _ = forward(params, x, base, mu_w, bf16_mode)
    e = (pred - np.asarray(target, dtype=np.float64)) / mu_w
    n = e.size
    loss = float(np.mean(e * e))
    g = np.zeros(acts[-1].shape[:3] + (16,))
    g[..., 0] = 2.0 * e / n
    g = rnd(g)
    grads = [None] * 8
    for l in range(7, -1, -1):
        w, _ = layers[l]
        dw, db = conv_wgrad(acts[l], g)
        grads[l] = (dw, db)
        if l == 0:
            break
        g = rnd(conv_bwd_data(g, rnd(w)) * (acts[l] > 0))
    flat = np.concatenate([np.concatenate([dw.ravel(), db]) for dw, db in grads])
    return loss, flat
