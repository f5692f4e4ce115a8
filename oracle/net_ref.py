"""CPU restatement of the learned continuation predictor (the sf_net_* entry
points of include/stratiflow_b200.h), for checking the GPU's forward pass and
gradients. Test infrastructure only: the library never calls it.

The network has no counterpart in the reference (it stands beside the secant
predictor of PseudoArclength.cpp:33-61), so this file restates the GPU
network's own definition: 1D convolutions along z with 5 taps and zero
padding 2, ReLU between layers, mean-square loss. With `bf16=True` it rounds
the operands of every contraction to BF16 (round to nearest even) at the same
points as the GPU and accumulates in FP64; with `bf16=False` it is the exact
FP64 network, whose gradient is checked against finite differences.
"""
from __future__ import annotations

import numpy as np

TAPS, PAD = 5, 2


def bf16_round(x):
    """float32 -> nearest BF16 value (ties to even), returned as float32."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def unpack(params, channels):
    """[(W[Cout][5][Cin], b[Cout]), ...] from the flat parameter vector."""
    out, off = [], 0
    for ci, co in zip(channels[:-1], channels[1:]):
        n = co * TAPS * ci
        W = params[off:off + n].reshape(co, TAPS, ci)
        off += n
        b = params[off:off + co]
        off += co
        out.append((W, b))
    assert off == params.size
    return out


def _conv(x, W):
    """y[b][z][co] = sum_tap,ci W[co][tap][ci] x[b][z+tap-2][ci], FP64."""
    B, Z, _ = x.shape
    xp = np.zeros((B, Z + 2 * PAD, x.shape[2]))
    xp[:, PAD:PAD + Z] = x
    y = np.zeros((B, Z, W.shape[0]))
    for t in range(TAPS):
        y += xp[:, t:t + Z] @ W[:, t, :].T.astype(np.float64)
    return y


def _conv_data(d, W):
    """dx[b][z][ci] = sum_co,tap W[co][tap][ci] d[b][z-tap+2][co], FP64."""
    B, Z, _ = d.shape
    dp = np.zeros((B, Z + 2 * PAD, d.shape[2]))
    dp[:, PAD:PAD + Z] = d
    y = np.zeros((B, Z, W.shape[2]))
    for t in range(TAPS):
        # z - t + 2 = (z + 4 - t) - 2 in the padded array
        y += dp[:, TAPS - 1 - t:TAPS - 1 - t + Z] @ W[:, t, :].astype(np.float64)
    return y


def _conv_weight(d, x):
    """dW[co][tap][ci] = sum_b,z d[b][z][co] x[b][z+tap-2][ci], FP64."""
    B, Z, _ = x.shape
    xp = np.zeros((B, Z + 2 * PAD, x.shape[2]))
    xp[:, PAD:PAD + Z] = x
    d2 = d.reshape(-1, d.shape[2]).astype(np.float64)
    return np.stack([d2.T @ xp[:, t:t + Z].reshape(-1, x.shape[2]) for t in range(TAPS)], axis=1)


def forward(params, channels, x, bf16=True):
    """Output [B][Z][Cout] and the layer inputs (for backward)."""
    rnd = bf16_round if bf16 else (lambda a: np.asarray(a, dtype=np.float64))
    layers = unpack(np.asarray(params), channels)
    acts = [rnd(x)]
    for l, (W, b) in enumerate(layers):
        pre = _conv(acts[-1], rnd(W)) + np.asarray(b, dtype=np.float64)
        if l < len(layers) - 1:
            acts.append(rnd(np.maximum(pre, 0.0).astype(np.float32) if bf16 else np.maximum(pre, 0.0)))
        else:
            out = pre.astype(np.float32) if bf16 else pre
    return out, acts


def gradient(params, channels, x, target, bf16=True):
    """(flat gradient of the mean-square loss, loss)."""
    rnd = bf16_round if bf16 else (lambda a: np.asarray(a, dtype=np.float64))
    layers = unpack(np.asarray(params), channels)
    out, acts = forward(params, channels, x, bf16)
    diff = (out - target).astype(np.float32) if bf16 else out - target
    n = diff.size
    loss = float(np.sum(diff.astype(np.float64) ** 2) / n)
    d = rnd(np.float32(2.0 / n) * diff) if bf16 else 2.0 * diff / n
    grads = [None] * len(layers)
    for l in range(len(layers) - 1, -1, -1):
        W, _ = layers[l]
        gW = _conv_weight(d, acts[l])
        gb = d.reshape(-1, d.shape[2]).astype(np.float64).sum(axis=0)
        grads[l] = (gW, gb)
        if l > 0:
            dx = _conv_data(d, rnd(W))
            dx = np.where(acts[l] > 0, dx, 0.0)
            d = rnd(dx.astype(np.float32)) if bf16 else dx
    flat = np.concatenate([np.concatenate([gW.ravel(), gb]) for gW, gb in grads])
    return flat, loss


def init_params(channels, seed):
    """A seeded parameter vector (for the CPU-only checks; the GPU's own
    initial weights come from sf_net_create)."""
    rng = np.random.default_rng(seed)
    parts = []
    for ci, co in zip(channels[:-1], channels[1:]):
        parts.append(rng.normal(0.0, np.sqrt(2.0 / (TAPS * ci)), co * TAPS * ci))
        parts.append(rng.normal(0.0, 0.1, co))
    return np.concatenate(parts).astype(np.float32)
