"""FP64 restatement of the learned-guess network's forward and backward pass -- TEST
INFRASTRUCTURE ONLY (the checker of the GPU library's hand-written BF16 training kernels).

The network has no counterpart in pm3-rs (its guesses are SAD, core and symmetry-broken SAD,
src/scf.rs:855-916), so this restates the GPU library's own definition: a 64 -> 256 -> 256 ->
256 -> 8 MLP with SiLU on the hidden layers, masked squared-error loss
loss = inv_count * sum mask * (Y - T)^2, parameters laid out W1 b1 W2 b2 W3 b3 W4 b4 (weights
row-major, inputs x outputs). Values are rounded to BF16 exactly where the GPU rounds them (the
GEMM operands: features, weights, hidden activations, dY and dZ); everything else is FP64, so
the comparison isolates the GPU's FP32 accumulation and its ordering.
"""
from __future__ import annotations

import numpy as np

SIZES = [(64, 256), (256, 256), (256, 256), (256, 8)]


def bf16(a):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    a = np.ascontiguousarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return (u.astype(np.uint32) << 16).view(np.float32).astype(np.float64)


def unpack(p):
    """Parameter vector -> [(W, b)] per layer (W as float64 of the FP32 master values)."""
    out, off = [], 0
    for fi, fo in SIZES:
        w = np.asarray(p[off:off + fi * fo], np.float64).reshape(fi, fo)
        off += fi * fo
        b = np.asarray(p[off:off + fo], np.float64)
        off += fo
        out.append((w, b))
    return out


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def loss_and_grad(p, x, t, m, inv_count, rnd=bf16):
    """Loss and gradient vector (same layout as p) of one pass over rows x (64), targets t (8),
    masks m (8). `rnd` is the rounding applied at the GPU's BF16 points (identity: exact FP64,
    which a finite-difference check can pin)."""
    layers = unpack(p)
    ins, zs = [], []
    h = rnd(x)
    for li, (w, b) in enumerate(layers):
        ins.append(h)
        z = h @ rnd(w) + b
        zs.append(z)
        h = rnd(silu(z)) if li < 3 else z
    y = h
    d = (y - t) * m
    loss = inv_count * float(np.sum(d * d))
    dy = rnd(2.0 * d * inv_count)
    grads = [None] * 4
    w4 = rnd(layers[3][0])
    grads[3] = (ins[3].T @ dy, dy.sum(axis=0))
    dh = dy @ w4.T
    for li in (2, 1, 0):
        dz = rnd(dh * dsilu(zs[li]))
        grads[li] = (ins[li].T @ dz, dz.sum(axis=0))
        if li > 0:
            dh = dz @ rnd(layers[li][0]).T
    flat = np.concatenate([np.concatenate([gw.ravel(), gb]) for gw, gb in grads])
    return loss, flat
