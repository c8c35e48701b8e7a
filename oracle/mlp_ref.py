"""CPU reference of the learned warm-start MLP (TEST INFRASTRUCTURE -- never the
product): forward pass, MSE loss and parameter gradients in float64 numpy.

The network (no counterpart in the reference repository): three GELU hidden
layers of 256 and a linear output layer, inputs normalised as
(x - mean) / std (zero where std <= 1e-6), targets as (t - mean) / std.
Parameter layout (flat float32): W0[256][in_pad], b0[256], W1[256][256], b1,
W2[256][256], b2, W3[out_pad][256], b3[out_pad].

`bf16=True` rounds to bfloat16 at the points where the GPU kernels store
bfloat16 (inputs, weights, pre-activations, activations, output gradients,
hidden gradients), so that the comparison isolates accumulation-order
differences; `bf16=False` is the exact float64 network.
"""
from __future__ import annotations

from math import erf, sqrt

import numpy as np

HIDDEN = 256
OUT_PAD = 64


def bf16_round(x):
    """Round float32 values to the nearest bfloat16 (ties to even)."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


_erf = np.vectorize(erf)


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z / sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + _erf(z / sqrt(2.0))) + z * np.exp(-0.5 * z * z) / sqrt(2.0 * np.pi)


def layer_shapes(in_pad, out_pad=OUT_PAD):
    return [(HIDDEN, in_pad), (HIDDEN, HIDDEN), (HIDDEN, HIDDEN), (out_pad, HIDDEN)]


def unpack(params, in_pad, out_pad=OUT_PAD):
    """Flat parameter vector -> [(W, b)] per layer (float64 copies)."""
    out, o = [], 0
    for r, c in layer_shapes(in_pad, out_pad):
        W = np.asarray(params[o:o + r * c], np.float64).reshape(r, c)
        o += r * c
        b = np.asarray(params[o:o + r], np.float64)
        o += r
        out.append((W, b))
    assert o == len(params)
    return out


def pack(layers):
    return np.concatenate([np.concatenate([W.ravel(), b]) for W, b in layers]).astype(np.float64)


def normalise(x, mean, std):
    istd = np.where(np.asarray(std) > 1e-6, 1.0 / np.maximum(std, 1e-30), 0.0)
    return (np.asarray(x, np.float64) - mean) * istd


def forward(params, xraw, in_mean, in_std, in_pad, bf16=True, keep=False):
    """Network output y[n][out_pad] (normalised target units)."""
    rnd = bf16_round if bf16 else (lambda v: np.asarray(v, np.float64))
    layers = unpack(params, in_pad)
    x = normalise(xraw, in_mean, in_std).astype(np.float32)
    xp = np.zeros((x.shape[0], in_pad))
    xp[:, : x.shape[1]] = x
    h = rnd(xp)
    cache = {"h": [h], "z": []}
    for W, b in layers[:3]:
        z = h @ rnd(W).T + b
        if bf16:
            z = z.astype(np.float32)
        zs = rnd(z)
        cache["z"].append(zs)
        h = rnd(gelu(z))
        cache["h"].append(h)
    W, b = layers[3]
    y = h @ rnd(W).T + b
    return (y, cache) if keep else y


def loss_and_grads(params, xraw, traw, in_mean, in_std, out_mean, out_std, in_pad, nout, bf16=True):
    """Mean squared error over rows and the nout real outputs (normalised
    units) and its gradient with respect to the flat parameters."""
    rnd = bf16_round if bf16 else (lambda v: np.asarray(v, np.float64))
    layers = unpack(params, in_pad)
    n = xraw.shape[0]
    y, cache = forward(params, xraw, in_mean, in_std, in_pad, bf16=bf16, keep=True)
    t = (np.asarray(traw, np.float64) - out_mean) / np.maximum(out_std, 1e-6)
    if bf16:
        t = t.astype(np.float32).astype(np.float64)
    d = np.zeros_like(y)
    d[:, :nout] = y[:, :nout] - t
    loss = float((d[:, :nout] ** 2).sum() / (n * nout))
    dy = rnd(2.0 / (n * nout) * d)
    grads = [None] * 4
    h3 = cache["h"][3]
    grads[3] = (dy.T @ h3, dy.sum(0))
    g = dy
    for l in (2, 1, 0):
        W_next = rnd(layers[l + 1][0])
        dh = g @ W_next
        dz = rnd(dh * gelu_grad(cache["z"][l]))
        hin = cache["h"][l]
        grads[l] = (dz.T @ hin, dz.sum(0))
        g = dz
    return loss, pack(grads)
