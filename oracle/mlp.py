"""Oracle of the perceptron (test infrastructure only): forward, mean-squared
error and its gradient in numpy, with the same BF16 rounding points as the
device kernels (inputs, weights, hidden activations and the back-propagated
pre-activation gradients are BF16; products accumulate in FP64 here, FP32 on
the device).  `bf16=False` gives the exact FP64 model for finite-difference
checks.

Parameter layout (flat): per layer W (n_out x n_in, row-major) then b.
GELU is the tanh form 0.5 x (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3))) of
Hendrycks & Gimpel, "Gaussian Error Linear Units" (arXiv:1606.08415, 2016),
an approximation of x Phi(x) = 0.5 x (1 + erf(x / sqrt 2)).
"""
from __future__ import annotations

import numpy as np

K_GELU = np.sqrt(2.0 / np.pi)


def bf16(a):
    """Round float32 values to bfloat16 (round to nearest even), as float32."""
    a = np.ascontiguousarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(x):
    return 0.5 * x * (1.0 + np.tanh(K_GELU * (x + 0.044715 * x ** 3)))


def gelu_grad(x):
    u = K_GELU * (x + 0.044715 * x ** 3)
    t = np.tanh(u)
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * K_GELU * (1.0 + 3 * 0.044715 * x * x)


def unpack(params, shapes):
    out, o = [], 0
    for (n_out, n_in) in shapes:
        W = np.asarray(params[o:o + n_out * n_in], np.float64).reshape(n_out, n_in)
        o += n_out * n_in
        b = np.asarray(params[o:o + n_out], np.float64)
        o += n_out
        out.append((W, b))
    return out


def forward(params, shapes, x, bf=True):
    r = bf16 if bf else (lambda a: np.asarray(a, np.float64))
    layers = unpack(params, shapes)
    h = r(x)
    cache = []
    for l, (W, b) in enumerate(layers):
        z = h @ r(W).T + b
        cache.append((h, z))
        h = r(gelu(z)) if l < len(layers) - 1 else z
    return h, cache


def loss_grad(params, shapes, x, t, bf=True):
    r = bf16 if bf else (lambda a: np.asarray(a, np.float64))
    layers = unpack(params, shapes)
    y, cache = forward(params, shapes, x, bf)
    B, n_out = t.shape
    d = y - t
    loss = float((d * d).sum() / (B * n_out))
    dz = r(2.0 * d / (B * n_out))
    grads = [None] * len(layers)
    for l in range(len(layers) - 1, -1, -1):
        h, _ = cache[l]
        W, _ = layers[l]
        grads[l] = (dz.T @ h, dz.sum(axis=0))
        if l > 0:
            dh = dz @ r(W)
            dz = r(dh * gelu_grad(cache[l - 1][1]))
    flat = np.concatenate([np.concatenate([gW.ravel(), gb]) for gW, gb in grads])
    return loss, flat
