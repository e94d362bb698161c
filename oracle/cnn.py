"""CPU restatement of the learned corrector's network (test infrastructure).

Checks the tensor-core kernels of ouc_b200/csrc/corrector.cu: the same
four-layer 5x5 CNN (10 -> 32 -> 32 -> 32 -> 8 channels, ReLU between, "same"
zero padding), computed in float64 with the operands rounded to bfloat16 at
the points where the GPU path rounds them (network input, weights, hidden
activations, output and hidden-layer gradients), so that the two differ only
by the order of the FP32 accumulations on the GPU.  The backward pass is
checked against finite differences in float64 without rounding
(tests/test_corrector.py).  Images are NHWC: [n][H][W][C].
"""
from __future__ import annotations

import numpy as np

DIMS = [(10, 32), (32, 32), (32, 32), (32, 8)]
TAPS = 25


def nparams():
    return sum(co * ci * TAPS + co for ci, co in DIMS)


def split(params):
    """Flat parameter vector -> [(W[co][ci][5][5], b[co])] per layer."""
    out, k = [], 0
    for ci, co in DIMS:
        w = params[k:k + co * ci * TAPS].reshape(co, ci, 5, 5)
        k += co * ci * TAPS
        b = params[k:k + co]
        k += co
        out.append((w, b))
    return out


def init_params(seed=0, gain=1.0):
    """He-style initialisation (normal, std = gain * sqrt(2 / fan_in)), zero bias."""
    rng = np.random.default_rng(seed)
    parts = []
    for ci, co in DIMS:
        parts.append(rng.normal(0.0, gain * np.sqrt(2.0 / (ci * TAPS)), size=co * ci * TAPS))
        parts.append(np.zeros(co))
    return np.concatenate(parts).astype(np.float32)


def bf16(a):
    """Round to bfloat16 (nearest, ties to even), returned as float64."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def _shift(x, dx, dz):
    """x[n, h + dx, w + dz, :] with zeros outside (dx, dz in -2..2)."""
    n, H, W, C = x.shape
    out = np.zeros_like(x)
    hs, he = max(0, -dx), min(H, H - dx)
    ws, we = max(0, -dz), min(W, W - dz)
    out[:, hs:he, ws:we] = x[:, hs + dx:he + dx, ws + dz:we + dz]
    return out


def conv(x, w):
    """y[p][co] = sum_tap sum_ci w[co][ci][tap] * x[p + tap - 2][ci]."""
    n, H, W, _ = x.shape
    y = np.zeros((n, H, W, w.shape[0]))
    for kx in range(5):
        for kz in range(5):
            y += np.einsum("nhwc,oc->nhwo", _shift(x, kx - 2, kz - 2), w[:, :, kx, kz], optimize=True)
    return y


def conv_input_grad(g, w):
    """dL/dx of conv(x, w) given dL/dy = g."""
    n, H, W, _ = g.shape
    dx = np.zeros((n, H, W, w.shape[1]))
    for kx in range(5):
        for kz in range(5):
            dx += np.einsum("nhwo,oc->nhwc", _shift(g, 2 - kx, 2 - kz), w[:, :, kx, kz], optimize=True)
    return dx


def conv_weight_grad(x, g):
    """dL/dw[co][ci][kx][kz] = sum_p x[p + (kx-2, kz-2)][ci] g[p][co]."""
    dw = np.zeros((g.shape[-1], x.shape[-1], 5, 5))
    for kx in range(5):
        for kz in range(5):
            dw[:, :, kx, kz] = np.einsum("nhwc,nhwo->oc", _shift(x, kx - 2, kz - 2), g, optimize=True)
    return dw


class Net:
    """Forward and backward of the corrector network; rounding=True models the
    GPU's bfloat16 operands, rounding=False is the exact float64 network."""

    def __init__(self, params, rounding=True):
        self.r = bf16 if rounding else (lambda a: np.asarray(a, np.float64))
        params = np.asarray(params, np.float32 if rounding else np.float64)
        self.layers = [(self.r(w), np.asarray(b, np.float64)) for w, b in split(params)]

    def forward(self, x):
        r = self.r
        self.acts = [r(x)]
        h = self.acts[0]
        for l, (w, b) in enumerate(self.layers):
            z = conv(h, w) + b
            if l < 3:
                h = r(np.maximum(z, 0.0))
                self.acts.append(h)
            else:
                out = z
        return out

    def backward(self, gout):
        """Parameter gradients as one flat vector (the layout of the parameters)."""
        r = self.r
        g = r(gout)
        grads = [None] * 4
        for l in range(3, -1, -1):
            w, _ = self.layers[l]
            x = self.acts[l]
            grads[l] = (conv_weight_grad(x, g), g.sum(axis=(0, 1, 2)))
            if l > 0:
                g = r(conv_input_grad(g, w) * (x > 0))
        return np.concatenate([np.concatenate([dw.ravel(), db]) for dw, db in grads])
