"""NumPy restatement of the surrogate network (test infrastructure).

The checker for the surrogate kernels (photonfdtd_b200/csrc/surrogate.cu
driven by photonfdtd_b200/surrogate.py). The reference has no learned
surrogate, so this oracle follows the architecture defined by
``photonfdtd_b200.surrogate.ARCH`` with the same layouts: NHWC activations,
weights W[cout][K] with K ordered (ky, kx, c), im2col rows (b, oy, ox).
Computed in float64. With ``bf16=True`` every GEMM operand (lowered
activations, weights, back-propagated pre-activation gradients) is rounded to
BF16 first, as the GPU path does, so GPU results can be compared at FP32
accumulation accuracy. Only tests/, __graft_entry__.smoke() and bench.py may
import it.
"""
from __future__ import annotations

from typing import List, Sequence, Tuple

import numpy as np


def bf16(a: np.ndarray) -> np.ndarray:
    """Nearest BF16 value (ties to even) of each element, as float64."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return (r & 0xFFFFFFFF).astype(np.uint32).view(np.float32).astype(np.float64)


def im2col(x: np.ndarray, kh, kw, stride, ph, pw) -> Tuple[np.ndarray, int, int]:
    """x (B, H, W, C) -> col (B*Ho*Wo, kh*kw*C), columns (ky, kx, c)."""
    B, H, W, C = x.shape
    Ho = (H + 2 * ph - kh) // stride + 1
    Wo = (W + 2 * pw - kw) // stride + 1
    xp = np.zeros((B, H + 2 * ph, W + 2 * pw, C), dtype=x.dtype)
    xp[:, ph:ph + H, pw:pw + W] = x
    cols = []
    for ky in range(kh):
        for kx in range(kw):
            cols.append(xp[:, ky:ky + stride * Ho:stride, kx:kx + stride * Wo:stride, :])
    col = np.stack(cols, axis=3)  # (B, Ho, Wo, taps, C)
    return col.reshape(B * Ho * Wo, kh * kw * C), Ho, Wo


def col2im(dcol: np.ndarray, shape, kh, kw, stride, ph, pw) -> np.ndarray:
    B, H, W, C = shape
    Ho = (H + 2 * ph - kh) // stride + 1
    Wo = (W + 2 * pw - kw) // stride + 1
    d = dcol.reshape(B, Ho, Wo, kh * kw, C)
    xp = np.zeros((B, H + 2 * ph, W + 2 * pw, C))
    t = 0
    for ky in range(kh):
        for kx in range(kw):
            xp[:, ky:ky + stride * Ho:stride, kx:kx + stride * Wo:stride, :] += d[:, :, :, t, :]
            t += 1
    return xp[:, ph:ph + H, pw:pw + W]


class RefNet:
    """Forward / backward of the surrogate network in NumPy."""

    def __init__(self, layers, params, bf16_ops: bool = False):
        self.layers = layers
        self.params = [(None if w is None else np.asarray(w, np.float64),
                        None if b is None else np.asarray(b, np.float64)) for w, b in params]
        self.q = bf16 if bf16_ops else (lambda a: np.asarray(a, np.float64))

    def forward(self, x: np.ndarray) -> np.ndarray:
        """x (B, 64, 64) -> (B, 32, 2)."""
        q = self.q
        B = x.shape[0]
        a = np.asarray(x, np.float64).reshape(B, 64, 64, 1)
        self.cache = []
        for L, (w, b) in zip(self.layers, self.params):
            if L.kind == "up":
                self.cache.append(("up", a.shape))
                a = np.repeat(a, 2, axis=2)
                continue
            if L.kind == "conv":
                col, Ho, Wo = im2col(q(a), L.kh, L.kw, L.stride, L.ph, L.pw)
                out_shape = (B, Ho, Wo, L.cout)
            else:
                col = q(a).reshape(B, -1)
                out_shape = (B, 1, L.cout // 64, 64)
            pre = col @ q(w).T + b
            y = np.maximum(pre, 0.0) if L.relu else pre
            self.cache.append((col, a.shape, pre))
            a = y.reshape(out_shape)
        return a.reshape(B, 32, 2)

    def backward(self, dy: np.ndarray):
        """dy (B, 32, 2) -> (weight grads [(gW, gb)], dx (B, 64, 64))."""
        q = self.q
        B = dy.shape[0]
        g = np.asarray(dy, np.float64).reshape(B, 1, 32, 2)
        grads: List = [None] * len(self.layers)
        for li in range(len(self.layers) - 1, -1, -1):
            L = self.layers[li]
            w, _ = self.params[li]
            c = self.cache[li]
            if L.kind == "up":
                shp = c[1]
                g = g.reshape(shp[0], shp[1], shp[2], 2, shp[3]).sum(axis=3)
                grads[li] = (None, None)
                continue
            col, in_shape, pre = c
            d = g.reshape(pre.shape)
            if L.relu:
                d = d * (pre > 0)
            dq = q(d)
            grads[li] = (dq.T @ col, d.sum(axis=0))
            dcol = dq @ q(w)
            if L.kind == "conv":
                g = col2im(dcol, in_shape, L.kh, L.kw, L.stride, L.ph, L.pw)
            else:
                g = dcol.reshape(in_shape)
        return grads, g.reshape(B, 64, 64)
