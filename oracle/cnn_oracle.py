"""CPU restatement of the learned closure's network and optimiser -- TEST INFRASTRUCTURE ONLY.

This module is the checker for ``qgn_fortran_b200/csrc/cnn.cu`` (the closure network has no
counterpart in the reference, so its oracle is the project's own restatement):

* periodic 3x3 convolutions on NHWC tensors, ``out[b,h,w,n] = sum_tap sum_k
  in[b,(h+dy)%H,(w+dx)%W,k] W[tap,n,k] + bias[n]`` with ``tap = 3(dy+1) + (dx+1)``;
* exact GELU ``0.5 z (1 + erf(z/sqrt 2))`` between layers, none after the last;
* MSE over the real output channels, backpropagation, Adam (beta 0.9/0.999, eps 1e-8,
  bias-corrected);
* ``emulate=True`` rounds what the GPU keeps in BF16 (weights, activations, layer gradients)
  to BF16 (round-to-nearest-even) and keeps FP32 where the GPU does (pre-activations and the
  network output); sums run in float64, so results differ from the GPU's FP32 accumulation
  only by summation order.  ``emulate=False`` is the exact float64 network, which the
  finite-difference test pins.

Only tests and the CPU legs of the benchmark import this module.
"""
from __future__ import annotations

import numpy as np
from scipy.special import erf

SQRT1_2 = 0.70710678118654752
INV_SQRT_2PI = 0.39894228040143268


def bf16(x):
    """Round float32 values to bfloat16 (nearest even); returned as float32."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return (r & 0xFFFFFFFF).astype(np.uint32).view(np.float32).reshape(a.shape)


def gelu(z):
    return 0.5 * z * (1.0 + erf(z * SQRT1_2))


def gelu_grad(z):
    return 0.5 * (1.0 + erf(z * SQRT1_2)) + z * INV_SQRT_2PI * np.exp(-0.5 * z * z)


def _shift(tap):
    return tap // 3 - 1, tap % 3 - 1


def conv(x, w, b=None):
    """x [B,H,W,Cin], w [9,Cout,Cin] -> [B,H,W,Cout] (float64)."""
    x = np.asarray(x, dtype=np.float64)
    out = np.zeros(x.shape[:3] + (w.shape[1],))
    for tap in range(9):
        dy, dx = _shift(tap)
        xs = np.roll(x, shift=(-dy, -dx), axis=(1, 2))        # xs[h, w] = x[h+dy, w+dx]
        out += xs @ np.asarray(w[tap], dtype=np.float64).T
    if b is not None:
        out += np.asarray(b, dtype=np.float64)
    return out


def conv_transpose(g, w):
    """Gradient of conv w.r.t. its input: g [B,H,W,Cout] -> [B,H,W,Cin]."""
    g = np.asarray(g, dtype=np.float64)
    out = np.zeros(g.shape[:3] + (w.shape[2],))
    for tap in range(9):
        dy, dx = _shift(tap)
        out += np.roll(g @ np.asarray(w[tap], dtype=np.float64), shift=(dy, dx), axis=(1, 2))
    return out


def weight_grad(x, g):
    """Gradient of conv w.r.t. w: sum over pixels of g[p, n] x[p + tap, k] -> [9, Cout, Cin]."""
    x = np.asarray(x, dtype=np.float64)
    g = np.asarray(g, dtype=np.float64)
    cin, cout = x.shape[3], g.shape[3]
    dw = np.zeros((9, cout, cin))
    gf = g.reshape(-1, cout)
    for tap in range(9):
        dy, dx = _shift(tap)
        xs = np.roll(x, shift=(-dy, -dx), axis=(1, 2)).reshape(-1, cin)
        dw[tap] = gf.T @ xs
    return dw


class CNNOracle:
    """layers = [(W [9,cout_p,cin_p], b [cout_p]), ...] (float32 masters); cout_real channels used."""

    def __init__(self, layers, cout_real):
        self.layers = [(np.asarray(w, dtype=np.float32), np.asarray(b, dtype=np.float32)) for w, b in layers]
        self.cout_real = cout_real

    def _w(self, l, emulate):
        w, b = self.layers[l]
        return (bf16(w) if emulate else w.astype(np.float64)), b

    def forward(self, x, emulate=True):
        a = np.asarray(x, dtype=np.float32)
        acts, zs = [a], []
        L = len(self.layers)
        for l in range(L):
            w, b = self._w(l, emulate)
            z = conv(a, w, b)
            z = z.astype(np.float32) if emulate else z
            zs.append(z)
            if l < L - 1:
                a = bf16(gelu(z.astype(np.float64))) if emulate else gelu(z)
                acts.append(a)
        return zs[-1], zs, acts

    def loss_and_grads(self, x, t, emulate=True):
        y, zs, acts = self.forward(x, emulate)
        cr = self.cout_real
        count = y.shape[0] * y.shape[1] * y.shape[2] * cr
        t = np.asarray(t, dtype=np.float32 if emulate else np.float64)
        diff = (y[..., :cr] - t[..., :cr])
        loss = float(np.sum(np.asarray(diff, dtype=np.float64) ** 2) / count)
        dy = np.zeros_like(y)
        if emulate:
            dy[..., :cr] = np.float32(2.0 / count) * diff.astype(np.float32)
            g = bf16(dy)
        else:
            dy[..., :cr] = 2.0 * diff / count
            g = dy
        grads = [None] * len(self.layers)
        for l in range(len(self.layers) - 1, -1, -1):
            dw = weight_grad(acts[l], g)
            db = np.sum(np.asarray(g, dtype=np.float64), axis=(0, 1, 2))
            grads[l] = (dw, db)
            if l > 0:
                w, _ = self._w(l, emulate)
                da = conv_transpose(g, w)
                gz = da * gelu_grad(np.asarray(zs[l - 1], dtype=np.float64))
                g = bf16(gz.astype(np.float32)) if emulate else gz
        return loss, grads


def adam_step(w, m, v, g, t, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One bias-corrected Adam step in float32, as the GPU kernel does it."""
    w, m, v, g = (np.asarray(a, dtype=np.float32) for a in (w, m, v, g))
    m = np.float32(b1) * m + np.float32(1 - b1) * g
    v = np.float32(b2) * v + np.float32(1 - b2) * g * g
    c1 = np.float32(1 - b1 ** t)
    c2 = np.float32(1 - b2 ** t)
    w = w - np.float32(lr) * (m / c1) / (np.sqrt(v / c2) + np.float32(eps))
    return w, m, v
