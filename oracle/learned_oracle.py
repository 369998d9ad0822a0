"""TEST INFRASTRUCTURE ONLY -- numpy oracle of the learned tail extrapolator.

A float64 numpy implementation of the network of tbplas_b200/learned.py
(three stride-s 1-D convolutions with GELU, then a dense layer; channel-last
activations; mean-squared-error loss) with forward and backward passes.  It
rounds to bfloat16 (round to nearest even) exactly where the GPU path feeds a
BF16 GEMM (inputs, weights, activations, output gradients), so the GPU
gradients can be checked against it to the precision of FP32 accumulation.
Used by tests/ only.
"""

import math

import numpy as np
from scipy.special import erf


def bf16(x: np.ndarray) -> np.ndarray:
    """Round to bfloat16 (nearest even), returned as float64."""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(x):
    return 0.5 * x * (1 + erf(x / math.sqrt(2)))


def gelu_grad(x):
    return 0.5 * (1 + erf(x / math.sqrt(2))) + x * np.exp(-0.5 * x * x) / math.sqrt(2 * math.pi)


def im2col(a, k, s, p, Lout):
    """a (B, L, C) -> (B*Lout, k*C) with [(b, lo), (j, c)] = a[b, lo*s + j - p, c]."""
    B, L, C = a.shape
    out = np.zeros((B, Lout, k, C))
    for j in range(k):
        for lo in range(Lout):
            l = lo * s + j - p
            if 0 <= l < L:
                out[:, lo, j, :] = a[:, l, :]
    return out.reshape(B * Lout, k * C)


def col2im(dcol, B, L, C, k, s, p, Lout):
    d = dcol.reshape(B, Lout, k, C)
    out = np.zeros((B, L, C))
    for j in range(k):
        for lo in range(Lout):
            l = lo * s + j - p
            if 0 <= l < L:
                out[:, l, :] += d[:, lo, j, :]
    return out


def forward_backward(params, convs, kernel, F, x_packed, target):
    """params: list of float arrays [W1, b1, W2, b2, W3, b3, Wd, bd] (the
    network's FP32 master weights); convs: layer geometry dicts (L, C, Lout,
    Cout, s, p); x_packed: (B, L0, C0) scaled, channel-padded input; target
    (B, O) scaled.  Returns (loss, output, grads)."""
    B = x_packed.shape[0]
    a = bf16(x_packed)
    cache = []
    for li, cv in enumerate(convs):
        W, b = params[2 * li], params[2 * li + 1]
        xcol = im2col(a, kernel, cv["s"], cv["p"], cv["Lout"])
        pre = xcol @ bf16(W).T + b
        a = bf16(gelu(pre)).reshape(B, cv["Lout"], cv["Cout"])
        cache.append((xcol, pre))
    Wd, bd = params[-2], params[-1]
    h = a.reshape(B, F)
    out = h @ bf16(Wd).T + bd
    diff = out - target
    loss = float(np.mean(diff ** 2))
    g = 2 * diff / diff.size
    grads = [None] * len(params)
    gb = bf16(g)
    grads[-2] = gb.T @ h
    grads[-1] = g.sum(axis=0)
    dA = gb @ bf16(Wd)
    for li in range(len(convs) - 1, -1, -1):
        cv = convs[li]
        W = params[2 * li]
        xcol, pre = cache[li]
        dz = dA.reshape(-1, cv["Cout"]) * gelu_grad(pre)
        grads[2 * li + 1] = dz.sum(axis=0)
        dzb = bf16(dz)
        grads[2 * li] = dzb.T @ xcol
        if li > 0:
            dxcol = dzb @ bf16(W)
            dA = col2im(dxcol, B, cv["L"], cv["C"], kernel, cv["s"], cv["p"], cv["Lout"])
    return loss, out, grads
