"""FP32 reference of the learned-bound MLP and its features (test
infrastructure only).

The GPU kernels multiply BF16 operands on the tensor cores with FP32
accumulation; this reference rounds the same tensors to BF16 at the same
points (inputs, weights, the layer-1 activations, the stored layer-2
activations and the backward operands) and accumulates in float64, so the two
agree to FP32 accumulation-order tolerance.  Parameter layout: W1 [128 x 128] |
b1 [128] | W2 [128 x 128] | b2 [128] | w3 [128] | b3.
"""
from __future__ import annotations

import numpy as np


def bf16(x) -> np.ndarray:
    """Round to bfloat16 (nearest even), returned as float32."""
    b = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16).astype(np.uint32) << 16
    return r.view(np.float32)


def unpack(p):
    p = np.asarray(p, np.float32)
    W1 = p[:16384].reshape(128, 128)
    b1 = p[16384:16512]
    W2 = p[16512:32896].reshape(128, 128)
    b2 = p[32896:33024]
    w3 = p[33024:33152]
    b3 = p[33152]
    return W1, b1, W2, b2, w3, b3


def forward(p, X):
    """X: float32 [n, 128] (already BF16 values).  Returns y and activations."""
    W1, b1, W2, b2, w3, b3 = unpack(p)
    X = np.asarray(X, np.float64)
    z1 = X @ bf16(W1).astype(np.float64).T + b1
    h1 = bf16(np.maximum(z1, 0).astype(np.float32))
    z2 = h1.astype(np.float64) @ bf16(W2).astype(np.float64).T + b2
    h2 = np.maximum(z2, 0)
    y = h2 @ w3.astype(np.float64) + float(b3)
    return y, h1, bf16(h2.astype(np.float32))


def gradients(p, X, t):
    """Gradients of mean (y - t)^2 in the flat parameter layout, and the loss."""
    W1, b1, W2, b2, w3, b3 = unpack(p)
    n = X.shape[0]
    y, h1, h2b = forward(p, X)
    e = y - np.asarray(t, np.float64)
    dy = 2.0 * e / n
    g = np.zeros(p.size, np.float64)
    g[33024:33152] = dy @ h2b.astype(np.float64)
    g[33152] = dy.sum()
    dz2 = dy[:, None] * w3.astype(np.float64)[None, :] * (h2b > 0)
    g[32896:33024] = dz2.sum(0)
    dz2b = bf16(dz2.astype(np.float32)).astype(np.float64)
    g[16512:32896] = (dz2b.T @ h1.astype(np.float64)).ravel()
    dh1 = dz2b @ bf16(W2).astype(np.float64)
    dz1 = dh1 * (h1 > 0)
    g[16384:16512] = dz1.sum(0)
    dz1b = bf16(dz1.astype(np.float32)).astype(np.float64)
    g[:16384] = (dz1b.T @ np.asarray(X, np.float64)).ravel()
    return g, float((e * e).mean())


def features(U, V, eb_a, idx):
    """The 99 features (float32, before BF16 rounding) of raster vertices idx."""
    U = np.asarray(U, np.float32)
    V = np.asarray(V, np.float32)
    r1, r2 = U.shape
    out = np.zeros((len(idx), 128), np.float32)
    for s, v in enumerate(idx):
        i, j = divmod(int(v), r2)
        pu = np.zeros((7, 7), np.float32)
        pv = np.zeros((7, 7), np.float32)
        for di in range(7):
            for dj in range(7):
                ii, jj = i + di - 3, j + dj - 3
                if 0 <= ii < r1 and 0 <= jj < r2:
                    pu[di, dj] = U[ii, jj]
                    pv[di, dj] = V[ii, jj]
        mx = np.float32(max(np.abs(pu).max(), np.abs(pv).max()))
        sc = np.float32(1.0) / mx if (mx > 0 and np.isfinite(mx)) else np.float32(1.0)
        out[s, :49] = pu.ravel() * sc
        out[s, 49:98] = pv.ravel() * sc
        out[s, 98] = np.float32(np.log2(max(float(eb_a[v]), 1e-30)) / 32.0)
    return out
