"""CPU oracle of the closure network (test infrastructure only).

The same computation as the GPU kernels of calypso_b200/csrc/cb2_closure.cu
in float64: weights rounded to bfloat16 (round to nearest even, as
__float2bfloat16_rn), biases float32, SiLU activations, mean squared error.
Used to check the GPU forward pass and gradients; nothing in the library
calls it."""
from __future__ import annotations

import numpy as np


def bf16_round(a: np.ndarray) -> np.ndarray:
    """float32 -> nearest bfloat16 (ties to even), returned as float64."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p: np.ndarray, nin: int, nhid: int, nout: int):
    o = 0
    W1 = p[o:o + nhid * nin].reshape(nhid, nin); o += nhid * nin
    b1 = p[o:o + nhid]; o += nhid
    W2 = p[o:o + nhid * nhid].reshape(nhid, nhid); o += nhid * nhid
    b2 = p[o:o + nhid]; o += nhid
    W3 = p[o:o + nout * nhid].reshape(nout, nhid); o += nout * nhid
    b3 = p[o:o + nout]
    return W1, b1, W2, b2, W3, b3


def _silu(z):
    return z / (1.0 + np.exp(-z))


def _dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(p, x, nin, nhid, nout):
    W1, b1, W2, b2, W3, b3 = unpack(np.asarray(p, np.float32), nin, nhid, nout)
    W1, W2, W3 = bf16_round(W1), bf16_round(W2), bf16_round(W3)
    b1, b2, b3 = (b.astype(np.float64) for b in (b1, b2, b3))
    x = np.asarray(x, np.float64)
    z1 = x @ W1.T + b1
    h1 = _silu(z1)
    z2 = h1 @ W2.T + b2
    h2 = _silu(z2)
    y = h2 @ W3.T + b3
    return y, (x, z1, h1, z2, h2, W1, W2, W3)


def loss_grad(p, x, t, nin, nhid, nout):
    """mean squared error and its gradient (same layout as the parameters)."""
    y, (x, z1, h1, z2, h2, W1, W2, W3) = forward(p, x, nin, nhid, nout)
    n = x.shape[0]
    d = y - np.asarray(t, np.float64)
    loss = float(np.mean(d * d))
    dy = 2.0 * d / (n * nout)
    gW3 = dy.T @ h2
    gb3 = dy.sum(0)
    dz2 = (dy @ W3) * _dsilu(z2)
    gW2 = dz2.T @ h1
    gb2 = dz2.sum(0)
    dz1 = (dz2 @ W2) * _dsilu(z1)
    gW1 = dz1.T @ x
    gb1 = dz1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return loss, g
