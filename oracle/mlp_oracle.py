"""Float64 NumPy restatement of the surrogate network's forward and backward
passes -- TEST INFRASTRUCTURE ONLY (the test oracle of traceon_b200's tb_mlp_*
kernels; nothing in the product imports it).

It emulates the BF16 roundings of the GPU path at the same places (inputs,
weights, hidden activations, back-propagated gradients) and otherwise works in
float64, so the GPU's FP32-accumulated results are compared against an exact
computation of the same rounded operands.
"""
from __future__ import annotations

import numpy as np

IN, H, OUT = 16, 128, 32
LAYERS = [('W1', 'b1', IN, H), ('W2', 'b2', H, H), ('W3', 'b3', H, H), ('W4', 'b4', H, H), ('W5', 'b5', H, OUT)]


def offsets():
    off, o = {}, 0
    for W, b, fin, fout in LAYERS:
        off[W] = (o, fout * fin)
        o += fout * fin
        off[b] = (o, fout)
        o += fout
    return off, o


def bf16(x):
    """Round to bfloat16 (nearest, ties to even) and return as float64."""
    a = np.asarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def silu(z):
    return z / (1 + np.exp(-z))


def silu_grad(z):
    s = 1 / (1 + np.exp(-z))
    return s * (1 + z * (1 - s))


def unpack(params):
    off, _ = offsets()
    p = np.asarray(params, dtype=np.float64)
    out = {}
    for W, b, fin, fout in LAYERS:
        o, n = off[W]
        out[W] = p[o:o + n].reshape(fout, fin)
        o, n = off[b]
        out[b] = p[o:o + n]
    return out


def forward(params, X):
    """X (M, 16) -> outputs (M, 32); returns (out, pre-activations, activations)."""
    P = unpack(params)
    a = bf16(X)
    acts, pre = [a], []
    for W, b, fin, fout in LAYERS:
        z = a @ bf16(P[W]).T + P[b]
        if W != 'W5':
            pre.append(z)
            a = bf16(silu(z))
            acts.append(a)
        else:
            out = z
    return out, pre, acts


def loss_and_grad(params, X, T, n_out):
    """MSE over the first n_out outputs and its gradient (flat, float64)."""
    P = unpack(params)
    off, n = offsets()
    out, pre, acts = forward(params, X)
    M = len(X)
    d = out[:, :n_out] - T
    loss = np.mean(d ** 2)
    g = np.zeros((M, OUT))
    g[:, :n_out] = 2 * d / (M * n_out)
    g = bf16(g)
    grad = np.zeros(n)
    for li in range(len(LAYERS) - 1, -1, -1):
        W, b, fin, fout = LAYERS[li]
        o, k = off[W]
        grad[o:o + k] = (g.T @ acts[li]).reshape(-1)
        o, k = off[b]
        grad[o:o + k] = g.sum(0)
        if li == 0:
            break
        dA = g @ bf16(P[W])
        g = bf16(dA * silu_grad(pre[li - 1]))
    return loss, grad
