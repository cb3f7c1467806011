"""Test infrastructure only: a float64 numpy restatement of the engine's cost-model MLP
(neonufft_b200/csrc/mlp.cu), the checker for its forward pass, gradients and Adam step.

Network: L weight layers with widths w_0..w_L; hidden layers tanh, output linear; parameters
per layer W_l (w_l x w_{l-1}, row-major) then b_l, concatenated. Loss: mean squared error.
The reference has no learned component; this oracle pins the engine's own kernels.
"""
from __future__ import annotations

import numpy as np


def param_count(widths) -> int:
    return int(sum(widths[l] * widths[l - 1] + widths[l] for l in range(1, len(widths))))


def unpack(widths, params):
    out, off = [], 0
    for l in range(1, len(widths)):
        n_in, n_out = widths[l - 1], widths[l]
        W = params[off:off + n_out * n_in].reshape(n_out, n_in)
        off += n_out * n_in
        b = params[off:off + n_out]
        off += n_out
        out.append((W, b))
    return out


def forward(widths, params, x):
    """Activations of every layer (list, batch-major); the last one is the output."""
    acts = []
    a = np.asarray(x, dtype=np.float64)
    layers = unpack(widths, np.asarray(params, dtype=np.float64))
    for l, (W, b) in enumerate(layers):
        z = a @ W.T + b
        a = np.tanh(z) if l < len(layers) - 1 else z
        acts.append(a)
    return acts


def backward(widths, params, x, acts, dy):
    """Gradient of the parameters for output gradient dy (same layout as params)."""
    layers = unpack(widths, np.asarray(params, dtype=np.float64))
    grads = [None] * len(layers)
    d = np.asarray(dy, dtype=np.float64)
    for l in range(len(layers) - 1, -1, -1):
        W, _ = layers[l]
        if l < len(layers) - 1:
            d = d * (1.0 - acts[l] ** 2)
        prev = acts[l - 1] if l > 0 else np.asarray(x, dtype=np.float64)
        grads[l] = (d.T @ prev, d.sum(axis=0))
        d = d @ W
    return np.concatenate([np.concatenate([gW.reshape(-1), gb]) for gW, gb in grads])


def mse(y, target):
    e = np.asarray(y, dtype=np.float64).reshape(-1) - np.asarray(target, dtype=np.float64)
    n = e.size
    return float((e * e).sum() / n), 2.0 * e / n


def adam(params, grads, m, v, lr, b1, b2, eps, step):
    m = b1 * m + (1 - b1) * grads
    v = b2 * v + (1 - b2) * grads * grads
    p = params - lr * (m / (1 - b1 ** step)) / (np.sqrt(v / (1 - b2 ** step)) + eps)
    return p, m, v
