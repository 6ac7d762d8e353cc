"""mlp_oracle -- float64 numpy restatement of the autotuner cost model's
network (saruman_b200/csrc/costmodel.cu): forward pass, mean squared error,
its gradient by backpropagation, and one Adam step.

TEST INFRASTRUCTURE, NOT THE PRODUCT.  Only tests/ use it, as the checker of
the CUDA kernels' gradients.  The cost model has no counterpart in the
reference; this restates the standard mathematics of a tanh network (linear
output layer) and of Adam (Kingma and Ba, 2015), with the same parameter
layout as the kernels: per layer W (fan_out x fan_in, row-major), then the
bias.
"""
from __future__ import annotations

import numpy as np


def split(params: np.ndarray, dims: list[int]) -> list[tuple[np.ndarray, np.ndarray]]:
    out, off = [], 0
    for a, b in zip(dims[:-1], dims[1:]):
        W = params[off:off + a * b].reshape(b, a)
        off += a * b
        out.append((W, params[off:off + b]))
        off += b
    assert off == params.size
    return out


def forward(params: np.ndarray, dims: list[int], x: np.ndarray) -> list[np.ndarray]:
    """Activations of every layer (tanh hidden, linear last); [-1] is (n, 1)."""
    h = np.asarray(x, np.float64)
    acts = []
    layers = split(np.asarray(params, np.float64), dims)
    for i, (W, b) in enumerate(layers):
        z = h @ W.T + b
        h = z if i == len(layers) - 1 else np.tanh(z)
        acts.append(h)
    return acts


def loss_grad(params: np.ndarray, dims: list[int], x: np.ndarray,
              y: np.ndarray) -> tuple[float, np.ndarray]:
    """Mean squared error over the rows and its gradient (same layout)."""
    x = np.asarray(x, np.float64)
    y = np.asarray(y, np.float64).reshape(-1)
    n = x.shape[0]
    acts = forward(params, dims, x)
    layers = split(np.asarray(params, np.float64), dims)
    pred = acts[-1][:, 0]
    loss = float(np.mean((pred - y) ** 2))
    delta = (2.0 * (pred - y) / n)[:, None]
    grads = []
    for i in range(len(layers) - 1, -1, -1):
        W, _ = layers[i]
        h_in = acts[i - 1] if i else x
        grads.append((delta.T @ h_in, delta.sum(axis=0)))
        if i:
            delta = (delta @ W) * (1.0 - h_in ** 2)
    flat = []
    for gW, gb in reversed(grads):
        flat += [gW.reshape(-1), gb]
    return loss, np.concatenate(flat)


def adam(params, grad, m, v, lr, b1, b2, eps, step):
    m = b1 * m + (1 - b1) * grad
    v = b2 * v + (1 - b2) * grad * grad
    p = params - lr * (m / (1 - b1 ** step)) / (np.sqrt(v / (1 - b2 ** step)) + eps)
    return p, m, v
