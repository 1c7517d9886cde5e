"""CPU checker for the warm-start network (test infrastructure only: tests import it, the
product never does).

The network has no counterpart in the reference, so its oracle is a plain FP64 numpy
restatement of the same model — fully connected layers, tanh on the hidden layers,
identity output, mean squared error — with the textbook backpropagation equations.  It is
itself checked against central finite differences (tests/test_mlp_oracle.py); parity of the
CUDA kernels is pinned to it, not to the reference.

Parameter layout (shared with csrc/mlp.cu): for each layer l, W_l (dims[l+1] x dims[l],
row-major) then b_l (dims[l+1]).
"""
from __future__ import annotations

import numpy as np


def split(params: np.ndarray, dims) -> list:
    """Views (W_l, b_l) of a flat parameter vector."""
    out, at = [], 0
    for l in range(len(dims) - 1):
        n_w = dims[l + 1] * dims[l]
        w = params[at:at + n_w].reshape(dims[l + 1], dims[l])
        at += n_w
        b = params[at:at + dims[l + 1]]
        at += dims[l + 1]
        out.append((w, b))
    assert at == params.size
    return out


def forward(params: np.ndarray, dims, x: np.ndarray) -> list:
    """Activations of every layer, input first; the last entry is the output (batch x 1)."""
    acts = [np.asarray(x, dtype=np.float64)]
    layers = split(np.asarray(params, dtype=np.float64), dims)
    for l, (w, b) in enumerate(layers):
        z = acts[-1] @ w.T + b
        acts.append(np.tanh(z) if l + 1 < len(layers) else z)
    return acts


def loss_and_gradients(params: np.ndarray, dims, x: np.ndarray, t: np.ndarray):
    """Mean squared error and its gradient (flat, same layout as params)."""
    p = np.asarray(params, dtype=np.float64)
    acts = forward(p, dims, x)
    y = acts[-1][:, 0]
    t = np.asarray(t, dtype=np.float64)
    batch = y.size
    loss = float(np.mean((y - t) ** 2))
    dz = (2.0 * (y - t) / batch)[:, None]
    layers = split(p, dims)
    grads = [None] * len(layers)
    for l in range(len(layers) - 1, -1, -1):
        w, _ = layers[l]
        grads[l] = (dz.T @ acts[l], dz.sum(axis=0))
        if l == 0:
            break
        da = dz @ w
        dz = da * (1.0 - acts[l] ** 2)
    flat = np.concatenate([np.concatenate([gw.ravel(), gb]) for gw, gb in grads])
    return loss, flat
