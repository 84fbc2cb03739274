"""CPU oracle of libmfgpu's cost-model MLP (test infrastructure only).

The network of csrc/costmodel.cu restated in numpy (float64): layers
nin -> h -> h -> 1 with tanh hidden activations, loss (1/n) sum (f(x) - y)^2,
parameters laid out as W1 (h x nin, row-major), b1, W2 (h x h), b2, w3 (h),
b3.  Used to check the GPU forward pass and gradients; it has no counterpart
in the reference (PureUMFPACK.jl has no learned components).
"""

from __future__ import annotations

import numpy as np


def split(p, nin, h):
    p = np.asarray(p, dtype=np.float64)
    o = 0
    W1 = p[o:o + h * nin].reshape(h, nin); o += h * nin
    b1 = p[o:o + h]; o += h
    W2 = p[o:o + h * h].reshape(h, h); o += h * h
    b2 = p[o:o + h]; o += h
    w3 = p[o:o + h]; o += h
    b3 = p[o]
    return W1, b1, W2, b2, w3, b3


def nparams(nin, h):
    return h * nin + h + h * h + h + h + 1


def forward(p, X, nin, h):
    W1, b1, W2, b2, w3, b3 = split(p, nin, h)
    X = np.asarray(X, dtype=np.float64)
    a1 = np.tanh(X @ W1.T + b1)
    a2 = np.tanh(a1 @ W2.T + b2)
    return a2 @ w3 + b3, a1, a2


def loss_grad(p, X, Y, nin, h):
    """Loss and its gradient, by the chain rule written out layer by layer."""
    W1, b1, W2, b2, w3, b3 = split(p, nin, h)
    X = np.asarray(X, dtype=np.float64)
    Y = np.asarray(Y, dtype=np.float64)
    n = len(Y)
    out, a1, a2 = forward(p, X, nin, h)
    r = out - Y
    loss = float(np.mean(r * r))
    d3 = 2.0 * r / n                      # dL/d out
    d2 = (d3[:, None] * w3[None, :]) * (1.0 - a2 * a2)
    d1 = (d2 @ W2) * (1.0 - a1 * a1)
    g = np.concatenate([(d1.T @ X).ravel(), d1.sum(0), (d2.T @ a1).ravel(), d2.sum(0), a2.T @ d3, [d3.sum()]])
    return loss, g
