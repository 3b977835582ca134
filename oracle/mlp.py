"""Test infrastructure only: a float64 numpy restatement of the learned SGS closure's
MLP (aerosim_b200/csrc/sgs_mlp.cuh) -- forward pass, mean-squared-error loss and its
gradient by explicit back-propagation -- against which the GPU training kernels are
checked.  The product never imports this module.

The closure has no counterpart in the reference (its closure is Smagorinsky,
src/solver/lbmCpuReference.ts:264-282); this oracle is pinned by central finite
differences of its own loss (tests/test_sgs_oracle.py).
"""
from __future__ import annotations

import numpy as np

N_IN, N_HID = 8, 32
_K = np.sqrt(2.0 / np.pi)


def unpack(p):
    p = np.asarray(p, np.float64)
    o = 0
    W1 = p[o:o + N_HID * N_IN].reshape(N_HID, N_IN); o += N_HID * N_IN
    b1 = p[o:o + N_HID]; o += N_HID
    W2 = p[o:o + N_HID * N_HID].reshape(N_HID, N_HID); o += N_HID * N_HID
    b2 = p[o:o + N_HID]; o += N_HID
    W3 = p[o:o + N_HID]; o += N_HID
    b3 = p[o]
    return W1, b1, W2, b2, W3, b3


def gelu(x):
    return 0.5 * x * (1.0 + np.tanh(_K * (x + 0.044715 * x ** 3)))


def gelu_grad(x):
    t = np.tanh(_K * (x + 0.044715 * x ** 3))
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * _K * (1.0 + 3.0 * 0.044715 * x * x)


def softplus(o):
    return np.where(o > 20.0, o, np.log1p(np.exp(np.minimum(o, 20.0))))


def forward(p, X):
    W1, b1, W2, b2, W3, b3 = unpack(p)
    X = np.asarray(X, np.float64)
    z1 = X @ W1.T + b1
    z2 = gelu(z1) @ W2.T + b2
    o = gelu(z2) @ W3 + b3
    return softplus(o), (X, z1, z2, o)


def loss_and_grad(p, X, Y):
    """Mean of (prediction - Y)^2 and its gradient (same layout as p)."""
    W1, b1, W2, b2, W3, b3 = unpack(p)
    pred, (X, z1, z2, o) = forward(p, X)
    n = X.shape[0]
    e = pred - np.asarray(Y, np.float64)
    loss = float(np.mean(e * e))
    d_o = 2.0 * e / (1.0 + np.exp(-o)) / n
    h1, h2 = gelu(z1), gelu(z2)
    gW3 = h2.T @ d_o
    gb3 = d_o.sum()
    d2 = np.outer(d_o, W3) * gelu_grad(z2)
    gW2 = d2.T @ h1
    gb2 = d2.sum(0)
    d1 = (d2 @ W2) * gelu_grad(z1)
    gW1 = d1.T @ X
    gb1 = d1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3, [gb3]])
    return loss, g
