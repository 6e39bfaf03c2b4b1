"""numpy FP64 restatement of the shock-sensor network (test infrastructure only).

Layout and arithmetic as the library's dgk_mlp_* kernels: W1[32][nin], b1[32], W2[32][32], b2[32], w3[32], b3;
h1 = tanh(W1 x + b1), h2 = tanh(W2 h1 + b2), out = sigmoid(w3 . h2 + b3); loss = mean (out - y)^2.  The
gradient is the textbook backward pass of that composition (chain rule), checked here against finite
differences before it is used to check the GPU gradient.
"""
from __future__ import annotations

import numpy as np

H = 32


def unpack(p, nin):
    p = np.asarray(p, dtype=np.float64)
    o = 0
    W1 = p[o:o + H * nin].reshape(H, nin); o += H * nin
    b1 = p[o:o + H]; o += H
    W2 = p[o:o + H * H].reshape(H, H); o += H * H
    b2 = p[o:o + H]; o += H
    w3 = p[o:o + H]; o += H
    b3 = p[o]
    return W1, b1, W2, b2, w3, b3


def forward(p, X, nin):
    W1, b1, W2, b2, w3, b3 = unpack(p, nin)
    X = np.asarray(X, dtype=np.float64)
    h1 = np.tanh(X @ W1.T + b1)
    h2 = np.tanh(h1 @ W2.T + b2)
    z = h2 @ w3 + b3
    return 1.0 / (1.0 + np.exp(-z)), (h1, h2)


def loss_grad(p, X, y, nin):
    W1, b1, W2, b2, w3, b3 = unpack(p, nin)
    X = np.asarray(X, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    n = X.shape[0]
    o, (h1, h2) = forward(p, X, nin)
    r = o - y
    loss = float(np.mean(r * r))
    dz = 2.0 * r * o * (1.0 - o) / n
    gw3 = h2.T @ dz
    gb3 = dz.sum()
    d2 = np.outer(dz, w3) * (1.0 - h2 * h2)
    gW2 = d2.T @ h1
    gb2 = d2.sum(0)
    d1 = (d2 @ W2) * (1.0 - h1 * h1)
    gW1 = d1.T @ X
    gb1 = d1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gw3, [gb3]])
    return loss, g


def to_fp16(p):
    """Parameters rounded to FP16 (the stage's inference weights), back in FP64."""
    return np.asarray(p, dtype=np.float32).astype(np.float16).astype(np.float64)
