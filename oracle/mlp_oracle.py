"""Test infrastructure only: FP64 CPU restatement of the learned k-th-score model.

The model is this library's own (no reference counterpart): in_dim -> 64 -> 64 -> 1
with ReLU, mean squared error, parameters in one flat array
W1[64][in_dim] b1[64] W2[64][64] b2[64] w3[64] b3 (the layout of
topk_b200/csrc/mlp.cu).  Used to check the device's forward pass and gradients.
Pinned by finite differences in tests/test_mlp_oracle.py.
"""
import numpy as np

H = 64


def unpack(p, F):
    p = np.asarray(p, np.float64)
    o = 0
    W1 = p[o:o + H * F].reshape(H, F); o += H * F
    b1 = p[o:o + H]; o += H
    W2 = p[o:o + H * H].reshape(H, H); o += H * H
    b2 = p[o:o + H]; o += H
    w3 = p[o:o + H]; o += H
    b3 = p[o]
    return W1, b1, W2, b2, w3, b3


def forward(p, X):
    X = np.asarray(X, np.float64)
    W1, b1, W2, b2, w3, b3 = unpack(p, X.shape[1])
    h1 = np.maximum(X @ W1.T + b1, 0.0)
    h2 = np.maximum(h1 @ W2.T + b2, 0.0)
    return h2 @ w3 + b3, h1, h2


def loss_grad(p, X, y):
    """(mean squared error, gradient) in float64."""
    X = np.asarray(X, np.float64)
    y = np.asarray(y, np.float64)
    B, F = X.shape
    W1, b1, W2, b2, w3, b3 = unpack(p, F)
    out, h1, h2 = forward(p, X)
    r = out - y
    loss = float(np.mean(r * r))
    dy = 2.0 * r / B
    gw3 = h2.T @ dy
    gb3 = dy.sum()
    d2 = np.outer(dy, w3) * (h2 > 0)
    gW2 = d2.T @ h1
    gb2 = d2.sum(axis=0)
    d1 = (d2 @ W2) * (h1 > 0)
    gW1 = d1.T @ X
    gb1 = d1.sum(axis=0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gw3, [gb3]])
    return loss, g
