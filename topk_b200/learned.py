"""The learned k-th-score model: standalone MLP entry points of the C ABI.

The model (in_dim -> 64 -> 64 -> 1, ReLU, FP32) is trained and served by the
library's own CUDA kernels (mlp.cu); these wrappers move host arrays in and out.
Parameter layout: W1[64][in_dim] b1[64] W2[64][64] b2[64] w3[64] b3.
"""
import ctypes as C

import numpy as np

from . import _lib
from ._lib import check

HIDDEN = 64


def param_count(in_dim):
    return int(_lib.load().topk_mlp_param_count(int(in_dim)))


def _f32(a):
    return np.ascontiguousarray(a, np.float32)


def grad(params, X, y, device=0):
    """(loss, gradient) of the mean squared error over one batch (<= 128 rows)."""
    X = _f32(X)
    y = _f32(y).reshape(-1)
    params = _f32(params).reshape(-1)
    g = np.empty_like(params)
    loss = C.c_float()
    check(_lib.load().topk_mlp_grad(int(device), X.shape[1], params, X.reshape(-1), y, len(y), g, C.byref(loss)))
    return loss.value, g


def predict(params, X, device=0):
    X = _f32(X)
    out = np.empty(X.shape[0], np.float32)
    check(_lib.load().topk_mlp_predict(int(device), X.shape[1], _f32(params).reshape(-1), X.reshape(-1), X.shape[0],
                                       out))
    return out


def train(params, X, y, epochs, batch=128, lr=1e-3, seed=0, device=0):
    """Adam on the device; returns (trained params, per-epoch loss)."""
    X = _f32(X)
    p = _f32(params).reshape(-1).copy()
    losses = np.zeros(max(int(epochs), 1), np.float32)
    check(_lib.load().topk_mlp_train(int(device), X.shape[1], p, X.reshape(-1), _f32(y).reshape(-1), X.shape[0],
                                     int(epochs), int(batch), float(lr), int(seed), losses.ctypes.data))
    return p, losses[: int(epochs)]


def init_params(in_dim, seed=0, bias=0.0):
    """Uniform +-sqrt(6 / fan_in) weights, zero hidden biases, output bias `bias`."""
    rng = np.random.default_rng(seed)
    p = np.zeros(param_count(in_dim), np.float32)
    o = 0
    p[o:o + HIDDEN * in_dim] = rng.uniform(-1, 1, HIDDEN * in_dim) * np.sqrt(6.0 / in_dim)
    o += HIDDEN * in_dim + HIDDEN
    p[o:o + HIDDEN * HIDDEN] = rng.uniform(-1, 1, HIDDEN * HIDDEN) * np.sqrt(6.0 / HIDDEN)
    o += HIDDEN * HIDDEN + HIDDEN
    p[o:o + HIDDEN] = rng.uniform(-1, 1, HIDDEN) * np.sqrt(6.0 / HIDDEN)
    p[-1] = bias
    return p
