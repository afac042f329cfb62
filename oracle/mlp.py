"""CPU restatement of the learned probe predictor (numpy, float64).

TEST INFRASTRUCTURE ONLY: the tests use it to check the CUDA training and
inference kernels; nothing in the product imports it.

The predictor has no counterpart in the reference (whose nprobe is fixed per
call, src/Index.cpp search path); its specification is this project's:

* features of a query from its P best coarse scores s[0..P-1] (ascending for
  L2): f0 = log(|s0| + 1e-6), fi = log1p(max(s[min(i, P-1)] - s0, 0) /
  (|s0| + 1e-6)) for i = 1..63, then standardised with the training mean/sd;
* stop label = 1 + the largest probe rank among the lists holding the exact
  top-k rows (the smallest nprobe that finds all of them);
* network 64 -> 256 -> 256 -> 1, GELU (erf form) on the hidden layers, matrix
  products whose inputs are rounded to bf16 (round to nearest even) with
  wide accumulation, MSE loss on log2(label);
* parameters packed as W1[64x256] b1[256] W2[256x256] b2[256] W3[256] b3[1],
  row-major, y = x W + b.
"""
import math

import numpy as np
from scipy.special import erf

IN, H = 64, 256
W1 = 0
B1 = W1 + IN * H
W2 = B1 + H
B2 = W2 + H * H
W3 = B2 + H
B3 = W3 + H
NPARAM = B3 + 1


def bf16_round(a):
    """Round float32 values to the nearest bf16 (ties to even), as float64."""
    f = np.ascontiguousarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    r = ((u + 0x7FFF + lsb) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32).astype(np.float64)
    nan = np.isnan(f)
    if nan.any():
        out[nan] = np.nan
    return out


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    return (p[W1:B1].reshape(IN, H), p[B1:W2], p[W2:B2].reshape(H, H), p[B2:W3], p[W3:B3].reshape(H, 1), p[B3:NPARAM])


def _mm(a, b, rounding):
    if rounding:
        return bf16_round(a) @ bf16_round(b)
    return np.asarray(a, np.float64) @ np.asarray(b, np.float64)


def gelu(z):
    return 0.5 * z * (1.0 + erf(z / math.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + erf(z / math.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / math.sqrt(2.0 * math.pi)


def forward(p, X, rounding=True):
    w1, b1, w2, b2, w3, b3 = unpack(p)
    z1 = _mm(X, w1, rounding) + b1
    a1 = gelu(z1)
    z2 = _mm(a1, w2, rounding) + b2
    a2 = gelu(z2)
    y = (_mm(a2, w3, rounding) + b3)[:, 0]
    return y, (z1, a1, z2, a2)


def loss_grad(p, X, t, rounding=True):
    """MSE loss and its gradient with respect to every parameter."""
    X = np.asarray(X, np.float64)
    t = np.asarray(t, np.float64)
    B = X.shape[0]
    w1, b1, w2, b2, w3, b3 = unpack(p)
    y, (z1, a1, z2, a2) = forward(p, X, rounding)
    e = y - t
    loss = float(np.mean(e * e))
    dy = (2.0 * e / B)[:, None]
    g = np.zeros(NPARAM)
    g[W3:B3] = _mm(a2.T, dy, rounding)[:, 0]
    g[B3] = dy.sum()
    dz2 = _mm(dy, w3.T, rounding) * gelu_grad(z2)
    g[W2:B2] = _mm(a1.T, dz2, rounding).ravel()
    g[B2:W3] = dz2.sum(0)
    dz1 = _mm(dz2, w2.T, rounding) * gelu_grad(z1)
    g[W1:B1] = _mm(X.T, dz1, rounding).ravel()
    g[B1:W2] = dz1.sum(0)
    return loss, g


def features(scores):
    """Raw (unstandardised) features of each row of `scores` (n x P, best first)."""
    s = np.asarray(scores, np.float32)
    n, P = s.shape
    a0 = np.abs(s[:, 0]) + np.float32(1e-6)
    X = np.empty((n, IN), np.float64)
    X[:, 0] = np.log(a0)
    for f in range(1, IN):
        X[:, f] = np.log1p(np.maximum(s[:, min(f, P - 1)] - s[:, 0], 0.0) / a0)
    return X


def stop_labels(row_lists, probes):
    """row_lists: n x k list id of each exact top-k row (-1 = none); probes:
    n x P lists best first.  Returns 1 + the largest probe rank."""
    n, P = probes.shape
    out = np.ones(n, np.float64)
    for i in range(n):
        rank = {int(l): j for j, l in enumerate(probes[i])}
        worst = 0
        for l in row_lists[i]:
            if l >= 0:
                worst = max(worst, rank.get(int(l), P - 1))
        out[i] = worst + 1
    return out


def nprobe_from_prediction(y, margin, P):
    return np.clip(np.ceil(np.exp2(np.minimum(np.asarray(y, np.float64) + margin, 30.0))), 1, P).astype(np.int64)
