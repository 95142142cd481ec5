"""CPU reference of the learned index's root network -- TEST INFRASTRUCTURE.

Float64 forward pass, mean-squared-error loss and its analytic gradient for
the one-hidden-layer network of ramp units the engine trains on the GPU
(y = b2 + sum_j w2[j] * ramp(w1[j] * x + b1[j]), ramp = clamp to [0, 1];
parameter vector [w1, b1, w2, b2]).  The tests check the GPU gradient kernel against it and it
against central finite differences.  The engine never imports this file.
"""
import numpy as np


def unpack(p, H):
    p = np.asarray(p, dtype=np.float64)
    return p[:H], p[H:2 * H], p[2 * H:3 * H], p[3 * H]


def forward(p, H, x):
    w1, b1, w2, b2 = unpack(p, H)
    h = np.outer(np.asarray(x, dtype=np.float64), w1) + b1
    return b2 + np.clip(h, 0.0, 1.0) @ w2


def loss(p, H, x, y):
    e = forward(p, H, x) - np.asarray(y, dtype=np.float64)
    return float(np.mean(e * e))


def loss_grad(p, H, x, y):
    w1, b1, w2, b2 = unpack(p, H)
    x = np.asarray(x, dtype=np.float64)
    h = np.outer(x, w1) + b1
    a = np.clip(h, 0.0, 1.0)
    e = b2 + a @ w2 - np.asarray(y, dtype=np.float64)
    n = len(x)
    dout = 2.0 * e / n
    g_w2 = a.T @ dout
    dh = ((h > 0) & (h < 1)) * np.outer(dout, w2)
    g_w1 = dh.T @ x
    g_b1 = dh.sum(axis=0)
    g_b2 = dout.sum()
    return float(np.mean(e * e)), np.concatenate([g_w1, g_b1, g_w2, [g_b2]])


def finite_diff_grad(p, H, x, y, h=1e-6):
    p = np.asarray(p, dtype=np.float64)
    g = np.zeros_like(p)
    for k in range(len(p)):
        a, b = p.copy(), p.copy()
        a[k] += h
        b[k] -= h
        g[k] = (loss(a, H, x, y) - loss(b, H, x, y)) / (2 * h)
    return g
