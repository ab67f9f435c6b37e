"""float64 CPU oracle of the planner network (forward, loss, gradients).

TEST INFRASTRUCTURE ONLY (see graph_oracle.py).  Restates, in numpy float64,
the network that libmgbfs2's mlp kernels train and evaluate: inputs -> 64 ->
64 -> 2 with ReLU, parameters in one flat buffer
    W1[64][in] | b1[64] | W2[64][64] | b2[64] | W3[2][64] | b3[2],
loss = sum_s (w0 (y_s0 - t_s0)^2 + w1 (y_s1 - t_s1)^2) / batch.
The network has no counterpart in the reference; this oracle pins the GPU
kernels' gradients by analytic backpropagation cross-checked against central
finite differences.
"""
from __future__ import annotations

import numpy as np

HIDDEN, OUT = 64, 2


def split(params, inputs):
    p = np.asarray(params, dtype=np.float64)
    o = 0
    W1 = p[o:o + HIDDEN * inputs].reshape(HIDDEN, inputs); o += HIDDEN * inputs
    b1 = p[o:o + HIDDEN]; o += HIDDEN
    W2 = p[o:o + HIDDEN * HIDDEN].reshape(HIDDEN, HIDDEN); o += HIDDEN * HIDDEN
    b2 = p[o:o + HIDDEN]; o += HIDDEN
    W3 = p[o:o + OUT * HIDDEN].reshape(OUT, HIDDEN); o += OUT * HIDDEN
    b3 = p[o:o + OUT]; o += OUT
    assert o == p.size
    return W1, b1, W2, b2, W3, b3


def param_count(inputs):
    return HIDDEN * inputs + HIDDEN + HIDDEN * HIDDEN + HIDDEN + OUT * HIDDEN + OUT


def forward(params, x, inputs):
    W1, b1, W2, b2, W3, b3 = split(params, inputs)
    x = np.asarray(x, dtype=np.float64)
    a1 = x @ W1.T + b1
    h1 = np.maximum(a1, 0)
    a2 = h1 @ W2.T + b2
    h2 = np.maximum(a2, 0)
    return h2 @ W3.T + b3, (x, a1, h1, a2, h2)


def loss_and_grad(params, x, target, inputs, w=(1.0, 1.0)):
    W1, b1, W2, b2, W3, b3 = split(params, inputs)
    y, (x, a1, h1, a2, h2) = forward(params, x, inputs)
    t = np.asarray(target, dtype=np.float64)
    wv = np.asarray(w, dtype=np.float64)
    batch = x.shape[0]
    err = y - t
    loss = float((wv * err * err).sum() / batch)
    dy = 2.0 * wv * err / batch
    gW3 = dy.T @ h2
    gb3 = dy.sum(0)
    dh2 = (dy @ W3) * (a2 > 0)
    gW2 = dh2.T @ h1
    gb2 = dh2.sum(0)
    dh1 = (dh2 @ W2) * (a1 > 0)
    gW1 = dh1.T @ x
    gb1 = dh1.sum(0)
    grad = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return loss, grad


def finite_difference(params, x, target, inputs, w=(1.0, 1.0), idx=None, h=1e-6):
    p = np.asarray(params, dtype=np.float64).copy()
    idx = range(p.size) if idx is None else idx
    out = {}
    for i in idx:
        old = p[i]
        p[i] = old + h
        lp, _ = loss_and_grad(p, x, target, inputs, w)
        p[i] = old - h
        lm, _ = loss_and_grad(p, x, target, inputs, w)
        p[i] = old
        out[i] = (lp - lm) / (2 * h)
    return out
