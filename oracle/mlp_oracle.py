"""CPU oracle of the learned MDF warm start's network (test infrastructure).

numpy restatement, in float64, of the MLP that csrc/mlp.cuh evaluates and
csrc/mlp_f32.cu trains: 64 -> 64 -> 64 -> 64 -> 2 with ReLU, inputs normalised
by the parameter block's header, mean squared error on the scaled targets,
back-propagation and one Adam step (beta1 0.9, beta2 0.999, eps 1e-8).  The
network has no counterpart in the reference, so this oracle is pinned by a
finite-difference check of its own gradient (tests/test_mlp_oracle.py), and
the GPU kernels are checked against it.
"""
from __future__ import annotations

import numpy as np

HDR = 132
SHAPES = [(64, 64), (64, 64), (64, 64), (64, 2)]


def unpack(P):
    P = np.asarray(P, dtype=np.float64)
    mean, inv, yinv = P[0:64], P[64:128], P[128:130]
    layers, off = [], HDR
    for fi, fo in SHAPES:
        W = P[off:off + fi * fo].reshape(fi, fo)
        off += fi * fo
        b = P[off:off + fo]
        off += fo
        layers.append((W, b))
    return mean, inv, yinv, layers, off


def forward(P, X):
    mean, inv, yinv, layers, _ = unpack(P)
    a = (np.asarray(X, dtype=np.float64) - mean) * inv
    acts = [a]
    for k, (W, b) in enumerate(layers):
        z = acts[-1] @ W + b
        acts.append(np.maximum(z, 0.0) if k < 3 else z)
    return acts


def predict(P, X):
    _, _, yinv, _, _ = unpack(P)
    return forward(P, X)[-1] / yinv


def loss_and_grad(P, X, T):
    """L = (1/n) sum (y - t * yinv)^2 and dL/dP (header entries zero)."""
    mean, inv, yinv, layers, npar = unpack(P)
    n = X.shape[0]
    acts = forward(P, X)
    r = acts[-1] - np.asarray(T, dtype=np.float64) * yinv
    L = float((r * r).sum() / n)
    d = 2.0 * r / n
    grads = []
    for k in range(3, -1, -1):
        W, b = layers[k]
        grads.append((acts[k].T @ d, d.sum(0)))
        if k > 0:
            d = (d @ W.T) * (acts[k] > 0.0)
    grads.reverse()
    g = np.zeros(npar)
    off = HDR
    for (gW, gb), (fi, fo) in zip(grads, SHAPES):
        g[off:off + fi * fo] = gW.ravel()
        off += fi * fo
        g[off:off + fo] = gb
        off += fo
    return L, g


def adam_step(P, g, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    P, g, m, v = (np.asarray(x, dtype=np.float64).copy() for x in (P, g, m, v))
    sl = slice(HDR, None)
    m[sl] = b1 * m[sl] + (1 - b1) * g[sl]
    v[sl] = b2 * v[sl] + (1 - b2) * g[sl] ** 2
    c1, c2 = 1.0 / (1.0 - b1 ** step), 1.0 / (1.0 - b2 ** step)
    P[sl] -= lr * (m[sl] * c1) / (np.sqrt(v[sl] * c2) + eps)
    return P, m, v
