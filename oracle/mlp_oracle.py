"""CPU oracle of the learned MDF warm start's network (test infrastructure).

numpy restatement, in float64, of the MLP that csrc/mlp.cuh evaluates and
csrc/mlp_f32.cu trains: 64 -> 64 -> 64 -> 64 -> 2 with ReLU, inputs normalised
by the parameter block's header, mean squared error on the scaled targets,
back-propagation and one Adam step (beta1 0.9, beta2 0.999, eps 1e-8).  With
tc=True the hidden layers' products take TF32-rounded operands, as the
kernels' tensor-core layers do, so the comparison isolates accumulation order.  The
network has no counterpart in the reference, so this oracle is pinned by a
finite-difference check of its own gradient (tests/test_mlp_oracle.py), and
the GPU kernels are checked against it.
"""
from __future__ import annotations

import numpy as np

HDR = 132
SHAPES = [(64, 64), (64, 64), (64, 64), (64, 2)]
WLD = 72  # row stride of the 64 x 64 weight matrices in the parameter block


def _layout():
    out, off = [], HDR
    for fi, fo in SHAPES:
        ld = WLD if fo == 64 else fo
        out.append((off, ld, off + fi * ld, fi, fo))
        off += fi * ld + fo
    return out, off


def tf32(x):
    """Round float values to TF32 (10 explicit mantissa bits, to nearest, ties
    away from zero): the operand rounding of the tensor-core layers (PTX
    cvt.rna.tf32.f32)."""
    b = np.asarray(x, dtype=np.float32).view(np.uint32)
    return ((b + np.uint32(0x1000)) & np.uint32(0xFFFFE000)).view(np.float32).astype(np.float64)


def unpack(P):
    P = np.asarray(P, dtype=np.float64)
    mean, inv, yinv = P[0:64], P[64:128], P[128:130]
    lay, end = _layout()
    layers = []
    for w0, ld, b0, fi, fo in lay:
        W = P[w0:w0 + fi * ld].reshape(fi, ld)[:, :fo]
        layers.append((W, P[b0:b0 + fo]))
    return mean, inv, yinv, layers, end


def forward(P, X, tc=False):
    """Activations of every layer.  With tc, the operands of the three hidden
    layers' products are rounded to TF32 first, as the tensor cores take them
    (the normalised inputs in FP32 first, as the kernel forms them)."""
    mean, inv, yinv, layers, _ = unpack(P)
    if tc:
        a = ((np.asarray(X, dtype=np.float32) - mean.astype(np.float32)) * inv.astype(np.float32)).astype(np.float64)
    else:
        a = (np.asarray(X, dtype=np.float64) - mean) * inv
    acts = [a]
    for k, (W, b) in enumerate(layers):
        if tc and k < 3:
            z = tf32(acts[-1]) @ tf32(W) + b
        else:
            z = acts[-1] @ W + b
        acts.append(np.maximum(z, 0.0) if k < 3 else z)
    return acts


def predict(P, X, tc=False):
    _, _, yinv, _, _ = unpack(P)
    return forward(P, X, tc)[-1] / yinv


def loss_and_grad(P, X, T, tc=False):
    """L = (1/n) sum (y - t * yinv)^2 and dL/dP (header and padding entries
    zero).  With tc, the hidden layers' products (forward, weight gradients,
    back-propagated deltas) take TF32-rounded operands as on the tensor cores."""
    mean, inv, yinv, layers, npar = unpack(P)
    n = X.shape[0]
    acts = forward(P, X, tc)
    r = acts[-1] - np.asarray(T, dtype=np.float64) * yinv
    L = float((r * r).sum() / n)
    d = 2.0 * r / n
    rnd = tf32 if tc else (lambda x: x)
    grads = []
    for k in range(3, -1, -1):
        W, b = layers[k]
        hid = k < 3  # the output layer runs on CUDA cores
        grads.append(((rnd(acts[k]).T @ rnd(d)) if hid else acts[k].T @ d, d.sum(0)))
        if k > 0:
            d = ((rnd(d) @ rnd(W).T) if hid else d @ W.T) * (acts[k] > 0.0)
    grads.reverse()
    g = np.zeros(npar)
    for (gW, gb), (w0, ld, b0, fi, fo) in zip(grads, _layout()[0]):
        g[w0:w0 + fi * ld].reshape(fi, ld)[:, :fo] = gW
        g[b0:b0 + fo] = gb
    return L, g


def adam_step(P, g, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    P, g, m, v = (np.asarray(x, dtype=np.float64).copy() for x in (P, g, m, v))
    sl = slice(HDR, None)
    m[sl] = b1 * m[sl] + (1 - b1) * g[sl]
    v[sl] = b2 * v[sl] + (1 - b2) * g[sl] ** 2
    c1, c2 = 1.0 / (1.0 - b1 ** step), 1.0 / (1.0 - b2 ** step)
    P[sl] -= lr * (m[sl] * c1) / (np.sqrt(v[sl] * c2) + eps)
    return P, m, v
