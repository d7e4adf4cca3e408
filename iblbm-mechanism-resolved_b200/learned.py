"""Learned MDF warm start: a small MLP that predicts each marker's converged
multi-direct-forcing force from its state before the first iteration.

Per marker the band kernel forms 64 features (csrc/band_kernel.cuh): the slip
velocity before any correction, the working velocities at its stencil nodes,
its sub-node offset, its angular position on the body, the delta kernel, the
Reynolds number, the interpolated density and the slips of its two
neighbouring markers.  The target is the force the plain MDF loop applies to
it in total, sum over iterations of omega * Lf (``collect`` can run the loop
past its usual limit to record forces closer to convergence).
Training pairs come from plain MDF runs (``collect``); training and inference
run on the GPU in this library's own kernels (``iblbm_mlp_train_step``: fused
forward and backward per block of 64 samples, then an ordered sum of the
blocks' gradients and Adam, so training is deterministic;
``iblbm_mlp_infer``), the hidden layers on the tensor cores (TF32 operands,
FP32 accumulation).  With the warm
start on, the band kernel spreads the predicted forces before the first
iteration and then iterates as plain MDF does, to the same residual
tolerance: plain MDF is both the fallback and the arbiter of the slip.
"""
from __future__ import annotations

import numpy as np

from ._lib import check, lib, ptr

N_FEATURES = 64
N_OUT = 2
HIDDEN = 64
HDR = 132   # header of the parameter block (normalisation and target scales)
WLD = 72    # row stride of the hidden layers' weight matrices (csrc/mlp.cuh)


def layer_offsets():
    """(weight offset, row stride, bias offset, fan_in, fan_out) of the four
    layers in the parameter block."""
    out, off = [], HDR
    for fan_in, fan_out in ((N_FEATURES, HIDDEN), (HIDDEN, HIDDEN), (HIDDEN, HIDDEN), (HIDDEN, N_OUT)):
        ld = WLD if fan_out == HIDDEN else fan_out
        out.append((off, ld, off + fan_in * ld, fan_in, fan_out))
        off += fan_in * ld + fan_out
    return out


class MdfNet:
    """The network's parameters and Adam state on one device."""

    def __init__(self, device=None, seed=0):
        import torch
        self.torch = torch
        self.L = lib()
        self.dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.NP = int(self.L.iblbm_mlp_param_count())
        rng = np.random.default_rng(seed)
        p = np.zeros(self.NP, dtype=np.float32)
        p[64:128] = 1.0
        p[128:130] = 1.0
        for w0, ld, b0, fan_in, fan_out in layer_offsets():
            W = rng.standard_normal((fan_in, fan_out)).astype(np.float32) * np.float32(np.sqrt(2.0 / fan_in))
            for i in range(fan_in):  # row i of W, then the row's unused floats; biases start at zero
                p[w0 + i * ld:w0 + i * ld + fan_out] = W[i]
        assert b0 + fan_out <= self.NP  # the block is padded to a multiple of 4 floats
        self.params = torch.as_tensor(p, device=self.dev)
        self.m = torch.zeros(self.NP, dtype=torch.float32, device=self.dev)
        self.v = torch.zeros_like(self.m)
        self.grad = torch.zeros(int(self.L.iblbm_mlp_grad_floats(512)), dtype=torch.float32, device=self.dev)
        self.loss = torch.zeros(1, dtype=torch.float32, device=self.dev)
        self.step = 0

    def set_normalisation(self, X, T):
        """Feature mean / inverse spread and target scale from training data
        (features that never vary get scale 1)."""
        torch = self.torch
        mean = X.mean(0)
        std = X.std(0)
        inv = torch.where(std > 1e-6, 1.0 / std.clamp_min(1e-6), torch.ones_like(std))
        tscale = T.abs().mean(0).clamp_min(1e-12)
        with torch.no_grad():
            self.params[0:64] = mean
            self.params[64:128] = inv
            self.params[128:130] = 1.0 / tscale

    def train_step(self, X, T, lr=1e-3, apply=True):
        """One optimiser step on the rows of X (n x 64) and T (n x 2); returns
        nothing (the loss accumulates in self.loss)."""
        s = self.torch.cuda.current_stream(self.dev).cuda_stream
        n = int(X.shape[0])
        need = int(self.L.iblbm_mlp_grad_floats(n))
        if self.grad.numel() < need:
            self.grad = self.torch.zeros(need, dtype=self.torch.float32, device=self.dev)
        self.step += 1 if apply else 0
        check(self.L.iblbm_mlp_train_step(ptr(self.params), ptr(self.m), ptr(self.v), ptr(self.grad), ptr(X),
                                          ptr(T), n, float(lr), max(self.step, 1), ptr(self.loss), int(apply), s),
              "iblbm_mlp_train_step")

    def summed_gradient(self):
        """The gradient a train_step(..., apply=False) left (param_count floats)."""
        return self.grad[: self.NP]

    def fit(self, X, T, epochs=30, batch=512, lr=1e-3, seed=0):
        """Minibatch Adam over shuffled data; returns the mean loss of each epoch."""
        torch = self.torch
        X = X.to(self.dev, torch.float32).contiguous()
        T = T.to(self.dev, torch.float32).contiguous()
        self.set_normalisation(X, T)
        g = torch.Generator(device=self.dev)
        g.manual_seed(seed)
        n = X.shape[0]
        hist = []
        for _ in range(epochs):
            perm = torch.randperm(n, device=self.dev, generator=g)
            self.loss.zero_()
            nb = 0
            for s in range(0, n - batch + 1, batch):
                idx = perm[s:s + batch]
                self.train_step(X[idx].contiguous(), T[idx].contiguous(), lr)
                nb += 1
            hist.append(float(self.loss.item()) / max(nb, 1))
        return hist

    def predict(self, X):
        torch = self.torch
        X = X.to(self.dev, torch.float32).contiguous()
        Y = torch.empty(X.shape[0], 2, dtype=torch.float32, device=self.dev)
        check(self.L.iblbm_mlp_infer(ptr(self.params), ptr(X), int(X.shape[0]), ptr(Y),
                                     self.torch.cuda.current_stream(self.dev).cuda_stream), "iblbm_mlp_infer")
        return Y


def collect(engine, steps, iterations=None):
    """Run `steps` timesteps of an FP32 MDF engine in plain MDF, recording each
    marker's features and accumulated force every step.  With `iterations` the
    MDF loop runs exactly that many iterations during collection (far past the
    usual limit, so the targets are the converged forces) and the engine's own
    limits are restored afterwards.  Returns (X, T) as device tensors of
    (steps * markers) rows and the MDF iteration counts."""
    torch = engine.torch
    saved = [(a.mdf_iterations, a.mdf_min_iterations) for a in engine.ibm_args]
    if iterations:
        for a in engine.ibm_args:
            a.mdf_iterations = a.mdf_min_iterations = int(iterations)
    engine.set_mlp(mode=1)
    X, T, its = [], [], []
    for _ in range(steps):
        engine.advance(1, outputs_last=False, use_graph=False)
        X.append(engine.d_mlp_feat.clone())
        T.append(engine.d_mlp_targ.clone())
        its.append(int(engine.d_stats[0].item()))
    engine.set_mlp(mode=0)
    for a, (n, m) in zip(engine.ibm_args, saved):
        a.mdf_iterations, a.mdf_min_iterations = n, m
    return torch.cat(X), torch.cat(T), its
