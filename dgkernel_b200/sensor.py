"""Learned shock sensor: the network's parameters, its training with the library's CUDA kernels, and the
collection of training pairs from viscosity-stage runs.

The network maps an element's unit-norm modal coefficients (Np values) to the Persson-Peraire activation in
[0, 1]: Np -> 32 -> 32 -> 1 with tanh, tanh, sigmoid.  Training minimises the mean squared difference to the
PP activation with Adam; forward, gradient and Adam steps are the library's kernels (dgk_mlp_*), and torch
supplies only the device buffers and the stream.  The stage evaluates the network with FP16 weights and FP32
sums and falls back to the PP activation where the output lies in a low-confidence band.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from ._lib import check, lib
from .burgers import RK4A, RK4B, mlp_param_count
from . import mesh as M

HIDDEN = 32


def init_params(nin: int, seed: int = 7) -> np.ndarray:
    """Glorot-uniform weights (splitmix64 stream), zero biases; float32 in the library's layout."""
    P = mlp_param_count(nin)
    u = M.splitmix_uniform(seed, P)
    p = np.zeros(P, dtype=np.float64)
    o = 0
    for fan_in, fan_out in ((nin, HIDDEN), (HIDDEN, HIDDEN), (HIDDEN, 1)):
        lim = math.sqrt(6.0 / (fan_in + fan_out))
        n = fan_in * fan_out
        p[o:o + n] = (2.0 * u[o:o + n] - 1.0) * lim
        o += n + fan_out  # weights, then zero biases
    return p.astype(np.float32)


class SensorNet:
    """Parameters and Adam state on the GPU (torch float32 buffers), trained by the library's kernels."""

    def __init__(self, nin: int, params=None, seed: int = 7):
        import torch
        self.torch = torch
        self.nin = nin
        self.P = mlp_param_count(nin)
        p = init_params(nin, seed) if params is None else np.asarray(params, dtype=np.float32)
        dev = torch.device("cuda")
        self.p = torch.tensor(p, device=dev)
        self.m = torch.zeros_like(self.p)
        self.v = torch.zeros_like(self.p)
        self.g = torch.zeros_like(self.p)
        self.loss = torch.zeros(1, device=dev)
        self.half = torch.zeros(self.P + 8, dtype=torch.int16, device=dev)
        self.t = 0

    def _stream(self):
        return C.c_void_p(self.torch.cuda.current_stream().cuda_stream)

    @staticmethod
    def _ptr(t):
        return C.c_void_p(t.data_ptr())

    def forward(self, X, fp16: bool = False):
        X = X.contiguous()
        out = self.torch.empty(X.shape[0], device=X.device, dtype=self.torch.float32)
        check(lib().dgk_mlp_forward(self._ptr(self.p), self._ptr(X), X.shape[0], self.nin, int(fp16), self._ptr(out),
                                    self._ptr(self.half), self._stream()))
        return out

    def loss_grad(self, X, y):
        X, y = X.contiguous(), y.contiguous()
        check(lib().dgk_mlp_loss_grad(self._ptr(self.p), self._ptr(X), self._ptr(y), X.shape[0], self.nin,
                                      self._ptr(self.g), self._ptr(self.loss), self._stream()))
        return float(self.loss.item()), self.g

    def step(self, X, y, lr: float = 3e-3):
        loss, _ = self.loss_grad(X, y)
        self.t += 1
        check(lib().dgk_mlp_adam(self._ptr(self.p), self._ptr(self.g), self._ptr(self.m), self._ptr(self.v), self.P,
                                 lr, 0.9, 0.999, 1e-8, self.t, self._stream()))
        return loss

    def fit(self, X, y, epochs: int = 20, batch: int = 8192, lr: float = 3e-3, seed: int = 11):
        """Mini-batch Adam over (X, y) (torch CUDA tensors); returns the mean loss of every epoch."""
        torch = self.torch
        gen = torch.Generator(device=X.device)
        gen.manual_seed(seed)
        hist = []
        n = X.shape[0]
        for ep in range(epochs):
            perm = torch.randperm(n, device=X.device, generator=gen)
            tot, cnt = 0.0, 0
            for s in range(0, n, batch):
                idx = perm[s:s + batch]
                tot += self.step(X[idx], y[idx], lr * (0.5 * (1 + math.cos(math.pi * ep / epochs)) + 0.02))
                cnt += 1
            hist.append(tot / max(cnt, 1))
        return hist

    def numpy(self) -> np.ndarray:
        return self.p.detach().cpu().numpy().astype(np.float32)


def collect_pairs(problem, t_end: float, every: int = 20, max_pairs: int = 0, sensor: str = "pp", rng_seed: int = 3):
    """Run a viscosity-stage problem with the PP sensor to t_end and take (modal features, PP activation) of
    every element every `every` steps.  Returns (X [n, Np] float32, y [n] float32)."""
    X, Y = [], []
    nsteps = int(math.ceil(t_end / problem.dt))
    for s in range(nsteps):
        if s % every == 0:
            f, sig, _ = problem.sensor_features("pp")
            X.append(f)
            Y.append(sig)
        problem.run_stages(5)
    f, sig, _ = problem.sensor_features("pp")
    X.append(f)
    Y.append(sig)
    X, Y = np.concatenate(X), np.concatenate(Y)
    ok = np.isfinite(Y) & np.all(np.isfinite(X), axis=1)  # a run that left the stable range contributes nothing
    X, Y = X[ok], Y[ok]
    if max_pairs and len(Y) > max_pairs:
        pick = np.random.default_rng(rng_seed).choice(len(Y), max_pairs, replace=False)
        X, Y = X[pick], Y[pick]
    return X, Y


def balance(X, y, active_frac: float = 0.5, seed: int = 5):
    """Resample so that about `active_frac` of the pairs have a non-zero activation (shocks are rare)."""
    rng = np.random.default_rng(seed)
    act = np.nonzero(y > 0)[0]
    idle = np.nonzero(y <= 0)[0]
    if len(act) == 0 or len(idle) == 0:
        return X, y
    n_idle = int(len(act) * (1 - active_frac) / active_frac)
    keep = np.concatenate([act, rng.choice(idle, min(n_idle, len(idle)), replace=False)])
    rng.shuffle(keep)
    return X[keep], y[keep]
