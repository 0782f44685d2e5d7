"""Learned control variate for ensemble averages (no counterpart in the reference).

An observable f of a trajectory depends on the Wiener increments that drive it.
A small network g(x) fitted to f from coarse projections x of those increments
gives the unbiased two-level estimator

    E[f] ~ mean_N(f - g(x)) + mean_M(g(x')),   x' fresh samples of x, M >> N,

whose sampling error is set by Var(f - g) instead of Var(f).  The projections
computed by xs_noise_features are independent N(0, 1) variables, so the M
fresh inputs are drawn directly from N(0, 1) without integrating anything.
The network (xs_mlp_*) is trained on pairs the solver itself produces, with
the project's forward, backward and Adam kernels (BF16 operands, FP32
accumulation); xSPDE's block-mean sampling error (Simulator/xsim.m:95)
judges both estimators.
"""
import ctypes
import math

import numpy as np

from . import _lib


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


class ControlVariateNet:
    """MLP in -> hidden x3 -> 1 with GELU, trained on (features, observable)."""

    def __init__(self, n_in=256, hidden=256, seed=0, device="cuda"):
        import torch
        self.n_in, self.hidden, self.device = n_in, hidden, device
        npar = ctypes.c_size_t()
        _lib.lib().xs_mlp_sizes(n_in, hidden, 1, ctypes.byref(npar))
        self.nparams = npar.value
        g = torch.Generator().manual_seed(seed)
        parts = []
        for rows, cols in ((hidden, n_in), (hidden, hidden), (hidden, hidden)):
            parts.append(torch.randn(rows * cols, generator=g, dtype=torch.float64) * math.sqrt(2.0 / cols))
            parts.append(torch.zeros(rows, dtype=torch.float64))
        parts.append(torch.randn(hidden, generator=g, dtype=torch.float64) * math.sqrt(1.0 / hidden))
        parts.append(torch.zeros(1, dtype=torch.float64))
        self.params = torch.cat(parts).float().to(device)
        assert self.params.numel() == self.nparams
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.grad = torch.zeros_like(self.params)
        self.step = 0
        self.mean = 0.0
        self.scale = 1.0
        self._work = {}

    def _workspace(self, B):
        import torch
        if B not in self._work:
            n = _lib.lib().xs_mlp_sizes(self.n_in, self.hidden, B, None)
            self._work = {B: torch.empty(n, dtype=torch.float32, device=self.device)}
        return self._work[B]

    def fit(self, X, f, epochs=30, batch=1024, lr=1e-3, seed=0, stream=None, weight_decay=0.0):
        """Fit g to (f - mean)/scale on device tensors X [n, n_in] (FP32), f [n]."""
        import torch
        L = _lib.lib()
        f = f.double()
        self.mean = float(f.mean())
        self.scale = float(f.std()) or 1.0
        t = ((f - self.mean) / self.scale).float().contiguous()
        n = X.shape[0]
        gen = torch.Generator(device=self.device).manual_seed(seed)
        work = self._workspace(batch)
        loss = torch.zeros(1, dtype=torch.float64, device=self.device)
        st = ctypes.c_void_p(stream.cuda_stream if stream is not None else torch.cuda.current_stream().cuda_stream)
        hist = []
        for _ in range(epochs):
            perm = torch.randperm(n, device=self.device, generator=gen)
            tot = 0.0
            for b0 in range(0, n - batch + 1, batch):
                idx = perm[b0:b0 + batch]
                xb = X.index_select(0, idx).contiguous()
                tb = t.index_select(0, idx).contiguous()
                _lib.check(L.xs_mlp_train_grad(batch, self.n_in, self.hidden, _ptr(xb), _ptr(self.params),
                                               _ptr(work), _ptr(tb), _ptr(self.grad), _ptr(loss), st))
                self.step += 1
                _lib.check(L.xs_mlp_adam(self.nparams, _ptr(self.params), _ptr(self.grad), _ptr(self.m),
                                         _ptr(self.v), lr, 0.9, 0.999, 1e-8, self.step, weight_decay, st))
                tot += float(loss.item()) if b0 == 0 else 0.0
            hist.append(tot)
        return hist

    def predict(self, X, batch=65536, stream=None):
        """g(X) in the units of f (device tensor, FP64)."""
        import torch
        L = _lib.lib()
        n = X.shape[0]
        out = torch.empty(n, dtype=torch.float32, device=self.device)
        st = ctypes.c_void_p(stream.cuda_stream if stream is not None else torch.cuda.current_stream().cuda_stream)
        for b0 in range(0, n, batch):
            B = min(batch, n - b0)
            xb = X[b0:b0 + B].contiguous()
            work = self._workspace(B)
            yb = out[b0:b0 + B]
            _lib.check(L.xs_mlp_forward(B, self.n_in, self.hidden, _ptr(xb), _ptr(self.params), _ptr(work),
                                        _ptr(yb), st))
        return out.double() * self.scale + self.mean


def block_sampling_error(values, nblocks):
    """xSPDE's sampling error of the mean from block means (Simulator/xsim.m:95):
    sqrt((<D^2> - <D>^2) / (nblocks - 1)) with D the block means."""
    v = np.asarray(values, dtype=np.float64)
    n = (v.size // nblocks) * nblocks
    D = v[:n].reshape(nblocks, -1).mean(axis=1)
    return float(np.mean(D)), float(np.sqrt(max(np.mean(D ** 2) - np.mean(D) ** 2, 0.0) / (nblocks - 1)))


def two_level(f, g_x, g_fresh, nblocks):
    """Two-level estimate mean(f - g(x)) + mean(g(x')) and its sampling error
    (block estimate of the first term combined with the error of the second).
    g_fresh is the array g(x') or its moments (mean, standard deviation, count)."""
    d = np.asarray(f, dtype=np.float64) - np.asarray(g_x, dtype=np.float64)
    m1, e1 = block_sampling_error(d, nblocks)
    if isinstance(g_fresh, tuple):
        m2, sd, n = g_fresh
        e2 = sd / math.sqrt(n)
    else:
        gf = np.asarray(g_fresh, dtype=np.float64)
        m2 = float(gf.mean())
        e2 = float(gf.std(ddof=1) / math.sqrt(gf.size))
    return m1 + m2, math.sqrt(e1 ** 2 + e2 ** 2)


def fresh_moments(g_fresh):
    """(mean, standard deviation, count) of a device tensor g(x'), reduced on the device."""
    gd = g_fresh.double()
    return float(gd.mean()), float(gd.std()), int(gd.numel())
