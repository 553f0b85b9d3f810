"""Learned Metropolis proposal: a small BF16 MLP trained on the plain sampler.

The reference proposes every move with a fixed-width Gaussian random walk
(``metropolis_move_alle``, OmegaQMC/vmc_gto.py:815-839).  Here a per-electron
network maps the electron's surroundings (position relative to the two
nearest nuclei, displacements to its 8 nearest electrons, spin) to an
8-component Gaussian mixture over its displacement.  Sampling stays exact:
each move is accepted with |psi(x')/psi(x)|^2 q(x|x') / q(x'|x), both mixture
densities evaluated by the same network (Metropolis-Hastings, as the
reference's basin move, vmc_gto.py:925-957).

Training data are the plain sampler's own trajectories: for walker
configurations x(t) and x(t+k) that the fixed-width sampler produced k
sweeps apart, each electron gives one row (features of x(t), displacement
x_e(t+k) - x_e(t)); the network maximises the mixture likelihood of those
displacements (a mixture-density fit of the k-sweep transition).  Forward,
backward and the Adam update run in the library's own kernels (tcgen05
tensor cores, BF16 operands, FP32 accumulation); this module only moves
buffers.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import _lib as L
from .context import GTOContext, _dptr, _stream_ptr
from .sampler import WalkerEnsemble

__all__ = ["MLPProposal", "collect_training_set", "train_proposal"]

K0, NOUT = 32, 48


class MLPProposal:
    """The network and its optimiser state on one device."""

    def __init__(self, seed=0, device=None):
        self.lib = L.load()
        self.device = torch.device("cuda", torch.cuda.current_device()
                                   if device is None else torch.device(device).index)
        self.n_params = int(self.lib.oqmc_mlp_num_params())
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            code = self.lib.oqmc_mlp_create(ctypes.byref(h), int(seed))
        L.check(code, None, mlp=True)
        self._h = h
        self._loss = torch.zeros(1, dtype=torch.float64, device=self.device)

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self.lib.oqmc_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, code):
        L.check(code, self._h, mlp=True)

    # -- parameters -----------------------------------------------------------
    def params(self):
        out = np.empty(self.n_params, dtype=np.float32)
        self._check(self.lib.oqmc_mlp_get_params(
            self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return out

    def set_params(self, theta):
        th = np.ascontiguousarray(theta, dtype=np.float32)
        if th.size != self.n_params:
            raise ValueError(f"expected {self.n_params} parameters")
        self._check(self.lib.oqmc_mlp_set_params(
            self._h, th.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))

    # -- kernels --------------------------------------------------------------
    def forward(self, feat, stream=None):
        """Outputs (R, 48) float32 of BF16 feature rows ``feat`` (R, 32)
        stored as int16 bit patterns."""
        R = feat.shape[0]
        out = torch.empty(R, NOUT, dtype=torch.float32, device=self.device)
        self._check(self.lib.oqmc_mlp_forward(self._h, _dptr(feat), R, _dptr(out),
                                              _stream_ptr(stream)))
        return out

    def backward(self, feat, target, stream=None):
        """(gradient of the mean NLL as a float32 CUDA tensor, mean NLL)."""
        R = feat.shape[0]
        g = torch.empty(self.n_params, dtype=torch.float32, device=self.device)
        self._check(self.lib.oqmc_mlp_backward(self._h, _dptr(feat), _dptr(target), R, _dptr(g),
                                               _dptr(self._loss), _stream_ptr(stream)))
        return g, float(self._loss.item()) / R

    def step(self, feat, target, lr, stream=None, loss=True):
        """One Adam step; returns the mean NLL of the batch (before the step)
        when ``loss`` is true (a device read), else None."""
        R = feat.shape[0]
        self._check(self.lib.oqmc_mlp_step(self._h, _dptr(feat), _dptr(target), R, float(lr),
                                           _dptr(self._loss), _stream_ptr(stream)))
        return float(self._loss.item()) / R if loss else None

    def flags(self, clear=True, stream=None):
        f = ctypes.c_uint()
        self._check(self.lib.oqmc_mlp_get_flags(self._h, ctypes.byref(f), int(clear),
                                                _stream_ptr(stream)))
        return f.value


def features(ctx: GTOContext, X0, X1=None, stream=None):
    """BF16 feature rows (W*n_e, 32) of walkers X0 and, with X1, the float32
    displacement targets X1 - X0 (row = walker * n_e + electron)."""
    X0 = ctx.walkers_tensor(X0)
    W = X0.shape[0]
    R = W * ctx.n_e
    feat = torch.empty(R, K0, dtype=torch.int16, device=ctx.device)
    tgt = None
    if X1 is not None:
        X1 = ctx.walkers_tensor(X1)
        tgt = torch.empty(R, 3, dtype=torch.float32, device=ctx.device)
    ctx._check(ctx.lib.oqmc_mlp_features(ctx._h, _dptr(X0), _dptr(X1), W, _dptr(feat),
                                         _dptr(tgt), _stream_ptr(stream)))
    return feat, tgt


def collect_training_set(ens: WalkerEnsemble, n_configs, k, step, drop_static=True):
    """Run the plain (fixed-width Gaussian) sampler ``ens`` and return the
    rows of ``n_configs`` walker configurations: features of x(t) and the
    displacement to x(t+k), k sweeps later.  Rows of electrons that did not
    move in those k sweeps are dropped when ``drop_static`` (a zero
    displacement carries no information about where moves should go)."""
    ctx = ens.ctx
    feats, tgts = [], []
    got = 0
    while got < n_configs:
        X0 = ens.X.clone()
        ens.run(k, step)
        f, t = features(ctx, X0, ens.X)
        if drop_static:
            keep = torch.any(t != 0, dim=1)
            f, t = f[keep], t[keep]
        feats.append(f)
        tgts.append(t)
        got += ens.W
    return torch.cat(feats), torch.cat(tgts)


def train_proposal(mlp: MLPProposal, feat, target, steps=2000, batch=8192, lr=2e-3,
                   lr_end=1e-4, seed=0, log_every=0):
    """Adam on random batches with a cosine learning-rate decay; returns the
    list of (step, mean NLL) recorded every ``log_every`` steps."""
    g = torch.Generator(device=feat.device)
    g.manual_seed(int(seed))
    R = feat.shape[0]
    hist = []
    for i in range(steps):
        idx = torch.randint(0, R, (batch,), generator=g, device=feat.device)
        f = feat.index_select(0, idx).contiguous()
        t = target.index_select(0, idx).contiguous()
        a = lr_end + 0.5 * (lr - lr_end) * (1.0 + math.cos(math.pi * i / max(1, steps - 1)))
        want = bool(log_every) and (i % log_every == 0 or i == steps - 1)
        loss = mlp.step(f, t, a, loss=want)
        if want:
            hist.append((i, loss))
    return hist
