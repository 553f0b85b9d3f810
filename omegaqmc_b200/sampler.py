"""Walker ensemble driven by the single-electron sweep kernels.

``WalkerEnsemble`` owns the device buffers of one sampling run (positions,
inverse Slater matrices, per-sweep reductions) and advances them in chunks
of ``refresh_every`` sweeps, each chunk one persistent kernel launch
followed by a full FP64 LU refresh of the inverses.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib as L
from .context import GTOContext

__all__ = ["WalkerEnsemble", "init_walkers_gaussian", "init_walkers_ball",
           "NSUM", "PREC"]

NSUM = 8
PREC = {"fp64": L.PREC_FP64, "mixed": L.PREC_MIXED}


def init_walkers_gaussian(system, W, sigma, seed):
    """Electrons assigned to nuclei by charge, N(nucleus, sigma) per electron
    (the seeded initial state of the benchmark configurations)."""
    rng = np.random.default_rng(seed)
    idx = np.repeat(np.arange(system.natm), system.Z.astype(int))[: system.n_e]
    return system.nuc[idx][None] + sigma * rng.standard_normal((W, system.n_e, 3))


def init_walkers_ball(system, W, seed):
    """``_initialize_walkers`` (OmegaQMC/vmc_gto.py:64-118): electrons on
    nuclei by charge, scattered uniformly in a ball of radius 0.4 x the
    shortest bond (molecules) or as N(0, (0.5 sqrt(n_e))^2) (atoms)."""
    rng = np.random.default_rng(seed)
    idx = np.repeat(np.arange(system.natm), system.Z.astype(int))
    n_e = system.n_e
    if len(idx) < n_e:
        idx = np.concatenate([idx, np.zeros(n_e - len(idx), dtype=int)])
    idx = idx[:n_e]
    centers = system.nuc[idx]
    if system.natm > 1:
        i, j = np.triu_indices(system.natm, k=1)
        sep = 0.4 * np.min(np.linalg.norm(system.nuc[i] - system.nuc[j], axis=-1))
        d = rng.standard_normal((W, n_e, 3))
        d /= np.linalg.norm(d, axis=-1, keepdims=True)
        rad = sep * rng.random((W, n_e, 1)) ** (1.0 / 3.0)
        off = d * rad
    else:
        off = 0.5 * np.sqrt(float(n_e)) * rng.standard_normal((W, n_e, 3))
    return centers[None] + off


class WalkerEnsemble:
    """Device state of W walkers of one system.

    Args:
        ctx: the system's :class:`GTOContext`.
        walkers: (W, n_e, 3) initial positions (host or device).
        precision: ``"fp64"`` or ``"mixed"``.
        seed: 64-bit key of the Philox stream.
        refresh_every: sweeps between full FP64 LU refreshes (default 50).
        walkers_per_block: CTA size of the sweep kernel (0 = library default).
    """

    def __init__(self, ctx: GTOContext, walkers, precision="fp64", seed=0,
                 refresh_every=50, walkers_per_block=0):
        if precision not in PREC:
            raise ValueError(f"precision must be one of {list(PREC)}")
        self.ctx = ctx
        self.precision = precision
        self.prec = PREC[precision]
        self.X = ctx.walkers_tensor(walkers).clone()
        self.W = self.X.shape[0]
        self.state = ctx.new_state(self.W, self.prec)
        self.seed = int(seed)
        self.step_count = 0
        self.refresh_every = int(refresh_every)
        self.since_refresh = 0
        self.wpb = int(walkers_per_block)
        self.refresh()

    def refresh(self, stream=None):
        self.ctx.refresh(self.X, self.state, self.prec, stream=stream)
        self.since_refresh = 0

    def run(self, n_sweeps, step, measure_every=1, sums=None, el_trace=None,
            eparts_last=None, stream=None):
        """Advance n_sweeps sweeps; returns the (n_meas, 8) sums tensor.

        Chunks end at the refresh cadence, so a refresh happens after every
        ``refresh_every`` sweeps counted across calls."""
        n_meas = n_sweeps // measure_every
        if sums is None:
            sums = torch.zeros(max(n_meas, 1), NSUM, dtype=torch.float64,
                               device=self.X.device)
        done = 0
        meas_done = 0
        while done < n_sweeps:
            chunk = min(n_sweeps - done, self.refresh_every - self.since_refresh)
            if measure_every > 1:
                chunk = max(measure_every, chunk - chunk % measure_every)
                chunk = min(chunk, n_sweeps - done)
            m = chunk // measure_every
            tr = el_trace[meas_done:meas_done + m] if el_trace is not None else None
            self.ctx.sweeps(self.X, self.state, self.prec, chunk, step, self.seed,
                            self.step_count, sums[meas_done:], measure_every=measure_every,
                            el_trace=tr, eparts_last=eparts_last,
                            walkers_per_block=self.wpb, stream=stream)
            done += chunk
            meas_done += m
            self.step_count += chunk
            self.since_refresh += chunk
            if self.since_refresh >= self.refresh_every:
                self.refresh(stream=stream)
        return sums

    def equilibrate(self, n_steps, step, target=0.4, rate=0.05, stream=None):
        """Equilibration with the reference's per-step width adaptation
        (``vmc_gto.py:121-126, 1338-1357``) done on the device: n_steps
        sweeps, no host round trip between them.  Returns (final width,
        per-sweep acceptance ratios, per-sweep widths) as a float and two
        CUDA tensors."""
        dev = self.X.device
        s = torch.tensor([float(step)], dtype=torch.float64, device=dev)
        acc = torch.empty(max(int(n_steps), 1), dtype=torch.float64, device=dev)
        trace = torch.empty_like(acc)
        self.ctx.equilibrate(self.X, self.state, self.prec, n_steps, s, target, rate, self.seed,
                             self.step_count, self.refresh_every, self.since_refresh, acc,
                             trace, stream=stream)
        self.step_count += int(n_steps)
        self.since_refresh = (self.since_refresh + int(n_steps)) % self.refresh_every
        return float(s.item()), acc[:n_steps], trace[:n_steps]

    def basin(self, n_steps, sigma=1.5, stream=None):
        """Basin relocation moves (``vmc_gto.py:925-957``); returns the mean
        acceptance."""
        acc = torch.zeros(1, dtype=torch.float64, device=self.X.device)
        self.ctx.basin(self.X, self.state, self.prec, n_steps, sigma, self.seed ^ 0xBA5E,
                       self.step_count, acc_sum=acc, stream=stream)
        self.step_count += n_steps
        self.refresh(stream=stream)
        return float(acc.item()) / max(1, n_steps * self.W)

    def state_evaluate(self, stream=None):
        """Per-walker log|psi|, gradient, Laplacian and local-energy parts as
        the sampler sees them (tracked inverses, this ensemble's precision)."""
        return self.ctx.state_evaluate(self.state, self.W, self.prec, stream=stream)

    def logdet(self):
        off = self.state.numel() - ((self.W * 8 + 255) // 256) * 256
        return self.state[off:off + self.W * 8].view(torch.float64)
