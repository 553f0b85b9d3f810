"""Batched sampling of several molecules in one persistent launch.

:class:`BatchedSampler` drives the library's batch entry points
(``oqmc_batch_*``): one generated kernel holds every molecule's basis code,
each launch refreshes the Slater inverses in FP64 and runs ``n_sweeps``
single-electron sweeps with local-energy measurements for all molecules,
and consecutive launches can be captured in a CUDA graph.  The tile shape
(threads per CTA, walkers per tile of each molecule, register budget) is
chosen by the library's autotuner or set by hand.

For each molecule a launch reproduces ``GTOContext.refresh`` followed by
``GTOContext.sweeps`` with the same seed and sweep counter (the reference's
production step, ``OmegaQMC/vmc_gto.py:985-1034``, as single-electron
sweeps); the reference itself samples one molecule per driver call.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib as L
from .context import _stream_ptr
from .sampler import NSUM

__all__ = ["BatchedSampler", "PREC"]

PREC = {"fp64": L.PREC_FP64, "mixed": L.PREC_MIXED}
PROPOSALS = {"plain": 0, "fixed": 0, "scaled": 1}


class BatchedSampler:
    """Walkers of several :class:`GTOContext` molecules sampled together.

    ``walkers[k]`` is a (W_k, n_e_k, 3) float64 CUDA tensor, updated in
    place.  ``steps[k]`` is the Gaussian width (the scale of the
    nucleus-scaled proposal when ``proposal="scaled"``).  ``cap`` is the
    number of measurement slots kept per molecule (8 doubles each, the
    ``oqmc_sweeps`` layout: ee, en, ke, E_L, E_L^2, accepted moves, finite
    walkers)."""

    def __init__(self, contexts, walkers, steps, precision="mixed", proposal="scaled",
                 scale_r0=1.0, scale_fmin=0.05, cap=1024):
        if not (len(contexts) == len(walkers) == len(steps)) or not contexts:
            raise ValueError("contexts, walkers and steps must have the same non-zero length")
        if precision not in PREC:
            raise ValueError(f"precision must be one of {sorted(PREC)}")
        props = proposal if isinstance(proposal, (list, tuple)) else [proposal] * len(contexts)
        self.lib = L.load()
        self.contexts = list(contexts)
        self.device = contexts[0].device
        self.precision = PREC[precision]
        self.walkers = [c.walkers_tensor(X) for c, X in zip(contexts, walkers)]
        for X, c in zip(self.walkers, contexts):
            if X.shape[1:] != (c.n_e, 3):
                raise ValueError("walkers must be (W, n_e, 3) for their molecule")
        self.n = len(contexts)
        self.cap = int(cap)
        self.sums = [torch.zeros((max(self.cap, 1), NSUM), dtype=torch.float64,
                                 device=self.device) for _ in contexts]
        arr = (ctypes.c_void_p * self.n)(*[c._h.value for c in contexts])
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            code = self.lib.oqmc_batch_create(ctypes.byref(h), arr, self.n, self.precision)
        L.check(code, None, batch=True)
        self._h = h
        self._entries = (L.BatchSystem * self.n)()
        for k in range(self.n):
            e = self._entries[k]
            e.walkers = self.walkers[k].data_ptr()
            e.W = int(self.walkers[k].shape[0])
            e.proposal = PROPOSALS[props[k]]
            e.step = float(steps[k])
            e.scale_r0 = float(scale_r0)
            e.scale_fmin = float(scale_fmin)
            e.sums = self.sums[k].data_ptr()
            e.cap = self.cap
        self._check(self.lib.oqmc_batch_bind(self._h, self._entries))

    def set_proposal(self, k, step=None, proposal=None, scale_r0=None, scale_fmin=None):
        """Change molecule k's proposal settings (re-plans the tiles; a
        captured graph must be captured again)."""
        e = self._entries[k]
        if step is not None:
            e.step = float(step)
        if proposal is not None:
            e.proposal = PROPOSALS[proposal]
        if scale_r0 is not None:
            e.scale_r0 = float(scale_r0)
        if scale_fmin is not None:
            e.scale_fmin = float(scale_fmin)
        cfg = self.config() if getattr(self, "_h", None) is not None else None
        self._check(self.lib.oqmc_batch_bind(self._h, self._entries))
        if cfg is not None:
            self.configure(cfg["threads"], cfg["walkers_per_tile"], cfg["variant"])

    def steps(self):
        return [self._entries[k].step for k in range(self.n)]

    def adapt_steps(self, target=0.4, rounds=40, sweeps=5, seed=0x5EED, step_base=3 * 10**9):
        """Equilibrate with the reference's step rule, log s += 0.05 (acc -
        target) (OmegaQMC/vmc_gto.py:121-126), applied to every molecule
        once per round of ``sweeps`` sweeps (five times the rate, once per
        round); leaves the measurement slots cleared."""
        self.reset(step_base)
        for r in range(rounds):
            for sm in self.sums:
                sm[0].zero_()
            self.reset(step_base + r * sweeps, clear_sums=False)
            self.run(sweeps, sweeps, seed)
            for k in range(self.n):
                W = self.walkers[k].shape[0]
                acc = float(self.sums[k][0, 5]) / (sweeps * W * self.contexts[k].n_e)
                e = self._entries[k]
                e.step = float(np.exp(np.log(e.step) + 0.05 * sweeps * (acc - target)))
            cfg = self.config()
            self._check(self.lib.oqmc_batch_bind(self._h, self._entries))
            self.configure(cfg["threads"], cfg["walkers_per_tile"], cfg["variant"])
        self.reset(0)
        return self.steps()

    # -- lifetime --------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self.lib.oqmc_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, code):
        L.check(code, self._h, batch=True)

    # -- tile shape ------------------------------------------------------
    def configure(self, threads, walkers_per_tile, variant=0):
        wpt = (ctypes.c_int * self.n)(*[int(x) for x in walkers_per_tile])
        self._check(self.lib.oqmc_batch_configure(self._h, int(threads), wpt, int(variant)))

    def config(self):
        t, v, g, r, lb = (ctypes.c_int() for _ in range(5))
        wpt = (ctypes.c_int * self.n)()
        sm = ctypes.c_size_t()
        self._check(self.lib.oqmc_batch_get_config(self._h, ctypes.byref(t), wpt, ctypes.byref(v),
                                                   ctypes.byref(g), ctypes.byref(sm),
                                                   ctypes.byref(r), ctypes.byref(lb)))
        return {"threads": t.value, "walkers_per_tile": list(wpt), "variant": v.value,
                "grid": g.value, "smem": sm.value, "registers": r.value,
                "local_bytes": lb.value}

    def tune(self, n_sweeps=4, seed=0x7E57, stream=None):
        """Autotune the tile shape (moves the walkers); returns (config, ms)."""
        ms = ctypes.c_float()
        with torch.cuda.device(self.device):
            self._check(self.lib.oqmc_batch_tune(self._h, int(n_sweeps), int(seed),
                                                 _stream_ptr(stream), ctypes.byref(ms)))
        return self.config(), ms.value

    # -- sampling --------------------------------------------------------
    def reset(self, step_base=0, clear_sums=True, stream=None):
        """Next launch starts at sweep ``step_base`` and measurement slot 0."""
        if clear_sums:
            for s in self.sums:
                s.zero_()
        self._check(self.lib.oqmc_batch_reset(self._h, int(step_base), _stream_ptr(stream)))

    def run(self, n_sweeps, measure_every=1, seed=0, stream=None):
        """One persistent launch: FP64 refresh + ``n_sweeps`` sweeps."""
        self._check(self.lib.oqmc_batch_run(self._h, int(n_sweeps), int(measure_every), int(seed),
                                            _stream_ptr(stream)))

    def capture(self, n_launches, n_sweeps, measure_every=1, seed=0):
        """Record ``n_launches`` consecutive launches as one CUDA graph."""
        with torch.cuda.device(self.device):
            self._check(self.lib.oqmc_batch_capture(self._h, int(n_launches), int(n_sweeps),
                                                    int(measure_every), int(seed)))

    def replay(self, stream=None):
        self._check(self.lib.oqmc_batch_replay(self._h, _stream_ptr(stream)))

    def busy_ns(self, stream=None):
        """Per-molecule sum of tile durations (ns) since the last reset."""
        out = (ctypes.c_ulonglong * self.n)()
        self._check(self.lib.oqmc_batch_busy(self._h, out, _stream_ptr(stream)))
        return list(out)

    def flags(self, clear=True, stream=None):
        f = ctypes.c_uint()
        self._check(self.lib.oqmc_batch_get_flags(self._h, ctypes.byref(f), int(clear),
                                                  _stream_ptr(stream)))
        return f.value

    def energies(self, k, n_meas):
        """(walker-mean E_L per measurement, accepted moves, finite walkers)
        of molecule k over the first ``n_meas`` measurement slots."""
        s = self.sums[k][:n_meas].cpu().numpy()
        nw = s[:, 6]
        return s[:, 3] / nw, s[:, 5], nw
