"""Multi-GPU sampling as independent replicas (one process per GPU).

The reference shards its walker axis over a 1-D device mesh and lets XLA
reduce the block means (OmegaQMC/utils.py:1148-1159, vmc_gto.py:1331-1333).
Walkers never interact, so here every rank samples its own walker set with
its own random stream and the ranks only combine statistics: the
per-measurement sums (ee, en, ke, E_L, E_L^2, accepted moves, finite walkers)
are added over the ranks, which gives exactly the walker-mean series of the
union of all walkers.  Timing is the maximum over ranks.  These helpers work
with any ``torch.distributed`` backend (NCCL on GPUs, gloo on CPU).
"""
from __future__ import annotations

import numpy as np
import torch
import torch.distributed as dist

__all__ = ["world_info", "rank_seed", "combine_sums", "max_over_ranks", "walker_mean_series"]


def world_info():
    """(rank, world size) of the initialised process group, else (0, 1)."""
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(), dist.get_world_size()
    return 0, 1


def rank_seed(seed, rank=None):
    """Distinct 64-bit Philox key per rank (rank 0 keeps ``seed``)."""
    if rank is None:
        rank = world_info()[0]
    return (int(seed) + 0x9E3779B97F4A7C15 * int(rank)) & 0xFFFFFFFFFFFFFFFF


def combine_sums(sums):
    """Sum the (n_meas, 8) measurement sums over all ranks (in place for a
    tensor on the process group's device; a numpy array is copied).  Every
    rank must call it with the same shape."""
    rank, world = world_info()
    if isinstance(sums, np.ndarray):
        t = torch.as_tensor(sums, dtype=torch.float64).clone()
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.SUM)
        return t.numpy()
    if world > 1:
        dist.all_reduce(sums, op=dist.ReduceOp.SUM)
    return sums


def max_over_ranks(values, device=None):
    """Element-wise maximum over ranks of a list of floats (e.g. times)."""
    rank, world = world_info()
    t = torch.as_tensor(list(values), dtype=torch.float64,
                        device=device if device is not None else "cpu")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.cpu()]


def walker_mean_series(sums):
    """Walker-mean E_L per measurement from (n_meas, 8) sums (finite walkers
    only), the series the tau_int estimator and the block averages use."""
    s = np.asarray(sums, dtype=np.float64)
    return s[:, 3] / np.maximum(s[:, 6], 1.0)
