"""Replica combination across ranks (world size 2, gloo on CPU): the summed
measurement sums equal those of the union of both ranks' walkers, timing
is the maximum, seeds differ per rank."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from omegaqmc_b200 import replicas as R


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _fake_sums(rank, n_meas=50, W=100, seed=0):
    """Per-measurement sums of a rank's walkers from synthetic local energies."""
    rng = np.random.default_rng(seed + rank)
    el = -74.7 + 0.3 * rng.standard_normal((n_meas, W))
    s = np.zeros((n_meas, 8))
    s[:, 3] = el.sum(axis=1)
    s[:, 4] = (el ** 2).sum(axis=1)
    s[:, 5] = rng.integers(0, 10 * W, size=n_meas)
    s[:, 6] = W
    return s, el


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        s, _ = _fake_sums(rank)
        tot = R.combine_sums(s)
        t = R.max_over_ranks([1.0 + rank, 5.0 - rank])
        out[rank] = (tot, t, R.rank_seed(1234))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_rank_combination_matches_the_union_of_walkers():
    ctx = mp.get_context("spawn")
    man = ctx.Manager()
    out = man.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(90)
        assert p.exitcode == 0
    s0, e0 = _fake_sums(0)
    s1, e1 = _fake_sums(1)
    want = s0 + s1
    for r in range(2):
        tot, t, seed = out[r]
        np.testing.assert_allclose(tot, want, rtol=1e-15)
        assert t == [2.0, 5.0]
    assert out[0][2] == 1234 and out[1][2] != 1234
    # the combined walker-mean series is the mean over the union of walkers
    series = R.walker_mean_series(want)
    np.testing.assert_allclose(series, np.concatenate([e0, e1], axis=1).mean(axis=1), rtol=1e-13)


def test_single_process_is_identity():
    s, _ = _fake_sums(0)
    np.testing.assert_array_equal(R.combine_sums(s), s)
    assert R.max_over_ranks([3.0]) == [3.0]
    assert R.rank_seed(7, 0) == 7
