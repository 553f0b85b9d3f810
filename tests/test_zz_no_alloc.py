"""The allocation-free sampling entry point, through the C ABI.

``oqmc_sweeps_noalloc`` is for callers that cannot allocate device memory
(their GPU memory belongs to another allocator's arena, or a cudaMalloc would
synchronise the device on their path): it keeps the walker state in a
library-owned device array.  It must give the same walkers, reductions and
local energies as the allocating path (``oqmc_refresh`` + ``oqmc_sweeps``
with a caller buffer) on the same inputs, call after call.  This file is
collected last so that a run stopping at the first failure has run every
other test first.
"""
import ctypes

import numpy as np
import pytest
import torch

from helpers import seeded_walkers
from omegaqmc_b200 import _lib as L
from omegaqmc_b200 import molecules as M
from omegaqmc_b200.context import GTOContext
from omegaqmc_b200.system import build_system

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _p(t):
    return ctypes.c_void_p(t.data_ptr() if t is not None else 0)


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


@pytest.mark.parametrize("prec", [L.PREC_FP64, L.PREC_MIXED])
def test_noalloc_matches_allocating_path_twice(prec):
    lib = L.load()
    mf = M.make_mf("H2O")
    s = build_system(mf, M.benchmark_params_corr(mf.mol))
    ctx = GTOContext(s)
    h = ctx._h
    W, n, step, seed = 2048, 12, 0.5, 1234
    X0 = torch.tensor(seeded_walkers(s, W, 0.9, 7), dtype=torch.float64, device="cuda")
    Xa = X0.clone()
    Xb = X0.clone()
    state = torch.empty(lib.oqmc_state_bytes(h, W, prec), dtype=torch.uint8, device="cuda")
    for call in range(2):
        base = call * n
        sa = torch.zeros(n, 8, dtype=torch.float64, device="cuda")
        sb = torch.zeros(n, 8, dtype=torch.float64, device="cuda")
        ea = torch.empty(W, 4, dtype=torch.float64, device="cuda")
        eb = torch.empty(W, 4, dtype=torch.float64, device="cuda")
        rc = lib.oqmc_refresh(h, _p(Xa), W, _p(state), prec, _stream())
        assert rc == 0
        rc = lib.oqmc_sweeps(h, _p(Xa), W, _p(state), prec, n, 1, step,
                             ctypes.c_uint64(seed), ctypes.c_uint64(base), _p(sa), None,
                             _p(ea), 0, _stream())
        assert rc == 0
        rc = lib.oqmc_sweeps_noalloc(h, _p(Xb), W, prec, n, 1, step, ctypes.c_uint64(seed),
                                     ctypes.c_uint64(base), _p(sb), None, _p(eb), _stream())
        assert rc == 0, lib.oqmc_last_error(h)
        torch.cuda.synchronize()
        assert torch.allclose(Xa, Xb, rtol=TOL, atol=0), call
        assert torch.allclose(sa, sb, rtol=TOL, atol=TOL), call
        assert torch.allclose(ea, eb, rtol=TOL, atol=TOL), call
        assert not torch.equal(Xa, X0)
        assert float(sb[:, 6].min()) == W
    assert ctx.flags() == 0


def test_noalloc_rejects_oversized_batches():
    lib = L.load()
    mf = M.make_mf("H2O")
    s = build_system(mf, M.benchmark_params_corr(mf.mol))
    ctx = GTOContext(s)
    h = ctx._h
    W = 1
    while lib.oqmc_state_bytes(h, W, L.PREC_FP64) <= (16 << 20):
        W *= 2
    X = torch.zeros(W, s.n_e, 3, dtype=torch.float64, device="cuda")
    sums = torch.zeros(1, 8, dtype=torch.float64, device="cuda")
    rc = lib.oqmc_sweeps_noalloc(h, _p(X), W, L.PREC_FP64, 1, 1, 0.3, ctypes.c_uint64(1),
                                 ctypes.c_uint64(0), _p(sums), None, None, _stream())
    assert rc == L.OQ_ERR_ARG
    assert b"16 MiB" in lib.oqmc_last_error(h)
