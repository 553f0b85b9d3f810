"""The allocation-free sampling entry point, through the C ABI.

``oqmc_sweeps_noalloc`` is for callers that cannot allocate device memory
(their GPU memory belongs to another allocator's arena, or a cudaMalloc would
synchronise the device on their path): it keeps the walker state in a
library-owned device array.  It must give the same walkers, reductions and
local energies as the allocating path (``oqmc_refresh`` + ``oqmc_sweeps``
with a caller buffer) on the same inputs, call after call.  This file is
collected last so that a run stopping at the first failure has run every
other test first.  The last test repeats the calls in a fresh process and
checks that the device's free memory does not move across them.
"""
import ctypes
import json
import os
import subprocess
import sys

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


# Run in a fresh process: nothing else has raised the device's stack limit
# or loaded the library's kernels yet.  Every buffer is allocated before
# the measured calls; free device memory is read around each of them.
_FRESH = r"""
import ctypes, json, sys
import numpy as np
import torch
sys.path[:0] = [sys.argv[1], sys.argv[2]]
from helpers import golden_system, seeded_walkers
from omegaqmc_b200 import _lib as L
from omegaqmc_b200 import molecules as M
from omegaqmc_b200.context import GTOContext
from omegaqmc_b200.system import build_system

lib = L.load()
st = lambda: ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
p = lambda t: ctypes.c_void_p(t.data_ptr() if t is not None else 0)
out = {}


def call(h, X, W, sums, prec):
    torch.cuda.synchronize()
    before = torch.cuda.mem_get_info()[0]
    rc = lib.oqmc_sweeps_noalloc(h, p(X), W, prec, 4, 1, 0.4, ctypes.c_uint64(3),
                                 ctypes.c_uint64(0), p(sums), None, None, st())
    torch.cuda.synchronize()
    return rc, before - torch.cuda.mem_get_info()[0], lib.oqmc_last_error(h).decode()


# single determinant (H2O, mixed): a small first call loads the kernels,
# then a full call must leave free memory unchanged
mf = M.make_mf("H2O")
s = build_system(mf, M.benchmark_params_corr(mf.mol))
ctx = GTOContext(s)
W = 4096
X = torch.tensor(seeded_walkers(s, W, 0.9, 2), dtype=torch.float64, device="cuda")
sums = torch.zeros(4, 8, dtype=torch.float64, device="cuda")
out["warm"] = call(ctx._h, X, 64, sums, L.PREC_MIXED)[0]
out["single"] = call(ctx._h, X, W, sums, L.PREC_MIXED)

# multi-determinant (H2O, FP64): its kernels need more local memory per
# thread than the default stack reservation
s2, _ = golden_system("h2o_md")
ctx2 = GTOContext(s2)
W2 = 512
X2 = torch.tensor(seeded_walkers(s2, W2, 0.9, 4), dtype=torch.float64, device="cuda")
out["md_first"] = call(ctx2._h, X2, W2, sums, L.PREC_FP64)
out["md_again"] = call(ctx2._h, X2, W2, sums, L.PREC_FP64)
# an allocating call raises the stack limit; the entry point then accepts
state = torch.empty(lib.oqmc_state_bytes(ctx2._h, W2, L.PREC_FP64), dtype=torch.uint8,
                    device="cuda")
Xa = X2.clone()
assert lib.oqmc_refresh(ctx2._h, p(Xa), W2, p(state), L.PREC_FP64, st()) == 0
assert lib.oqmc_sweeps(ctx2._h, p(Xa), W2, p(state), L.PREC_FP64, 4, 1, 0.4,
                       ctypes.c_uint64(3), ctypes.c_uint64(0), p(sums), None, None, 0,
                       st()) == 0
out["md_after"] = call(ctx2._h, X2, W2, sums, L.PREC_FP64)
torch.cuda.synchronize()
out["md_match"] = bool(torch.allclose(Xa, X2, rtol=1e-12, atol=0))
print("RESULT " + json.dumps(out))
"""


def test_noalloc_leaves_free_memory_unchanged_in_fresh_process():
    here = os.path.dirname(os.path.abspath(__file__))
    env = dict(os.environ)
    env.pop("CUDA_MODULE_LOADING", None)
    r = subprocess.run([sys.executable, "-c", _FRESH, here, os.path.dirname(here)],
                       capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-3000:]
    line = [x for x in r.stdout.splitlines() if x.startswith("RESULT ")][-1]
    out = json.loads(line[len("RESULT "):])
    assert out["warm"] == 0
    rc, used, err = out["single"]
    assert rc == 0 and used == 0, out["single"]
    # the first multi-determinant call may load its kernels (lazy loading)
    # before it refuses; the repeated call must neither allocate nor launch
    rc1, _, err1 = out["md_first"]
    rc2, used2, _ = out["md_again"]
    assert rc1 == rc2 == L.OQ_ERR_UNSUPPORTED, out
    assert "local memory" in err1
    assert used2 == 0, out["md_again"]
    rc3, used3, err3 = out["md_after"]
    assert rc3 == 0 and used3 == 0, out["md_after"]
    assert out["md_match"]
