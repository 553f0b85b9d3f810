"""Tensor-core (tcgen05) local energy against the oracle and the CUDA-core
kernel, mixed build."""
import numpy as np
import pytest
import torch

from helpers import seeded_walkers
from oracle import gto_oracle as O
from omegaqmc_b200 import molecules as M
from omegaqmc_b200.context import GTOContext
from omegaqmc_b200.sampler import WalkerEnsemble
from omegaqmc_b200.system import build_system

pytestmark = pytest.mark.gpu


def _eloc_after(ctx, s, X, tc, n=3):
    ctx.use_tensor_cores(tc)
    ens = WalkerEnsemble(ctx, X, "mixed", seed=17)
    ep = torch.empty(X.shape[0], 4, dtype=torch.float64, device="cuda")
    sums = ens.run(n, 0.3, eparts_last=ep)
    torch.cuda.synchronize()
    return ens.X.cpu().numpy(), ep.cpu().numpy(), sums.cpu().numpy()


@pytest.mark.parametrize("name,W", [("H2O", 256), ("H2", 512), ("LiH", 1000), ("N2", 700),
                                    ("H2O_dimer", 300)])
def test_tensor_core_local_energy(name, W):
    mf = M.make_mf(name)
    s = build_system(mf, M.benchmark_params_corr(mf.mol))
    ctx = GTOContext(s)
    X = seeded_walkers(s, W, 0.9, 2)
    Xa, epa, sa = _eloc_after(ctx, s, X, True)
    Xb, epb, sb = _eloc_after(ctx, s, X, False)
    assert ctx.flags() == 0
    # identical moves (same kernel, seed), so positions agree exactly
    assert np.array_equal(Xa, Xb)
    ref = O.evaluate(s, Xa)
    err_tc = np.abs(epa[:, 3] - ref["e_loc"])
    err_cc = np.abs(epb[:, 3] - ref["e_loc"])
    assert np.median(err_tc) < 1e-4, np.median(err_tc)
    assert np.quantile(err_tc, 0.99) < 5e-3, np.quantile(err_tc, 0.99)
    assert np.median(err_tc) < 10 * np.median(err_cc) + 1e-6
    np.testing.assert_allclose(epa[:, 0], ref["e_ee"], rtol=1e-12)
    np.testing.assert_allclose(epa[:, 1], ref["e_en"], rtol=1e-12)
    assert sa[-1, 6] == W
