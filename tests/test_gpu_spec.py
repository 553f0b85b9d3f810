"""Run-time specialised kernels (oqmc_specialize) against the oracle."""
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


@pytest.mark.parametrize("name,cusp", [("H2", False), ("LiH", False), ("H2O", False),
                                       ("H2O", True), ("N2", False), ("H2O_dimer", False)])
def test_specialised_sweeps_track_fresh_evaluation(name, cusp):
    mf = M.make_mf(name)
    pc = M.synthetic_cusp_params(mf.mol) if cusp else None
    s = build_system(mf, M.default_params_corr(mf.mol, cusp=cusp), pc)
    ctx = GTOContext(s)
    ctx.specialize()
    W = 512
    ens = WalkerEnsemble(ctx, seeded_walkers(s, W, 0.8, 3), "fp64", seed=11,
                         refresh_every=10**9)
    ep = torch.empty(W, 4, dtype=torch.float64, device="cuda")
    ens.run(30, 0.4, eparts_last=ep)
    torch.cuda.synchronize()
    Xf = ens.X.cpu().numpy()
    ref = O.evaluate(s, Xf)
    ld = ens.logdet().cpu().numpy()
    ld_ref = O.log_slater(s, Xf)
    assert np.max(np.abs(ld - ld_ref) / (np.abs(ld_ref) + 1)) < 1e-8
    el = ep[:, 3].cpu().numpy()
    sc = 0.5 * (np.sum(np.abs(ref["lap"]), axis=1) + np.sum(ref["grad"] ** 2, axis=(1, 2))) + 1
    assert np.max(np.abs(el - ref["e_loc"]) / (np.abs(ref["e_loc"]) + sc)) < 1e-10
    assert ctx.flags() == 0


@pytest.mark.parametrize("name", ["H2O", "N2"])
def test_specialised_mixed_precision_error(name):
    mf = M.make_mf(name)
    s = build_system(mf, M.benchmark_params_corr(mf.mol))
    ctx = GTOContext(s)
    ctx.specialize()
    W = 4096
    ens = WalkerEnsemble(ctx, seeded_walkers(s, W, 1.0, 5), "mixed", seed=3)
    ep = torch.empty(W, 4, dtype=torch.float64, device="cuda")
    ens.run(20, 0.3, eparts_last=ep)
    torch.cuda.synchronize()
    ref = O.evaluate(s, ens.X.cpu().numpy())
    err = np.abs(ep[:, 3].cpu().numpy() - ref["e_loc"])
    assert np.median(err) < 1e-4, np.median(err)
    assert np.quantile(err, 0.99) < 5e-3, np.quantile(err, 0.99)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_specialised_kernels_with_f_and_g_shells(precision):
    """The generated straight-line code for f and g shells (the golden case
    the reference computed: s to g functions on three centres): sweeps of the
    specialised kernels keep the Sherman-Morrison state and E_L consistent
    with a fresh oracle evaluation (FP64 at the parity tolerances, mixed
    within the mixed-precision bounds)."""
    from helpers import golden_system
    s, _ = golden_system("fg_shells")
    ctx = GTOContext(s)
    ctx.specialize()
    W = 1024
    ens = WalkerEnsemble(ctx, seeded_walkers(s, W, 0.8, 9), precision, seed=13,
                         refresh_every=10**9)
    ep = torch.empty(W, 4, dtype=torch.float64, device="cuda")
    ens.run(30, 0.3, eparts_last=ep)
    torch.cuda.synchronize()
    Xf = ens.X.cpu().numpy()
    ref = O.evaluate(s, Xf)
    el = ep[:, 3].cpu().numpy()
    if precision == "fp64":
        ld = ens.logdet().cpu().numpy()
        ld_ref = O.log_slater(s, Xf)
        assert np.max(np.abs(ld - ld_ref) / (np.abs(ld_ref) + 1)) < 1e-8
        sc = 0.5 * (np.sum(np.abs(ref["lap"]), axis=1) + np.sum(ref["grad"] ** 2, axis=(1, 2))) + 1
        assert np.max(np.abs(el - ref["e_loc"]) / (np.abs(ref["e_loc"]) + sc)) < 1e-10
    else:
        err = np.abs(el - ref["e_loc"])
        assert np.median(err) < 1e-4, np.median(err)
        assert np.quantile(err, 0.99) < 5e-3, np.quantile(err, 0.99)
    assert ctx.flags() == 0
