"""GPU sampler: Sherman-Morrison consistency, mixed-precision error bounds
and statistical agreement with the oracle's reference-algorithm sampler."""
import numpy as np
import pytest
import torch

from helpers import seeded_walkers
from oracle import gto_oracle as O
from oracle import vmc_oracle as V
from omegaqmc_b200 import molecules as M
from omegaqmc_b200.context import GTOContext
from omegaqmc_b200.sampler import WalkerEnsemble
from omegaqmc_b200.system import build_system

pytestmark = pytest.mark.gpu


def _sys(name, cusp=False):
    mf = M.make_mf(name)
    pc = M.synthetic_cusp_params(mf.mol) if cusp else None
    return build_system(mf, M.default_params_corr(mf.mol, cusp=cusp), pc)


@pytest.mark.parametrize("name,cusp", [("H2", False), ("LiH", False), ("H2O", False),
                                       ("H2O", True), ("N2", False)])
def test_sherman_morrison_tracks_fresh_evaluation(name, cusp):
    s = _sys(name, cusp)
    ctx = GTOContext(s)
    W = 512
    ens = WalkerEnsemble(ctx, seeded_walkers(s, W, 0.8, 3), "fp64", seed=11,
                         refresh_every=10**9)
    ep = torch.empty(W, 4, dtype=torch.float64, device="cuda")
    sums = ens.run(40, 0.4, eparts_last=ep)
    torch.cuda.synchronize()
    Xf = ens.X.cpu().numpy()
    # positions moved and stayed finite
    assert np.isfinite(Xf).all()
    ref = O.evaluate(s, Xf)
    ld_ref = O.log_slater(s, Xf)
    ld = ens.logdet().cpu().numpy()
    assert np.max(np.abs(ld - ld_ref) / (np.abs(ld_ref) + 1)) < 1e-8
    el = ep[:, 3].cpu().numpy()
    assert np.max(np.abs(el - ref["e_loc"]) / (np.abs(ref["e_loc"]) + 1)) < 1e-8
    s_np = sums.cpu().numpy()
    # reductions agree with the per-walker last measurement
    assert abs(s_np[-1, 3] - el.sum()) < 1e-8 * (1 + abs(el.sum()))
    assert s_np[-1, 6] == W
    acc = s_np[:, 5].sum() / (40 * W * s.n_e)
    assert 0.05 < acc < 0.98
    assert ctx.flags() == 0


@pytest.mark.parametrize("name", ["LiH", "H2O", "N2"])
def test_mixed_precision_local_energy_error(name):
    s = _sys(name)
    ctx = GTOContext(s)
    W = 4096
    ens = WalkerEnsemble(ctx, seeded_walkers(s, W, 1.0, 5), "mixed", seed=3,
                         refresh_every=50)
    ep = torch.empty(W, 4, dtype=torch.float64, device="cuda")
    ens.run(20, 0.3, eparts_last=ep)
    ens.refresh()
    torch.cuda.synchronize()
    Xf = ens.X.cpu().numpy()
    ref = O.evaluate(s, Xf)
    err = np.abs(ep[:, 3].cpu().numpy() - ref["e_loc"])
    # stated mixed-precision tolerance on the local energy (hartree)
    assert np.median(err) < 1e-4, np.median(err)
    assert np.quantile(err, 0.99) < 5e-3, np.quantile(err, 0.99)
    ld = ens.logdet().cpu().numpy()
    assert np.max(np.abs(ld - O.log_slater(s, Xf))) < 1e-8


def test_energy_agrees_with_oracle_sampler_h2():
    s = _sys("H2")
    ctx = GTOContext(s)
    ens = WalkerEnsemble(ctx, seeded_walkers(s, 2048, 0.5, 0), "fp64", seed=5)
    ens.run(300, 0.6)
    sums = ens.run(3000, 0.6).cpu().numpy()
    series = sums[:, 3] / sums[:, 6]
    m_gpu, se_gpu, _, _ = O.binning_analysis(series)
    X0 = seeded_walkers(s, 512, 0.5, 1)
    ser, _, _, _ = V.run_vmc(s, X0, 300, 3000, seed=2)
    m_ref, se_ref, _, _ = O.binning_analysis(ser)
    z = abs(m_gpu - m_ref) / np.hypot(se_gpu, se_ref)
    assert z < 3.0, (m_gpu, se_gpu, m_ref, se_ref)


def test_mixed_and_fp64_energies_agree_h2o():
    s = _sys("H2O")
    ctx = GTOContext(s)
    means = {}
    for prec in ("fp64", "mixed"):
        ens = WalkerEnsemble(ctx, seeded_walkers(s, 8192, 1.0, 0), prec, seed=9)
        ens.run(200, 0.25)
        sums = ens.run(600, 0.25).cpu().numpy()
        ser = sums[:, 3] / sums[:, 6]
        means[prec] = O.binning_analysis(ser)
    z = abs(means["fp64"][0] - means["mixed"][0]) / np.hypot(means["fp64"][1],
                                                              means["mixed"][1])
    assert z < 3.0, means


def test_sampler_rejects_bad_arguments():
    s = _sys("H2")
    ctx = GTOContext(s)
    ens = WalkerEnsemble(ctx, seeded_walkers(s, 8, 0.5, 0), "fp64")
    with pytest.raises(ValueError):
        ens.run(4, -1.0)
    with pytest.raises(ValueError):
        WalkerEnsemble(ctx, seeded_walkers(s, 8, 0.5, 0), "fp16")


def test_basin_moves_keep_state_consistent():
    s = _sys("H2O")
    ctx = GTOContext(s)
    W = 512
    ens = WalkerEnsemble(ctx, seeded_walkers(s, W, 0.8, 3), "fp64", seed=5,
                         refresh_every=10**9)
    acc = torch.zeros(1, dtype=torch.float64, device="cuda")
    ctx.basin(ens.X, ens.state, ens.prec, 50, 1.5, 99, 0, acc_sum=acc)
    torch.cuda.synchronize()
    Xf = ens.X.cpu().numpy()
    ld = ens.logdet().cpu().numpy()
    ld_ref = O.log_slater(s, Xf)
    assert np.max(np.abs(ld - ld_ref) / (np.abs(ld_ref) + 1)) < 1e-8
    rate = float(acc.item()) / (50 * W)
    assert 0.0005 < rate < 0.95, rate


def test_basin_moves_sample_psi_squared_h2():
    """Basin relocations alone are an exact MH chain for |psi|^2: the mean
    local energy matches the oracle's reference-algorithm sampler."""
    s = _sys("H2")
    ctx = GTOContext(s)
    ens = WalkerEnsemble(ctx, seeded_walkers(s, 4096, 0.5, 2), "fp64", seed=8,
                         refresh_every=10**9)
    ctx.basin(ens.X, ens.state, ens.prec, 200, 1.5, 17, 0)
    series = []
    for k in range(300):
        ctx.basin(ens.X, ens.state, ens.prec, 4, 1.5, 17, 1000 + 4 * k)
        series.append(float(ctx.evaluate(ens.X, want_grad=False, want_lap=False)["e_loc"].mean()))
    m_b, se_b, _, _ = O.binning_analysis(np.array(series))
    X0 = seeded_walkers(s, 512, 0.5, 1)
    ser, _, _, _ = V.run_vmc(s, X0, 300, 3000, seed=3)
    m_ref, se_ref, _, _ = O.binning_analysis(ser)
    z = abs(m_b - m_ref) / np.hypot(se_b, se_ref)
    assert z < 3.0, (m_b, se_b, m_ref, se_ref)


@pytest.mark.parametrize("name", ["LiH", "H2O"])
def test_scaled_proposal_preserves_distribution(name):
    """The nucleus-scaled proposal with its exact MH correction samples the
    same |psi|^2: energies agree with the fixed-width sampler."""
    mf = M.make_mf(name)
    s = build_system(mf, M.benchmark_params_corr(mf.mol))
    res = {}
    for kind in (0, 1):
        ctx = GTOContext(s)
        ctx.set_proposal(kind, 1.0, 0.05)
        ens = WalkerEnsemble(ctx, seeded_walkers(s, 16384, 0.8, 4), "fp64", seed=21 + kind)
        ens.run(1500, 0.5)
        sums = ens.run(1500, 0.5).cpu().numpy()
        res[kind] = O.binning_analysis(sums[:, 3] / sums[:, 6])
        assert ctx.flags() == 0
    z = abs(res[0][0] - res[1][0]) / np.hypot(res[0][1], res[1][1])
    assert z < 3.0, res
