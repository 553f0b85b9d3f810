"""J3_eeI three-body Jastrow on the GPU: sampling agrees with the oracle's
reference-algorithm sampler, Sherman-Morrison-tracked sweeps (FP64 and
mixed) match a fresh oracle evaluation, the batched path matches the
per-system path, and the tensor-core local energy refuses it.  (Parameter
derivatives with J3 terms are checked in test_gpu_optim.py.)  (The FP64
evaluation itself is checked against the reference's golden vectors,
cases h2o_j3 and lih_j3, in test_gpu_eval.py.)"""
import numpy as np
import pytest
import torch

from helpers import seeded_walkers
from oracle import gto_oracle as O
from oracle import vmc_oracle as V
from omegaqmc_b200 import molecules as M
from omegaqmc_b200.batch import BatchedSampler
from omegaqmc_b200.context import GTOContext
from omegaqmc_b200.sampler import WalkerEnsemble
from omegaqmc_b200.system import build_system

pytestmark = pytest.mark.gpu


def _j3(syms, npar, scale, seed, skip=()):
    rng = np.random.default_rng(seed)
    return {p + s: rng.normal(size=npar) * scale for s in syms for p in ("like+", "unlike+")
            if p + s not in skip}


H2_PARAMS = {"J2_pade": {"like": np.array([0.25, 1.0]), "unlike": np.array([0.5, 1.0])},
             "J3_eeI": _j3(["H"], 26, 0.002, 3)}
H2O_PARAMS = {"J2_pade": {"like": np.array([0.25, 1.0]), "unlike": np.array([0.5, 1.0])},
              "J1_pade": {"O": np.array(1.2), "H": np.array(0.5)},
              "J3_eeI": _j3(["O", "H"], 8, 0.004, 5, skip=("like+H",))}
H2O_CFG = {"J3": {"N_eI": 2, "N_ee": 2, "r_cut": 4.0}}


def _h2():
    return build_system(M.make_mf("H2"), H2_PARAMS)


def _h2o():
    return build_system(M.make_mf("H2O"), H2O_PARAMS, None, H2O_CFG)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_j3_sampling_agrees_with_oracle_sampler(precision):
    s = _h2()
    ctx = GTOContext(s)
    ens = WalkerEnsemble(ctx, seeded_walkers(s, 2048, 0.5, 0), precision, seed=5)
    ens.run(300, 0.6)
    sums = ens.run(3000, 0.6).cpu().numpy()
    m_gpu, se_gpu, _, _ = O.binning_analysis(sums[:, 3] / sums[:, 6])
    ser, _, _, _ = V.run_vmc(s, seeded_walkers(s, 512, 0.5, 1), 300, 3000, seed=2)
    m_ref, se_ref, _, _ = O.binning_analysis(ser)
    assert abs(m_gpu - m_ref) < 3.0 * np.hypot(se_gpu, se_ref), (m_gpu, se_gpu, m_ref, se_ref)
    assert ctx.flags() == 0


def test_j3_sweeps_track_fresh_evaluation():
    s = _h2o()
    ctx = GTOContext(s)
    ctx.specialize()
    W = 512
    ens = WalkerEnsemble(ctx, seeded_walkers(s, W, 1.0, 3), "fp64", seed=11, refresh_every=10**9)
    ep = torch.empty(W, 4, dtype=torch.float64, device="cuda")
    ens.run(30, 0.4, eparts_last=ep)
    torch.cuda.synchronize()
    Xf = ens.X.cpu().numpy()
    ref = O.evaluate(s, Xf)
    ld = ens.logdet().cpu().numpy()
    ld_ref = O.log_slater(s, Xf)
    assert np.max(np.abs(ld - ld_ref) / (np.abs(ld_ref) + 1)) < 1e-8
    sc = 0.5 * (np.sum(np.abs(ref["lap"]), axis=1) + np.sum(ref["grad"] ** 2, axis=(1, 2))) + 1
    assert np.max(np.abs(ep[:, 3].cpu().numpy() - ref["e_loc"]) / (np.abs(ref["e_loc"]) + sc)) < 1e-10
    # the FP64 evaluation entry point on the same walkers
    ev = ctx.evaluate(torch.as_tensor(Xf, device="cuda"))
    np.testing.assert_allclose(ev["logpsi"].cpu().numpy(), ref["logpsi"], rtol=1e-10, atol=1e-10)
    # mixed precision against the same oracle values
    ens_m = WalkerEnsemble(ctx, Xf, "mixed", seed=12)
    ens_m.run(1, 1e-9, eparts_last=ep)
    torch.cuda.synchronize()
    ref_m = O.evaluate(s, ens_m.X.cpu().numpy())
    err = np.abs(ep[:, 3].cpu().numpy() - ref_m["e_loc"])
    assert np.median(err) < 1e-4 and np.quantile(err, 0.99) < 5e-3, (np.median(err), np.quantile(err, 0.99))
    assert ctx.flags() == 0


def test_j3_sampling_with_like_spin_pairs_agrees_with_oracle_sampler():
    """LiH has same-spin pairs, so both J3 blocks enter the move ratio."""
    s = build_system(M.make_mf("LiH"),
                     {"J2_pade": {"like": np.array([0.25, 1.0]), "unlike": np.array([0.5, 1.0])},
                      "J3_eeI": _j3(["Li", "H"], 8, 0.003, 8)}, None,
                     {"J3": {"N_eI": 2, "N_ee": 2, "r_cut": 5.0}})
    ctx = GTOContext(s)
    ens = WalkerEnsemble(ctx, seeded_walkers(s, 4096, 1.0, 0), "fp64", seed=6)
    ens.run(300, 0.5)
    sums = ens.run(2000, 0.5).cpu().numpy()
    m_gpu, se_gpu, _, _ = O.binning_analysis(sums[:, 3] / sums[:, 6])
    ser, _, _, _ = V.run_vmc(s, seeded_walkers(s, 512, 1.0, 1), 100, 800, seed=2)
    m_ref, se_ref, _, _ = O.binning_analysis(ser)
    assert abs(m_gpu - m_ref) < 3.0 * np.hypot(se_gpu, se_ref), (m_gpu, se_gpu, m_ref, se_ref)
    assert ctx.flags() == 0


def test_j3_batch_reproduces_per_system_path():
    s = _h2o()
    ctx = GTOContext(s)
    ctx.specialize()
    W = 300
    X0 = torch.as_tensor(seeded_walkers(s, W, 1.0, 7), device="cuda")
    b = BatchedSampler([ctx], [X0.clone()], [0.5], precision="fp64", proposal="plain", cap=8)
    b.configure(64, [64], variant=0)
    b.reset(40)
    b.run(10, 5, 77)
    torch.cuda.synchronize()
    X = X0.clone()
    st = ctx.new_state(W, 0)
    sums = torch.zeros(2, 8, dtype=torch.float64, device="cuda")
    ctx.refresh(X, st, 0)
    ctx.sweeps(X, st, 0, 10, 0.5, 77, 40, sums, measure_every=5)
    torch.cuda.synchronize()
    same = torch.all((b.walkers[0] == X).reshape(W, -1), dim=1)
    assert float(same.float().mean()) > 0.99
    np.testing.assert_allclose(b.sums[0][:2, 6].cpu().numpy(), sums[:, 6].cpu().numpy())
    assert b.flags() == 0


def test_j3_tensor_core_local_energy_is_refused():
    ctx = GTOContext(_h2())
    with pytest.raises(NotImplementedError):
        ctx.use_tensor_cores(True)
