"""Multi-determinant trials on the GPU (oqmc_set_multidet): sampling agrees
with the oracle's reference-algorithm sampler, Sherman-Morrison-tracked
sweeps match a fresh oracle evaluation, a one-term expansion follows the
single-determinant kernels, basin relocations run, and the paths built for
single determinants refuse it.  (The FP64 evaluation is checked against the
reference's golden vectors, cases h2o_md and lih_md_uhf, in
test_gpu_eval.py.)"""
import numpy as np
import pytest
import torch

from helpers import golden_system, seeded_walkers
from oracle import gto_oracle as O
from oracle import vmc_oracle as V
from omegaqmc_b200 import molecules as M
from omegaqmc_b200.batch import BatchedSampler
from omegaqmc_b200.context import GTOContext
from omegaqmc_b200.sampler import WalkerEnsemble
from omegaqmc_b200.system import build_system

pytestmark = pytest.mark.gpu

J2 = {"J2_pade": {"like": np.array([0.25, 1.0]), "unlike": np.array([0.5, 1.0])}}


def _h2_two_determinants():
    """H2 in a minimal basis with c_g |g g| + c_u |u u| (bonding and
    antibonding orbitals)."""
    mo = np.array([[0.55, 1.2], [0.55, -1.2]])
    trial = {"mo_coeff": mo, "ci_coeffs": np.array([0.97, -0.24]),
             "occ_up": np.array([[0], [1]]), "occ_dn": np.array([[0], [1]])}
    return build_system(M.make_mf("H2"), J2, None, None, trial)


def test_md_sampling_agrees_with_oracle_sampler():
    s = _h2_two_determinants()
    ctx = GTOContext(s)
    assert ctx.multidet_info() == (2, 2, 2, 8)
    ens = WalkerEnsemble(ctx, seeded_walkers(s, 2048, 0.5, 0), "fp64", seed=5)
    ens.run(300, 0.6)
    sums = ens.run(3000, 0.6).cpu().numpy()
    m_gpu, se_gpu, _, _ = O.binning_analysis(sums[:, 3] / sums[:, 6])
    ser, _, _, _ = V.run_vmc(s, seeded_walkers(s, 512, 0.5, 1), 300, 3000, seed=2)
    m_ref, se_ref, _, _ = O.binning_analysis(ser)
    assert abs(m_gpu - m_ref) < 3.0 * np.hypot(se_gpu, se_ref), (m_gpu, se_gpu, m_ref, se_ref)
    assert ctx.flags() == 0


@pytest.mark.parametrize("name", ["h2o_md", "lih_md_uhf"])
def test_md_sweeps_track_fresh_evaluation(name):
    s, _ = golden_system(name)
    ctx = GTOContext(s)
    W = 384
    ens = WalkerEnsemble(ctx, seeded_walkers(s, W, 0.9, 3), "fp64", seed=11, refresh_every=10**9)
    ep = torch.empty(W, 4, dtype=torch.float64, device="cuda")
    ens.run(30, 0.4, eparts_last=ep)
    torch.cuda.synchronize()
    Xf = ens.X.cpu().numpy()
    ref = O.evaluate(s, Xf)
    sc = 0.5 * (np.sum(np.abs(ref["lap"]), axis=1) + np.sum(ref["grad"] ** 2, axis=(1, 2))) + 1
    err = np.abs(ep[:, 3].cpu().numpy() - ref["e_loc"]) / (np.abs(ref["e_loc"]) + sc)
    assert np.max(err) < 1e-9, np.max(err)
    ev = ctx.evaluate(torch.as_tensor(Xf, device="cuda"))
    np.testing.assert_allclose(ev["logpsi"].cpu().numpy(), ref["logpsi"], rtol=1e-10, atol=1e-10)
    np.testing.assert_allclose(ev["e_loc"].cpu().numpy(), ref["e_loc"], rtol=1e-9,
                               atol=1e-9 * float(np.max(sc)))
    assert ctx.flags() == 0


def test_md_one_term_follows_single_determinant_kernels():
    mf = M.make_mf("H2O")
    C = np.asarray(mf.mo_coeff)[:, :5]
    trial = {"mo_coeff": C, "ci_coeffs": np.array([1.0]), "occ_up": np.array([[0, 1, 2, 3, 4]]),
             "occ_dn": np.array([[0, 1, 2, 3, 4]])}
    s1 = build_system(mf, J2)
    sm = build_system(mf, J2, None, None, trial)
    X0 = seeded_walkers(s1, 256, 1.0, 4)
    out = []
    for s in (s1, sm):
        ctx = GTOContext(s)
        ens = WalkerEnsemble(ctx, X0, "fp64", seed=7)
        sums = ens.run(20, 0.4).cpu().numpy()
        torch.cuda.synchronize()
        out.append((ens.X.cpu().numpy(), sums))
    same = np.all(np.abs(out[0][0] - out[1][0]).reshape(256, -1) < 1e-12, axis=1)
    assert same.mean() > 0.99
    np.testing.assert_allclose(out[1][1][:, 5], out[0][1][:, 5], rtol=2e-2)   # acceptances


def test_md_basin_relocations_run():
    s = _h2_two_determinants()
    ctx = GTOContext(s)
    W = 512
    X = torch.as_tensor(seeded_walkers(s, W, 0.5, 8), device="cuda")
    st = ctx.new_state(W, 0)
    ctx.refresh(X, st, 0)
    acc = torch.zeros(1, dtype=torch.float64, device="cuda")
    ctx.basin(X, st, 0, 50, 1.5, 3, 0, acc_sum=acc)
    torch.cuda.synchronize()
    assert 0.0 < float(acc) < 50 * W and torch.all(torch.isfinite(X))
    assert ctx.flags() == 0


def test_md_paths_without_support_refuse_it():
    s = _h2_two_determinants()
    ctx = GTOContext(s)
    X = seeded_walkers(s, 64, 0.5, 0)
    with pytest.raises(NotImplementedError):
        WalkerEnsemble(ctx, X, "mixed", seed=1).run(1, 0.5)
    with pytest.raises(NotImplementedError):
        ctx.use_tensor_cores(True)
    with pytest.raises(NotImplementedError):
        BatchedSampler([ctx], [torch.as_tensor(X, device="cuda")], [0.5], cap=1)
    ctx.set_multidet(None)
    assert ctx.multidet_info() == (0, 0, 0, 0)


def test_md_optimiser_inputs_match_oracle():
    """Jastrow-parameter derivatives with a multi-determinant trial (the
    linear-method inputs, vmcopt_gto_linear.py:686-703, which accepts
    trials): the Slater part enters only through the gradient of ln|psi|."""
    from omegaqmc_b200.optim import raw_to_flat, walker_derivatives
    s, d = golden_system("h2o_md")
    spec = __import__("json").loads(str(d["spec"]))
    pc = {k: {kk: np.asarray(vv, dtype=np.float64) for kk, vv in v.items()}
          for k, v in spec["params_corr"].items()}
    ctx = GTOContext(s)
    X = seeded_walkers(s, 130, 0.8, 21)
    e, dl, de = walker_derivatives(ctx, X, pc)
    rl, re_ = O.param_derivatives(s, X)
    ref_dl, ref_de = raw_to_flat(rl, pc, s), raw_to_flat(re_, pc, s)
    assert np.max(np.abs(dl - ref_dl) / (np.abs(ref_dl).max(axis=0) + 1.0)) < 1e-10
    assert np.max(np.abs(de - ref_de) / (np.abs(ref_de).max(axis=0) + 1.0)) < 1e-9
    ref_e = O.evaluate(s, X)["e_loc"]
    assert np.max(np.abs(e - ref_e)) / (0.5 * np.abs(ref_e).max() + 1.0) < 1e-9


def test_md_state_evaluate_matches_oracle():
    """oqmc_state_eval on a multi-determinant sampler state: log|psi| (tracked
    determinant sum + Jastrow), gradient, Laplacian and E_L as the oracle
    evaluates them at the same positions, fresh and after 20 sweeps of
    per-determinant Sherman-Morrison updates."""
    s, _ = golden_system("h2o_md")
    ctx = GTOContext(s)
    W = 256
    ens = WalkerEnsemble(ctx, seeded_walkers(s, W, 0.9, 5), "fp64", seed=3, refresh_every=10**9)
    for sweeps, tol in ((0, 1e-10), (20, 1e-8)):
        if sweeps:
            ens.run(sweeps, 0.4)
        out = {k: v.cpu().numpy() for k, v in ens.state_evaluate().items()}
        ref = O.evaluate(s, ens.X.cpu().numpy())
        sc = 0.5 * (np.sum(np.abs(ref["lap"]), axis=1) + np.sum(ref["grad"] ** 2, axis=(1, 2))) + 1
        assert np.max(np.abs(out["logpsi"] - ref["logpsi"]) / (np.abs(ref["logpsi"]) + 1)) < tol
        assert np.max(np.abs(out["grad"] - ref["grad"]) / (np.abs(ref["grad"]) + 1)) < tol
        assert np.max(np.abs(out["e_loc"] - ref["e_loc"]) / sc) < tol
    assert ctx.flags() == 0
