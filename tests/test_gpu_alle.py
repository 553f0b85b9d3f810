"""All-electron Metropolis steps on the GPU (oqmc_set_move_kind(ctx, 1), the
reference's metropolis_move_alle + metropolis_move_1w,
OmegaQMC/vmc_gto.py:815-905): the state after a run matches a fresh oracle
evaluation, the energy agrees with the oracle's all-electron sampler (the
same algorithm, vmc_oracle.run_vmc), and the paths built for
single-electron moves refuse it."""
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


@pytest.mark.parametrize("name,cusp,prec", [("LiH", False, "fp64"), ("H2O", True, "fp64"),
                                            ("H2O", False, "mixed")])
def test_alle_state_matches_fresh_evaluation(name, cusp, prec):
    s = _sys(name, cusp)
    ctx = GTOContext(s)
    ctx.set_move_kind(1)
    W = 1024
    X0 = seeded_walkers(s, W, 0.8, 3)
    ens = WalkerEnsemble(ctx, X0, prec, seed=11, refresh_every=10**9)
    ep = torch.empty(W, 4, dtype=torch.float64, device="cuda")
    sums = ens.run(40, 0.15, eparts_last=ep).cpu().numpy()
    torch.cuda.synchronize()
    Xf = ens.X.cpu().numpy()
    assert np.isfinite(Xf).all()
    # whole configurations move: an electron either stays with its walker's
    # previous configuration or every electron of that walker moved
    moved = np.any(Xf != X0, axis=2)
    assert np.all(moved.all(axis=1) | (~moved).all(axis=1))
    assert moved.all(axis=1).mean() > 0.5
    ld = ens.logdet().cpu().numpy()
    assert np.max(np.abs(ld - O.log_slater(s, Xf)) / (np.abs(ld) + 1)) < 1e-10
    ref = O.evaluate(s, Xf)
    el = ep[:, 3].cpu().numpy()
    err = np.abs(el - ref["e_loc"]) / (np.abs(ref["e_loc"]) + 1)
    if prec == "fp64":
        assert err.max() < 1e-8
    else:
        assert np.median(np.abs(el - ref["e_loc"])) < 1e-4
    # the accepted-move sum counts n_e electron moves per accepted step
    acc = sums[:, 5].sum() / (40 * W * s.n_e)
    assert 0.05 < acc < 0.95, acc
    assert np.all(np.fmod(sums[:, 5], s.n_e) == 0)
    assert ctx.flags() == 0


def test_alle_energy_agrees_with_oracle_sampler_h2():
    s = _sys("H2")
    ctx = GTOContext(s)
    ctx.set_move_kind(1)
    ens = WalkerEnsemble(ctx, seeded_walkers(s, 4096, 0.5, 0), "fp64", seed=5)
    ens.run(300, 0.5)
    sums = ens.run(3000, 0.5).cpu().numpy()
    m_gpu, se_gpu, _, _ = O.binning_analysis(sums[:, 3] / sums[:, 6])
    ser, acc_ref, _, _ = V.run_vmc(s, seeded_walkers(s, 512, 0.5, 1), 300, 3000, seed=2)
    m_ref, se_ref, _, _ = O.binning_analysis(ser)
    assert abs(m_gpu - m_ref) < 3.0 * np.hypot(se_gpu, se_ref), (m_gpu, se_gpu, m_ref, se_ref)


def test_alle_same_seed_is_deterministic():
    s = _sys("LiH")
    out = []
    for _ in range(2):
        ctx = GTOContext(s)
        ctx.set_move_kind(1)
        ens = WalkerEnsemble(ctx, seeded_walkers(s, 256, 0.8, 4), "fp64", seed=21)
        ens.run(30, 0.2)
        out.append(ens.X.cpu().numpy())
    assert np.array_equal(out[0], out[1])


def test_move_kind_arguments_and_refusals():
    s = _sys("H2")
    ctx = GTOContext(s)
    with pytest.raises(ValueError):
        ctx.set_move_kind(2)
    mo = np.array([[0.55, 1.2], [0.55, -1.2]])
    trial = {"mo_coeff": mo, "ci_coeffs": np.array([0.97, -0.24]),
             "occ_up": np.array([[0], [1]]), "occ_dn": np.array([[0], [1]])}
    J2 = {"J2_pade": {"like": np.array([0.25, 1.0]), "unlike": np.array([0.5, 1.0])}}
    md = GTOContext(build_system(M.make_mf("H2"), J2, None, None, trial))
    md.set_move_kind(1)
    ens = WalkerEnsemble(md, seeded_walkers(s, 64, 0.5, 0), "fp64", seed=1)
    with pytest.raises(NotImplementedError):
        ens.run(2, 0.5)


def test_noalloc_entry_runs_all_electron_steps_once_the_stack_allows():
    """The allocation-free entry point refuses a kernel only while its local
    memory exceeds the device's stack limit; after the allocating path has
    run the all-electron kernel (raising the limit where it needed more), the
    allocation-free call runs the same chain."""
    import ctypes
    from omegaqmc_b200 import _lib as L
    lib = L.load()
    s = _sys("H2O")
    ctx = GTOContext(s)
    ctx.set_move_kind(1)
    W = 64
    X0 = ctx.walkers_tensor(seeded_walkers(s, W, 0.9, 0))
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    p = lambda t: ctypes.c_void_p(t.data_ptr())
    Xa, Xb = X0.clone(), X0.clone()
    sa = torch.zeros(3, 8, dtype=torch.float64, device="cuda")
    sb = torch.zeros(3, 8, dtype=torch.float64, device="cuda")
    state = torch.empty(lib.oqmc_state_bytes(ctx._h, W, L.PREC_FP64), dtype=torch.uint8,
                        device="cuda")
    assert lib.oqmc_refresh(ctx._h, p(Xa), W, p(state), L.PREC_FP64, st) == 0
    assert lib.oqmc_sweeps(ctx._h, p(Xa), W, p(state), L.PREC_FP64, 3, 1, 0.2,
                           ctypes.c_uint64(1), ctypes.c_uint64(0), p(sa), None, None, 0, st) == 0
    rc = lib.oqmc_sweeps_noalloc(ctx._h, p(Xb), W, L.PREC_FP64, 3, 1, 0.2, ctypes.c_uint64(1),
                                 ctypes.c_uint64(0), p(sb), None, None, st)
    assert rc == 0, lib.oqmc_last_error(ctx._h)
    torch.cuda.synchronize()
    assert torch.equal(Xa, Xb) and torch.allclose(sa, sb, rtol=1e-12, atol=1e-12)
    assert not torch.equal(Xa, X0)
