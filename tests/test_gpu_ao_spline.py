"""Quintic radial-spline AO transform on the GPU: Sherman-Morrison-tracked
sweeps (FP64 and mixed) match a fresh oracle evaluation on the splined
basis, and the kernels built for analytic radials (specialised, batched,
tensor-core) refuse the transform.  (The FP64 evaluation is checked against
the reference's golden vectors, cases h2o_spline and lih_spline_cusp, in
test_gpu_eval.py.)"""
import numpy as np
import pytest
import torch

from helpers import golden_system, seeded_walkers
from oracle import gto_oracle as O
from omegaqmc_b200.batch import BatchedSampler
from omegaqmc_b200.context import GTOContext
from omegaqmc_b200.sampler import WalkerEnsemble

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["h2o_spline", "lih_spline_cusp"])
def test_spline_sweeps_track_fresh_evaluation(name):
    s, _ = golden_system(name)
    ctx = GTOContext(s)
    W = 512
    ens = WalkerEnsemble(ctx, seeded_walkers(s, W, 0.9, 3), "fp64", seed=11, refresh_every=10**9)
    ep = torch.empty(W, 4, dtype=torch.float64, device="cuda")
    ens.run(30, 0.4, eparts_last=ep)
    torch.cuda.synchronize()
    Xf = ens.X.cpu().numpy()
    ref = O.evaluate(s, Xf)
    sc = 0.5 * (np.sum(np.abs(ref["lap"]), axis=1) + np.sum(ref["grad"] ** 2, axis=(1, 2))) + 1
    err = np.abs(ep[:, 3].cpu().numpy() - ref["e_loc"]) / (np.abs(ref["e_loc"]) + sc)
    assert np.max(err) < 1e-10, np.max(err)
    ld = ens.logdet().cpu().numpy()
    assert np.max(np.abs(ld - O.log_slater(s, Xf)) / (np.abs(ld) + 1)) < 1e-8
    ens_m = WalkerEnsemble(ctx, Xf, "mixed", seed=12)
    ens_m.run(1, 1e-9, eparts_last=ep)
    torch.cuda.synchronize()
    ref_m = O.evaluate(s, ens_m.X.cpu().numpy())
    e = np.abs(ep[:, 3].cpu().numpy() - ref_m["e_loc"])
    assert np.median(e) < 1e-4 and np.quantile(e, 0.99) < 5e-3, (np.median(e), np.quantile(e, 0.99))
    assert ctx.flags() == 0


def test_spline_refused_by_analytic_radial_kernels():
    s, _ = golden_system("h2o_spline")
    ctx = GTOContext(s)
    with pytest.raises(NotImplementedError):
        ctx.specialize()
    with pytest.raises(NotImplementedError):
        ctx.use_tensor_cores(True)
    X = torch.as_tensor(seeded_walkers(s, 64, 0.9, 0), device="cuda")
    with pytest.raises(NotImplementedError):
        BatchedSampler([ctx], [X], [0.5], cap=1)


def test_spline_optimiser_inputs_match_oracle():
    """Jastrow-parameter derivatives on a splined basis: the orbitals enter
    only through the gradient of ln|psi|."""
    import json
    from omegaqmc_b200.optim import raw_to_flat, walker_derivatives
    s, d = golden_system("h2o_spline")
    pc = {k: {kk: np.asarray(vv, dtype=np.float64) for kk, vv in v.items()}
          for k, v in json.loads(str(d["spec"]))["params_corr"].items()}
    ctx = GTOContext(s)
    X = seeded_walkers(s, 130, 0.8, 22)
    e, dl, de = walker_derivatives(ctx, X, pc)
    rl, re_ = O.param_derivatives(s, X)
    ref_dl, ref_de = raw_to_flat(rl, pc, s), raw_to_flat(re_, pc, s)
    assert np.max(np.abs(dl - ref_dl) / (np.abs(ref_dl).max(axis=0) + 1.0)) < 1e-10
    assert np.max(np.abs(de - ref_de) / (np.abs(ref_de).max(axis=0) + 1.0)) < 1e-9
