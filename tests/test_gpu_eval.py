"""GPU parity of the FP64 evaluation kernel against the oracle.

Tolerance (FP64 build): |gpu - oracle| <= 1e-10 * (|oracle| + 1) per
element for log|psi|, grad log|psi|, the per-electron Laplacian and every
local-energy part."""
import numpy as np
import pytest
import torch

from helpers import golden_cases, golden_system, seeded_walkers
from oracle import gto_oracle as O
from omegaqmc_b200 import molecules as M
from omegaqmc_b200.context import GTOContext
from omegaqmc_b200.system import build_system

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _err(a, b):
    a = a.detach().cpu().numpy() if torch.is_tensor(a) else np.asarray(a)
    return float(np.max(np.abs(a - b) / (np.abs(b) + 1.0)))


def _ke_scale(o):
    """Magnitude of the terms the kinetic energy sums, -1/2 (sum lap + |grad|^2):
    near a node of the determinant they cancel, and the FP64 result is only
    defined to 1e-10 of this scale, in the reference as here."""
    return 0.5 * (np.sum(np.abs(o["lap"]), axis=1) + np.sum(o["grad"] ** 2, axis=(1, 2)))


def _check(ctx, s, X):
    r = ctx.evaluate(X)
    o = O.evaluate(s, X)
    for k in ("logpsi", "grad", "lap", "e_ee", "e_en"):
        assert _err(r[k], o[k]) < TOL, (k, _err(r[k], o[k]))
    sc = _ke_scale(o) + 1.0
    for k in ("e_ke", "e_loc"):
        e = np.max(np.abs(r[k].cpu().numpy() - o[k]) / (np.abs(o[k]) + sc))
        assert e < TOL, (k, e)
    lp = ctx.log_psi(X)
    assert _err(lp, o["logpsi"]) < TOL
    assert ctx.flags() == 0


@pytest.mark.parametrize("name", golden_cases())
def test_eval_matches_golden_and_oracle(name):
    s, d = golden_system(name)
    ctx = GTOContext(s)
    r = ctx.evaluate(d["X"])
    for k in ("logpsi", "grad", "lap", "e_ee", "e_en", "e_ke"):
        assert _err(r[k], d[k]) < TOL, (k, _err(r[k], d[k]))
    _check(ctx, s, d["X"])


@pytest.mark.parametrize("name,sigma", [("H2", 0.5), ("LiH", 1.0), ("H2O", 1.0),
                                        ("N2", 1.0), ("H2O_dimer", 1.0)])
def test_eval_4096_seeded_configurations(name, sigma):
    mf = M.make_mf(name)
    s = build_system(mf, M.default_params_corr(mf.mol))
    X = seeded_walkers(s, 4096 if name != "H2O_dimer" else 1024, sigma, 1234)
    _check(GTOContext(s), s, X)


def test_eval_cusp_named_system():
    mf = M.make_mf("H2O")
    cusp = M.synthetic_cusp_params(mf.mol)
    s = build_system(mf, M.default_params_corr(mf.mol, cusp=True), cusp)
    X = seeded_walkers(s, 2048, 0.8, 77)
    _check(GTOContext(s), s, X)


def test_eval_edge_cases():
    mf = M.make_mf("LiH")
    s = build_system(mf, M.default_params_corr(mf.mol))
    ctx = GTOContext(s)
    # empty batch
    r = ctx.evaluate(np.zeros((0, s.n_e, 3)))
    assert r["logpsi"].numel() == 0
    # ragged batch sizes around the CTA size
    for W in (1, 127, 129):
        _check(ctx, s, seeded_walkers(s, W, 1.0, W))
    # electron on a nucleus: finite (Gaussian AOs are regular there)
    X = seeded_walkers(s, 4, 1.0, 5)
    X[0, 0] = s.nuc[0]
    r = ctx.evaluate(X)
    assert torch.isfinite(r["logpsi"]).all()
    # bad shape raises ValueError
    with pytest.raises(ValueError):
        ctx.evaluate(np.zeros((3, s.n_e + 1, 3)))


def test_singular_slater_flags_and_minus_inf():
    mf = M.make_mf("LiH")
    s = build_system(mf, M.default_params_corr(mf.mol))
    ctx = GTOContext(s)
    X = seeded_walkers(s, 2, 1.0, 9)
    X[1, 2] = X[1, 0]   # two same-spin electrons coincide: det = 0
    r = ctx.evaluate(X)
    lp = r["logpsi"].cpu().numpy()
    assert np.isfinite(lp[0]) and (np.isneginf(lp[1]) or lp[1] < -30)
    ctx.flags(clear=True)
