"""Jastrow-parameter derivatives on the GPU (oqmc_param_derivs) against the
oracle, FP64, and the flat linear-method inputs end to end."""
import numpy as np
import pytest

from helpers import seeded_walkers
from oracle import gto_oracle as O
from omegaqmc_b200 import molecules as M
from omegaqmc_b200.context import GTOContext
from omegaqmc_b200.optim import build_matrices, raw_to_flat, walker_derivatives
from omegaqmc_b200.system import build_system

pytestmark = pytest.mark.gpu

CASES = [("LiH", True, None), ("H2O", False, None), ("N2", False, None), ("H2O", False, "bspline"),
         ("LiH", True, "bspline"), ("H2O", False, "j3"), ("LiH", True, "j3")]


def _params(mol, cusp, extra):
    pc = M.default_params_corr(mol, cusp=cusp, j1=True)
    if extra == "bspline":
        pc["J2_bspline"] = {"like": np.array([0.2, 0.1, 0.05, 0.02]),
                            "unlike": np.array([0.4, 0.25, 0.1, 0.05, 0.02])}
        pc["J1_bspline"] = {s: np.array([-0.1, 0.05, 0.02]) for s in set(mol.elements)}
    if extra == "j3":
        rng = np.random.default_rng(6)
        els = sorted(set(mol.elements))
        pc["J3_eeI"] = {p + e: rng.normal(size=8) * 0.02 for e in els for p in ("like+", "unlike+")
                        if p + e != "like+" + els[0]}
    return pc


def _config(mol, extra):
    if extra == "bspline":
        return {"J2": {"r_cut": 3.5}, "J1": {e: {"r_cut": 3.0} for e in set(mol.elements)}}
    if extra == "j3":
        return {"J3": {"N_eI": 2, "N_ee": 2, "r_cut": 4.5}}
    return None


@pytest.mark.filterwarnings("ignore::UserWarning")
@pytest.mark.parametrize("name,cusp,extra", CASES)
def test_param_derivatives_match_oracle(name, cusp, extra):
    mf = M.make_mf(name)
    pc = _params(mf.mol, cusp, extra)
    pcu = M.synthetic_cusp_params(mf.mol) if cusp else None
    cfg = _config(mf.mol, extra)
    s = build_system(mf, pc, pcu, cfg)
    ctx = GTOContext(s)
    X = seeded_walkers(s, 257, 0.9, 11)          # ragged: 3 CTAs of 128
    e, dl, de = walker_derivatives(ctx, X, pc)
    ref_dl_raw, ref_de_raw = O.param_derivatives(s, X)
    ref_dl = raw_to_flat(ref_dl_raw, pc, s)
    ref_de = raw_to_flat(ref_de_raw, pc, s)
    sc_l = np.abs(ref_dl).max(axis=0) + 1.0
    sc_e = np.abs(ref_de).max(axis=0) + 1.0
    assert np.max(np.abs(dl - ref_dl) / sc_l) < 1e-10
    assert np.max(np.abs(de - ref_de) / sc_e) < 1e-9
    ref_e = O.evaluate(s, X)["e_loc"]
    sc = 0.5 * np.abs(ref_e).max() + 1.0
    assert np.max(np.abs(e - ref_e)) / sc < 1e-9
    H, S = build_matrices(e, dl, de)
    assert np.all(np.isfinite(H)) and np.all(np.isfinite(S))
