"""Oracle of the Jastrow-parameter derivatives against finite differences of
the oracle's own log|psi| and E_L (central differences in each raw
parameter)."""
import copy

import numpy as np
import pytest

from helpers import seeded_walkers
from oracle import gto_oracle as O
from omegaqmc_b200 import molecules as M
from omegaqmc_b200.system import build_system


def _raw_get(s, k):
    return s.j2.reshape(-1)[k] if k < 4 else s.j1.reshape(-1)[k - 4]


def _raw_set(s, k, v):
    s2 = copy.deepcopy(s)
    if k < 4:
        j2 = s2.j2.copy().reshape(-1)
        j2[k] = v
        s2.j2 = j2.reshape(2, 2)
    else:
        j1 = s2.j1.copy().reshape(-1)
        j1[k - 4] = v
        s2.j1 = j1.reshape(-1, 2)
    return s2


@pytest.mark.parametrize("name", ["LiH", "H2O"])
def test_param_derivatives_match_finite_differences(name):
    mf = M.make_mf(name)
    pc = M.default_params_corr(mf.mol, cusp=False, j1=True)
    s = build_system(mf, pc)
    X = seeded_walkers(s, 6, 0.8, 3)
    dl, de = O.param_derivatives(s, X)
    for k in range(4 + 2 * s.natm):
        v = _raw_get(s, k)
        h = 1e-5 * max(1.0, abs(v))
        sp, sm = _raw_set(s, k, v + h), _raw_set(s, k, v - h)
        fd_l = (O.log_psi(sp, X) - O.log_psi(sm, X)) / (2 * h)
        fd_e = (O.evaluate(sp, X)["e_loc"] - O.evaluate(sm, X)["e_loc"]) / (2 * h)
        np.testing.assert_allclose(dl[:, k], fd_l, rtol=1e-6, atol=1e-7)
        np.testing.assert_allclose(de[:, k], fd_e, rtol=1e-5, atol=1e-5 * (1 + np.abs(fd_e).max()))


def test_bspline_param_derivatives_match_finite_differences():
    mf = M.make_mf("H2O")
    pc = {"J1_bspline": {"O": np.array([0.3, -0.2, 0.1, 0.05]), "H": np.array([0.1, 0.05, -0.03])},
          "J2_bspline": {"like": np.array([0.2, 0.1, 0.05, 0.02]),
                         "unlike": np.array([0.4, 0.25, 0.1, 0.05, 0.02])}}
    cfg = {"J2": {"r_cut": 3.0}, "J1": {"O": {"r_cut": 2.5}, "H": {"r_cut": 2.0}}}
    s = build_system(mf, pc, None, cfg)
    X = seeded_walkers(s, 5, 0.9, 4)
    dl, de = O.param_derivatives(s, X)
    assert dl.shape[1] == O.param_count(s) == 4 + 6 + 4 + 5 + 4 + 3
    keys = [("J2_bspline", "like", 4), ("J2_bspline", "unlike", 5), ("J1_bspline", "O", 4),
            ("J1_bspline", "H", 3)]
    col = 4 + 2 * s.natm
    for term, key, n in keys:
        for q in range(n):
            pp, pm = copy.deepcopy(pc), copy.deepcopy(pc)
            h = 1e-6
            pp[term][key] = pc[term][key].copy()
            pm[term][key] = pc[term][key].copy()
            pp[term][key][q] += h
            pm[term][key][q] -= h
            sp, sm = build_system(mf, pp, None, cfg), build_system(mf, pm, None, cfg)
            fd_l = (O.log_psi(sp, X) - O.log_psi(sm, X)) / (2 * h)
            fd_e = (O.evaluate(sp, X)["e_loc"] - O.evaluate(sm, X)["e_loc"]) / (2 * h)
            np.testing.assert_allclose(dl[:, col], fd_l, rtol=1e-6, atol=1e-7)
            np.testing.assert_allclose(de[:, col], fd_e, rtol=1e-5, atol=2e-5 * (1 + np.abs(fd_e).max()))
            col += 1


def test_j3_param_derivatives_match_finite_differences():
    """J3_eeI: the oracle's unique-gamma derivatives, mapped onto the free
    parameters through the constraint matrix (optim.raw_to_flat), against
    central differences in each free parameter."""
    from omegaqmc_b200.optim import flatten_params, raw_to_flat
    mf = M.make_mf("LiH")
    rng = np.random.default_rng(4)
    pc = {"J2_pade": {"like": np.array([0.25, 1.0]), "unlike": np.array([0.5, 1.0])},
          "J3_eeI": {"like+Li": rng.normal(size=8) * 0.02, "unlike+Li": rng.normal(size=8) * 0.02,
                     "unlike+H": rng.normal(size=8) * 0.02}}
    cfg = {"J3": {"N_eI": 2, "N_ee": 2, "r_cut": 5.0}}
    s = build_system(mf, pc, None, cfg)
    X = seeded_walkers(s, 4, 0.9, 5)
    dl, de = O.param_derivatives(s, X)
    assert dl.shape[1] == O.param_count(s) == 4 + 2 * s.natm + 3 * 18
    fl, fe = raw_to_flat(dl, pc, s), raw_to_flat(de, pc, s)
    _, layout = flatten_params(pc)
    col = 0
    for term, key, n in layout:
        if term != "J3_eeI":
            col += n
            continue
        for q in range(n):
            pp, pm = copy.deepcopy(pc), copy.deepcopy(pc)
            h = 1e-6
            pp[term][key][q] += h
            pm[term][key][q] -= h
            sp, sm = build_system(mf, pp, None, cfg), build_system(mf, pm, None, cfg)
            fd_l = (O.log_psi(sp, X) - O.log_psi(sm, X)) / (2 * h)
            fd_e = (O.evaluate(sp, X)["e_loc"] - O.evaluate(sm, X)["e_loc"]) / (2 * h)
            np.testing.assert_allclose(fl[:, col], fd_l, rtol=1e-6, atol=1e-7)
            np.testing.assert_allclose(fe[:, col], fd_e, rtol=1e-5, atol=2e-5 * (1 + np.abs(fd_e).max()))
            col += 1
