"""J3_eeI three-body Jastrow: host-side tables and the oracle.

* the constraint map (free parameters -> symmetric gammas) of the package
  and of the oracle equal the reference's ``_build_eeI_constraint_map``
  (gto.py:321-463) on stored orders and cutoffs;
* ``parse_j3`` follows the driver's validation (vmc_gto.py:595-611) and
  ``_sanitize_J3_eeI_params`` (gto.py:254-306);
* the oracle's analytic gradient and Laplacian agree with finite
  differences of its value.
"""
import warnings

import numpy as np
import pytest

from helpers import GOLDEN, golden_system
from oracle import gto_oracle as O
from omegaqmc_b200 import molecules as M
from omegaqmc_b200.system import build_system, eeI_constraint_map, eeI_num_params, parse_j3


def _maps():
    g = np.load(f"{GOLDEN}/golden_eeI_map.npz")
    for k in g.files:
        if k.startswith("A_"):
            n_ei, n_ee, rc = k[2:].split("_")
            yield (int(n_ei), int(n_ee), float(rc)), g[k], g["lmn_" + k[2:]]


@pytest.mark.parametrize("case", list(_maps()), ids=lambda c: "%d_%d_%g" % c[0])
def test_constraint_map_matches_reference(case):
    (n_ei, n_ee, rc), A_ref, lmn_ref = case
    A, lmn = eeI_constraint_map(n_ei, n_ee, rc)
    assert A.shape == A_ref.shape == (len(lmn), eeI_num_params(n_ei, n_ee))
    np.testing.assert_array_equal(np.array(lmn), lmn_ref)
    np.testing.assert_allclose(A, A_ref, rtol=0, atol=1e-13)
    A_o, lmn_o = O.eeI_constraint_map(n_ei, n_ee, rc)
    np.testing.assert_allclose(A_o, A_ref, rtol=0, atol=1e-13)


def test_num_params_default_orders():
    assert eeI_num_params(3, 3) == 26
    assert eeI_num_params(2, 2) == 8


def test_gammas_are_cusp_free():
    """The constrained polynomial times the envelope has zero slope in r_ee
    at r_ee = 0 and in r_1I at r_1I = 0 (the two no-cusp conditions)."""
    rng = np.random.default_rng(0)
    n_ei, n_ee, rc = 3, 3, 5.0
    A, lmn = eeI_constraint_map(n_ei, n_ee, rc)
    vec = A @ rng.normal(size=A.shape[1])
    g = np.zeros((n_ei + 1, n_ei + 1, n_ee + 1))
    for k, (l, m, n) in enumerate(lmn):
        g[l, m, n] = g[m, l, n] = vec[k]
    L = 0.5 * rc
    for r in (0.3, 1.1, 1.7, 2.2):
        # coincident electrons sit at the same distance from the nucleus
        _, _, u12, _, _, _ = O._eeI_poly_derivs(g, 0.0, r, r, L)
        assert abs(u12) < 1e-12
        # an electron at the nucleus is r_ee = r_2I from the other one
        _, u1, _, _, _, _ = O._eeI_poly_derivs(g, r, 0.0, r, L)
        assert abs(u1) < 1e-12


def _mol():
    return M.make_mf("H2O").mol


def test_parse_j3_validation():
    mol = _mol()
    with pytest.raises(TypeError):
        parse_j3({"J3_eeI": [0.1] * 26}, mol)
    with pytest.raises(ValueError):
        parse_j3({"J3_eeI": {"O": np.zeros(26)}}, mol)
    with pytest.warns(UserWarning, match="expected 26 params"):
        j3 = parse_j3({"J3_eeI": {"like+O": np.ones(25), "unlike+H": np.ones(26)}}, mol)
    assert np.all(j3["params"]["like+O"] == 0.0)
    with pytest.warns(UserWarning, match="1-D"):
        parse_j3({"J3_eeI": {"like+O": np.ones((2, 13))}}, mol)
    # keys of absent elements are ignored; no block left -> no term
    assert parse_j3({"J3_eeI": {"like+N": np.ones(26)}}, mol) is None
    assert parse_j3({}, mol) is None


def test_parse_j3_types_and_orders():
    mol = _mol()
    rng = np.random.default_rng(1)
    j3 = parse_j3({"J3_eeI": {"unlike+H": rng.normal(size=8)}}, mol,
                  {"J3": {"N_eI": 2, "N_ee": 2, "r_cut": 4.0}})
    assert (j3["n_eI"], j3["n_ee"], j3["r_cut"]) == (2, 2, 4.0)
    assert j3["elements"] == ["H"]
    assert j3["types"] == [-1 if mol.atom_symbol(i) == "O" else 0 for i in range(mol.natm)]
    assert j3["on"].tolist() == [[0, 1]]
    g = j3["gamma"][0, 1]
    assert g.shape == (3, 3, 3)
    np.testing.assert_array_equal(g, np.transpose(g, (1, 0, 2)))
    np.testing.assert_allclose(g, O.eeI_gamma3d(j3["params"]["unlike+H"], 2, 2, 4.0),
                               rtol=0, atol=1e-15)
    with pytest.raises(ValueError):
        parse_j3({"J3_eeI": {"like+H": np.zeros(8)}}, mol, {"J3": {"N_eI": 2, "N_ee": 0}})


@pytest.mark.parametrize("name", ["h2o_j3", "lih_j3"])
def test_oracle_j3_vgl_vs_finite_differences(name):
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        s, d = golden_system(name)
    X = d["X"][:4].copy()
    g, lap = O.j3_vgl(s, X)
    h = 1e-4
    W, n_e, _ = X.shape
    for e in range(n_e):
        fd_l = np.zeros(W)
        for c in range(3):
            Xp, Xm = X.copy(), X.copy()
            Xp[:, e, c] += h
            Xm[:, e, c] -= h
            jp, jm, j0 = O.j3_value(s, Xp), O.j3_value(s, Xm), O.j3_value(s, X)
            np.testing.assert_allclose((jp - jm) / (2 * h), g[:, e, c], rtol=1e-5, atol=1e-5)
            fd_l += (jp - 2 * j0 + jm) / (h * h)
        np.testing.assert_allclose(fd_l, lap[:, e], rtol=1e-3, atol=1e-3)


def test_build_system_carries_j3_next_to_other_terms():
    mf = M.make_mf("H2O")
    rng = np.random.default_rng(2)
    s = build_system(mf, {"J2_pade": {"like": [0.25, 1.0], "unlike": [0.5, 1.0]},
                          "J3_eeI": {"like+O": rng.normal(size=26) * 0.01}})
    assert s.has_j2 and s.j3 is not None and s.j3["on"].tolist() == [[1, 0]]
