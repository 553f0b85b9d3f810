"""Multi-determinant trial dicts on the host: parsing (restricted and UHF
layouts, gto.py:846-863), validation, and the oracle's expansion against
the single determinant it reduces to."""
import numpy as np
import pytest

from helpers import golden_system, seeded_walkers
from oracle import gto_oracle as O
from omegaqmc_b200 import molecules as M
from omegaqmc_b200.system import build_system, parse_trial


def _mf():
    return M.make_mf("LiH")


def _trial(mf, uhf=False):
    rng = np.random.default_rng(0)
    C = np.asarray(mf.mo_coeff)[:, :2]
    mo = np.concatenate([C, rng.normal(size=(C.shape[0], 2)) * 0.3], axis=1)
    if uhf:
        mo = np.stack([mo, mo + 0.01])
    return {"mo_coeff": mo, "ci_coeffs": np.array([0.9, 0.3]),
            "occ_up": np.array([[0, 1], [0, 2]]), "occ_dn": np.array([[0, 1], [0, 3]])}


def test_parse_restricted_and_uhf_layouts():
    mf = _mf()
    t = parse_trial(_trial(mf), 2, 2)
    assert t["C"].shape[1] == 4 and t["occ_dn"].tolist() == [[0, 1], [0, 3]]
    tu = parse_trial(_trial(mf, uhf=True), 2, 2)
    assert tu["C"].shape[1] == 8
    assert tu["occ_dn"].tolist() == [[4, 5], [4, 7]]          # beta half
    np.testing.assert_array_equal(tu["C"][:, 4:], _trial(mf, uhf=True)["mo_coeff"][1])


def test_trial_validation():
    mf = _mf()
    t = _trial(mf)
    with pytest.raises(ValueError):
        parse_trial(dict(t, occ_up=np.array([[0, 1, 2], [0, 1, 3]])), 2, 2)
    with pytest.raises(ValueError):
        parse_trial(dict(t, ci_coeffs=np.array([1.0])), 2, 2)
    with pytest.raises(ValueError):
        parse_trial(dict(t, occ_dn=np.array([[0, 1], [0, 9]])), 2, 2)
    with pytest.raises(ValueError):
        parse_trial(dict(t, mo_coeff=np.zeros((3, 19, 4))), 2, 2)


def test_build_system_takes_the_first_up_determinant_as_orbitals():
    mf = _mf()
    t = _trial(mf)
    s = build_system(mf, None, None, None, t)
    np.testing.assert_array_equal(s.C, np.asarray(t["mo_coeff"])[:, [0, 1]])
    assert s.md is not None and len(s.md["ci"]) == 2


def test_single_term_expansion_equals_single_determinant():
    mf = _mf()
    pc = {"J2_pade": {"like": np.array([0.25, 1.0]), "unlike": np.array([0.5, 1.0])}}
    C = np.asarray(mf.mo_coeff)[:, :2]
    t = {"mo_coeff": C, "ci_coeffs": np.array([-0.7]), "occ_up": np.array([[0, 1]]),
         "occ_dn": np.array([[0, 1]])}
    s1 = build_system(mf, pc)
    sm = build_system(mf, pc, None, None, t)
    X = seeded_walkers(s1, 6, 1.0, 2)
    a, b = O.evaluate(s1, X), O.evaluate(sm, X)
    np.testing.assert_allclose(b["logpsi"], a["logpsi"] + np.log(0.7), rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(b["e_loc"], a["e_loc"], rtol=1e-10, atol=1e-10)


@pytest.mark.parametrize("name", ["h2o_md", "lih_md_uhf"])
def test_multidet_gradient_and_laplacian_vs_finite_differences(name):
    s, d = golden_system(name)
    X = d["X"][:3].copy()
    _, g, lap = O.multidet_assemble(s, X)
    h = 1e-4
    for e in range(X.shape[1]):
        fd_l = np.zeros(X.shape[0])
        for c in range(3):
            Xp, Xm = X.copy(), X.copy()
            Xp[:, e, c] += h
            Xm[:, e, c] -= h
            lp, lm, l0 = O.log_slater(s, Xp), O.log_slater(s, Xm), O.log_slater(s, X)
            np.testing.assert_allclose((lp - lm) / (2 * h), g[:, e, c], rtol=1e-5, atol=1e-5)
            fd_l += (lp - 2 * l0 + lm) / (h * h)
        np.testing.assert_allclose(fd_l, lap[:, e], rtol=2e-3, atol=2e-3)
