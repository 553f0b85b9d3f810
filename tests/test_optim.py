"""Linear-method inputs: flat parameter order, the raw -> flat mapping
against finite differences of the oracle in the flat parameters, and the
H / S matrices."""
import copy

import numpy as np

from helpers import seeded_walkers
from oracle import gto_oracle as O
from omegaqmc_b200 import molecules as M
from omegaqmc_b200.optim import build_matrices, flatten_params, raw_to_flat
from omegaqmc_b200.system import build_system


def _set_flat(pc, flat):
    pc = copy.deepcopy(pc)
    _, layout = flatten_params(pc)
    o = 0
    for term, key, n in layout:
        v = np.asarray(flat[o:o + n])
        pc[term][key] = v if n > 1 else float(v[0])
        o += n
    return pc


def test_flatten_order_follows_sorted_keys():
    pc = {"J2_pade": {"unlike": [0.5, 3.0], "like": [0.25, 2.0]}, "J1_pade": {"O": 1.5, "H": [1.0, 2.0]}}
    flat, layout = flatten_params(pc)
    assert [(t, k) for t, k, _ in layout] == [("J1_pade", "H"), ("J1_pade", "O"),
                                              ("J2_pade", "like"), ("J2_pade", "unlike")]
    np.testing.assert_array_equal(flat, [1.0, 2.0, 1.5, 0.25, 2.0, 0.5, 3.0])


def test_flat_derivatives_match_finite_differences():
    mf = M.make_mf("H2O")
    pc = {"J1_pade": {"H": 1.2, "O": 2.0}, "J2_pade": {"like": [0.25, 3.0], "unlike": [0.5, 3.0]}}
    s = build_system(mf, pc)
    X = seeded_walkers(s, 5, 0.8, 2)
    dl_raw, de_raw = O.param_derivatives(s, X)
    dl = raw_to_flat(dl_raw, pc, s)
    de = raw_to_flat(de_raw, pc, s)
    flat, _ = flatten_params(pc)
    for k in range(flat.size):
        h = 1e-5 * max(1.0, abs(flat[k]))
        fp, fm = flat.copy(), flat.copy()
        fp[k] += h
        fm[k] -= h
        sp = build_system(mf, _set_flat(pc, fp))
        sm = build_system(mf, _set_flat(pc, fm))
        fd_l = (O.log_psi(sp, X) - O.log_psi(sm, X)) / (2 * h)
        fd_e = (O.evaluate(sp, X)["e_loc"] - O.evaluate(sm, X)["e_loc"]) / (2 * h)
        np.testing.assert_allclose(dl[:, k], fd_l, rtol=1e-6, atol=1e-7)
        np.testing.assert_allclose(de[:, k], fd_e, rtol=1e-5, atol=1e-5 * (1 + np.abs(fd_e).max()))


def test_build_matrices_definitions():
    rng = np.random.default_rng(0)
    E = -1.0 + 0.1 * rng.normal(size=200)
    dl = rng.normal(size=(200, 3))
    de = rng.normal(size=(200, 3))
    H, S = build_matrices(E, dl, de)
    assert H.shape == S.shape == (4, 4)
    assert S[0, 0] == 1.0 and np.allclose(S, S.T)
    assert np.all(np.linalg.eigvalsh(S[1:, 1:]) > 0)
    assert np.isclose(H[0, 0], E.mean())
    dD = dl - dl.mean(axis=0)
    np.testing.assert_allclose(H[1:, 0], (dD * E[:, None]).mean(axis=0))
    np.testing.assert_allclose(H[1:, 1:], dD.T @ (de + dD * E[:, None]) / 200)


def test_flat_bspline_derivatives_match_finite_differences():
    mf = M.make_mf("H2O")
    pc = {"J1_bspline": {"O": np.array([0.3, -0.2, 0.1]), "H": np.array([0.1, 0.05, -0.03])},
          "J2_bspline": {"like": np.array([0.2, 0.1, 0.05]), "unlike": np.array([0.4, 0.25, 0.1])},
          "J2_pade": {"like": [0.25, 3.0], "unlike": [0.5, 3.0]}}
    cfg = {"J2": {"r_cut": 3.0}, "J1": {"O": {"r_cut": 2.5}, "H": {"r_cut": 2.0}}}
    import warnings
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        s = build_system(mf, pc, None, cfg)
        X = seeded_walkers(s, 4, 0.9, 5)
        dl_raw, de_raw = O.param_derivatives(s, X)
        dl = raw_to_flat(dl_raw, pc, s)
        de = raw_to_flat(de_raw, pc, s)
        flat, _ = flatten_params(pc)
        for k in range(flat.size):
            h = 1e-6
            fp, fm = flat.copy(), flat.copy()
            fp[k] += h
            fm[k] -= h
            sp = build_system(mf, _set_flat(pc, fp), None, cfg)
            sm = build_system(mf, _set_flat(pc, fm), None, cfg)
            fd_l = (O.log_psi(sp, X) - O.log_psi(sm, X)) / (2 * h)
            fd_e = (O.evaluate(sp, X)["e_loc"] - O.evaluate(sm, X)["e_loc"]) / (2 * h)
            np.testing.assert_allclose(dl[:, k], fd_l, rtol=1e-5, atol=1e-6)
            np.testing.assert_allclose(de[:, k], fd_e, rtol=1e-4, atol=5e-5 * (1 + np.abs(fd_e).max()))
