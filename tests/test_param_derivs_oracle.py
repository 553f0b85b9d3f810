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
