"""B-spline Jastrow parameters: coefficient layout and the reference's
validation rules (vmc_gto.py:580-617, gto.py:18-33, 948-968)."""
import numpy as np
import pytest

from omegaqmc_b200 import molecules as M
from omegaqmc_b200.system import build_system, bspline_coefs


def test_coefficients_carry_cusp_and_boundary():
    c = bspline_coefs([0.4, 0.3, 0.2], 0.5, 0.25)
    np.testing.assert_allclose(c, [0.3 - 2 * 0.5 * 0.25, 0.4, 0.3, 0.2, 0, 0, 0])


def test_defaults_and_cusp_values():
    mf = M.make_mf("H2O")
    s = build_system(mf, {"J2_bspline": {"like": [0.1, 0.2], "unlike": [0.3, 0.1, 0.05]},
                          "J1_bspline": {"O": [0.1, 0.2], "H": [0.3, 0.4]}})
    assert s.bs2["r_cut"] == 10.0
    assert s.bs2["like"].shape == (6,) and s.bs2["unlike"].shape == (7,)
    # no cusp correction: J1 cusp value -Z -> c0 = p[1] + 2 dr Z
    c, rc = s.bs1[0]
    assert rc == 10.0 and np.isclose(c[0], 0.2 + 2 * (10.0 / 3) * 8.0)
    sc = build_system(mf, {"J1_bspline": {"O": [0.1, 0.2], "H": [0.3, 0.4]}},
                      M.synthetic_cusp_params(mf.mol))
    assert np.isclose(sc.bs1[0][0][0], 0.2)          # cusp-corrected: cusp value 0


def test_validation_errors_and_warnings():
    mf = M.make_mf("H2O")
    with pytest.raises(ValueError):
        build_system(mf, {"J2_bspline": {"like": [0.1], "unlike": [0.3, 0.1]}})
    with pytest.raises(TypeError):
        build_system(mf, {"J1_bspline": [0.1, 0.2]})
    with pytest.raises(ValueError):
        build_system(mf, {"J2_bspline": {"like": [0.1, 0.2], "unlike": [0.3, 0.1]}}, None,
                     {"J1": {"O": {"r_cut": 3.0}}})
    with pytest.warns(UserWarning):
        build_system(mf, {"J2_pade": {"like": [0.25, 1.0], "unlike": [0.5, 1.0]},
                          "J2_bspline": {"like": [0.1, 0.2], "unlike": [0.3, 0.1]}})
    with pytest.raises(NotImplementedError):
        build_system(mf, {"J4_unknown": {}})
    assert build_system(mf, {"J3_eeI": {}}).j3 is None
    # an element without a configured cutoff has no one-body spline
    s = build_system(mf, {"J1_bspline": {"O": [0.1, 0.2], "H": [0.3, 0.4]}}, None,
                     {"J1": {"O": {"r_cut": 3.0}}})
    assert s.bs1[0] is not None and s.bs1[1] is None and s.bs1[2] is None
