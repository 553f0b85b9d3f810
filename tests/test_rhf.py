"""RHF front end: integrals against textbook values and the variational
consistency of the whole evaluation chain (VMC of the bare determinant
reproduces E_RHF)."""
import numpy as np

from helpers import seeded_walkers
from omegaqmc_b200 import molecules as M
from omegaqmc_b200.rhf import integrals, run_rhf
from omegaqmc_b200.system import build_system
from oracle import cref
from oracle import gto_oracle as O


def test_h2_sto3g_textbook_values():
    mol = M.named_system("H2")
    S, T, V, g = integrals(mol)
    assert abs(S[0, 1] - 0.6593) < 1e-4           # Szabo & Ostlund, R = 1.4 bohr
    mf = run_rhf(mol)
    assert abs(mf.e_tot - (-1.1167)) < 1e-4


def test_overlap_is_unit_diagonal_and_symmetric():
    for name in ("LiH", "H2O"):
        S, T, V, g = integrals(M.named_system(name))
        assert np.allclose(np.diag(S), 1.0, atol=1e-10)
        assert np.allclose(S, S.T, atol=1e-13)
        assert np.allclose(g, g.transpose(1, 0, 2, 3), atol=1e-12)
        assert np.allclose(g, g.transpose(2, 3, 0, 1), atol=1e-12)


def test_vmc_of_bare_determinant_reproduces_rhf_energy():
    mol = M.named_system("H2O")
    mf = run_rhf(mol)
    s = build_system(M.MeanField(mol, mf.mo_coeff, mf.mo_occ), {})
    X = np.ascontiguousarray(seeded_walkers(s, 256, 0.8, 0))
    step = 0.3
    for k in range(300):
        _, acc = cref.run(s, X, 1, step, seed=k)
        step = float(np.exp(np.log(step) + 0.05 * (acc - 0.4)))
    ser, _ = cref.run(s, X, 1500, step, seed=5)
    m, se, _, _ = O.binning_analysis(ser[:, 3])
    assert abs(m - mf.e_tot) < 3.5 * se + 0.02, (m, se, mf.e_tot)
