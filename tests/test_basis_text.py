"""Basis-set text (NWChem and Gaussian94 exports) read into the PySCF
internal format, and RHF from text equal to RHF from the dict.  The numbers
below are made up for the test; they are not a published basis set."""
import numpy as np
import pytest

from omegaqmc_b200 import generate_molecular_orbitals
from omegaqmc_b200.basis import load_basis, parse_basis_text

NWCHEM = """
# made-up two-element set
BASIS "ao basis" SPHERICAL PRINT
H    S
     12.5000000              0.0200000
      1.9000000              0.1400000
      0.4400000              0.4800000
H    S
      0.1250000              1.0000000
H    P
      0.7500000              1.0000000
Li    S
    600.0000000              0.0007000   -0.0001000
     90.0000000              0.0055000   -0.0009000
      2.0000000              0.2600000   -0.0600000
Li    SP
      0.5000000             -0.1000000    0.1500000
      0.0600000              1.0500000    0.9000000
END
"""

G94 = """****
H     0
S   3   1.00
     12.5000000              0.0200000
      1.9000000              0.1400000
      0.4400000              0.4800000
S   1   1.00
      0.1250000              1.0000000
P   1   1.00
      0.7500000              1.0000000
****
Li     0
S   3   1.00
    600.0000000              0.0007000
     90.0000000              0.0055000
      2.0D+00                0.2600000
SP   2   1.00
      0.5000000             -0.1000000    0.1500000
      0.0600000              1.0500000    0.9000000
****
"""


def test_nwchem_text():
    b = parse_basis_text(NWCHEM)
    assert sorted(b) == ["H", "Li"]
    assert b["H"][0] == [0, [12.5, 0.02], [1.9, 0.14], [0.44, 0.48]]
    assert b["H"][2] == [1, [0.75, 1.0]]
    # general contraction: two coefficient columns
    assert b["Li"][0][0] == 0 and b["Li"][0][1] == [600.0, 0.0007, -0.0001]
    # SP splits into s and p with shared exponents
    assert b["Li"][1] == [0, [0.5, -0.1], [0.06, 1.05]]
    assert b["Li"][2] == [1, [0.5, 0.15], [0.06, 0.9]]


def test_gaussian94_text():
    b = parse_basis_text(G94)
    n = parse_basis_text(NWCHEM)
    assert b["H"] == n["H"]
    assert b["Li"][0] == [0, [600.0, 0.0007], [90.0, 0.0055], [2.0, 0.26]]
    assert b["Li"][1:] == n["Li"][1:]


def test_bad_text_is_refused():
    with pytest.raises(ValueError):
        parse_basis_text("H Q\n 1.0 1.0\n")
    with pytest.raises(ValueError):
        parse_basis_text("H SP\n 1.0 1.0\n")
    with pytest.raises(ValueError):
        load_basis(NWCHEM, ["H", "O"])
    with pytest.raises(ValueError):
        parse_basis_text("****\nH 0\nS 3 1.00\n 1.0 0.5\n****\n")     # truncated shell


def test_rhf_from_text_matches_dict(tmp_path):
    astr = "H 0 0 -0.7; H 0 0 0.7"
    mf_t = generate_molecular_orbitals(astr, basis=NWCHEM)
    mf_d = generate_molecular_orbitals(astr, basis={"H": parse_basis_text(NWCHEM)["H"]})
    np.testing.assert_allclose(mf_t.mo_coeff, mf_d.mo_coeff, atol=1e-12)
    p = tmp_path / "basis.nw"
    p.write_text(NWCHEM)
    mf_f = generate_molecular_orbitals(astr, basis=str(p))
    np.testing.assert_allclose(mf_f.mo_coeff, mf_d.mo_coeff, atol=1e-12)
    mf_e = generate_molecular_orbitals(astr, basis={"H": G94})
    np.testing.assert_allclose(mf_e.mo_coeff, mf_d.mo_coeff, atol=1e-12)
