"""The canonical molecular frame of generate_molecular_orbitals
(symmetrization_level >= 1, OmegaQMC/vmc_gto.py:314-352) against the
reference's own charge_inertia_axes (OmegaQMC/symm/point_groups.py:524-568),
whose outputs tests/golden/make_golden.py stored for asymmetric geometries,
rotated and shifted copies, and a degenerate (linear) case."""
import numpy as np
import pytest

from helpers import GOLDEN
from omegaqmc_b200 import generate_molecular_orbitals
from omegaqmc_b200.frame import canonical_coordinates, charge_inertia_axes, has_point_symmetry


def _golden():
    return dict(np.load(f"{GOLDEN}/golden_frame.npz"))


def test_charge_inertia_axes_match_reference():
    g = _golden()
    tags = sorted({k.split("_")[1] for k in g if k.startswith("coords_")})
    assert len(tags) == 8
    for t in tags:
        r = charge_inertia_axes(g[f"coords_{t}"], g[f"charges_{t}"])
        if f"none_{t}" in g:
            assert r is None, t
            continue
        np.testing.assert_allclose(r[0], g[f"centre_{t}"], rtol=0, atol=1e-12)
        np.testing.assert_allclose(r[1], g[f"axes_{t}"], rtol=0, atol=1e-10)


def test_frame_does_not_depend_on_input_orientation():
    g = _golden()
    for k in (0, 2):                 # non-planar, no symmetry (three atoms are at least Cs)
        a = canonical_coordinates(g[f"coords_{k}a"], g[f"charges_{k}a"])
        b = canonical_coordinates(g[f"coords_{k}b"], g[f"charges_{k}b"])
        np.testing.assert_allclose(a, b, atol=1e-9)
        # centred on the nuclear charge, moments ascending along x, y, z
        q = g[f"charges_{k}a"]
        np.testing.assert_allclose(q @ a / q.sum(), 0, atol=1e-12)
        m = [float(np.sum(q * (np.sum(a * a, 1) - a[:, i] ** 2))) for i in range(3)]
        assert m[0] <= m[1] <= m[2]


def test_symmetric_molecules_keep_their_frame():
    water = np.array([[0.0, 0.0, 0.0], [0.0, 1.43, 1.11], [0.0, -1.43, 1.11]])
    assert has_point_symmetry(water, [8, 1, 1])                          # C2v
    ammonia = np.array([[0, 0, 0.0], [1.77, 0, -0.72], [-0.885, 1.533, -0.72],
                        [-0.885, -1.533, -0.72]])
    assert has_point_symmetry(ammonia, [7, 1, 1, 1])                     # C3v, degenerate
    hooh_like = np.array([[0.0, 1.37, 0.0], [0.0, -1.37, 0.0], [1.8, 1.7, 0.3], [-1.8, -1.7, 0.3]])
    assert has_point_symmetry(hooh_like, [8, 8, 1, 1])                   # C2
    g = _golden()
    assert not has_point_symmetry(g["coords_0a"], g["charges_0a"])
    assert has_point_symmetry(g["coords_1a"], g["charges_1a"])           # planar: Cs
    np.testing.assert_array_equal(canonical_coordinates(water, [8, 1, 1]), water)


def test_generate_molecular_orbitals_uses_the_frame():
    basis = {"H": [[0, [1.2, 1.0]], [0, [0.3, 1.0]]], "Li": [[0, [3.0, 1.0]], [0, [0.5, 1.0]]]}
    astr = "Li 0.3 -0.2 0.1; H 0.9 2.1 -0.4; H -1.7 0.6 1.3; H 0.2 -1.1 -2.2"   # no symmetry
    mf = generate_molecular_orbitals(astr, basis=basis)
    c = mf.mol.atom_coords()
    q = mf.mol.atom_charges()
    np.testing.assert_allclose(q @ c / q.sum(), 0, atol=1e-12)
    mf0 = generate_molecular_orbitals(astr, basis=basis, symmetrization_level=0)
    np.testing.assert_allclose(mf0.mol.atom_coords()[0], [0.3, -0.2, 0.1])
    # same distances, same RHF energy in either frame
    d = lambda x: np.linalg.norm(x[:, None] - x[None], axis=-1)
    np.testing.assert_allclose(d(c), d(mf0.mol.atom_coords()), atol=1e-12)
    assert mf.e_tot == pytest.approx(mf0.e_tot, abs=1e-9)
