"""B200-native GTO variational Monte Carlo hot path of ΩQMC (myung-group/OmegaQMC).

Public surface mirrors the reference's: :func:`get_psi_fun`,
:func:`get_vmc_gto_func`, :class:`VMCTrialState` and
:func:`generate_molecular_orbitals` (here backed by this package's RHF).
The arithmetic runs in ``liboqmc_b200.so`` (sm_100a CUDA, C ABI in
``include/oqmc_b200.h``)."""
from __future__ import annotations

import os

from .system import Mole, MeanField, build_system, read_shell  # noqa: F401

__version__ = "0.1.0"

__all__ = ["get_psi_fun", "get_vmc_gto_func", "VMCTrialState", "generate_molecular_orbitals",
           "Mole", "MeanField", "build_system", "read_shell"]


def get_psi_fun(*a, **k):
    from .psi import get_psi_fun as f
    return f(*a, **k)


def get_vmc_gto_func(*a, **k):
    from .vmc import get_vmc_gto_func as f
    return f(*a, **k)


def __getattr__(name):
    if name == "VMCTrialState":
        from .psi import VMCTrialState
        return VMCTrialState
    raise AttributeError(name)


def generate_molecular_orbitals(astr, units="Bohr", basis="cc-pvdz-shaped", spin=0,
                                charge=0, ao_splines=None, symmetrization_level=1, **kw):
    """RHF mean-field object for ``astr`` (``OmegaQMC/vmc_gto.py:217-452`` runs
    PySCF; here the package's own RHF).  ``basis`` is a PySCF-format dict
    ``{element: [[am, [alpha, c...], ...], ...]}``, basis-set text in NWChem
    or Gaussian94 format (or the path of such a file, or a dict of texts per
    element; :mod:`omegaqmc_b200.basis`), or one of the generated sets
    ``"cc-pvdz-shaped"`` / ``"sto-3g"`` (H only).  ``ao_splines``
    (True or a dict of grid options) switches on the quintic radial-spline
    AO transform, stored on ``mf.mol.ao_radial_transform`` as in the
    reference (``vmc_gto.py:278-290, 415``).  With ``symmetrization_level``
    >= 1 (the reference's default) a molecule without point-group symmetry
    is moved to the reference's canonical frame (centre of nuclear charge,
    charge-inertia principal axes; :mod:`omegaqmc_b200.frame`); molecules
    with symmetry keep their input frame."""
    from . import molecules as M
    from .rhf import run_rhf
    if spin != 0:
        raise NotImplementedError("only closed-shell RHF is supported")
    from .basis import load_basis
    atoms = Mole(astr, {s: [] for s in M.ELEMENT_Z}, unit=units)._atom
    syms = sorted({s for s, _ in atoms})
    if isinstance(basis, str):
        name = basis.lower()
        if name == "cc-pvdz-shaped":
            basis = {s: M.ccpvdz_shaped(s) for s in syms}
        elif name == "sto-3g" and syms == ["H"]:
            basis = {"H": M.sto3g_h()}
        elif "\n" in basis or os.path.exists(basis):
            basis = load_basis(basis, syms)
        else:
            raise ValueError(f"unknown basis {basis!r}; pass a PySCF-format dict or the "
                             "NWChem / Gaussian94 text of the basis set")
    elif isinstance(basis, dict) and any(isinstance(v, str) for v in basis.values()):
        basis = load_basis(basis, syms)
    mol = Mole(astr, basis, unit=units, charge=charge, basis_name="gen")
    if symmetrization_level >= 1:
        from .frame import canonical_coordinates
        xyz = canonical_coordinates(mol.atom_coords(), mol.atom_charges())
        mol = Mole([(a, tuple(c)) for (a, _), c in zip(mol._atom, xyz)], basis, unit="Bohr",
                   charge=charge, basis_name="gen")
    mol.ao_radial_transform = ao_splines
    return run_rhf(mol, **kw)
