"""The named benchmark systems and their synthetic basis sets.

No quantum-chemistry package is available to this project, so the basis
sets of the named systems are generated here:

* ``sto3g_h`` uses the hydrogen STO-3G-shaped primitives that the
  reference's own tests carry (``tests/test_gto_kinetic_energy.py:677-683``).
* ``ccpvdz_shaped(sym)`` is a *shape-matched synthetic* basis: the same
  angular momenta, number of basis entries, contraction depths and general
  contraction layout as cc-pVDZ (H: 2s1p = 5 functions; Li-Ne: 3s2p1d = 14
  functions, the core s entry a two-column general contraction), built from
  even-tempered primitives with contraction coefficients fitted to
  Slater-type orbitals.  The function counts (LiH 19, H2O 24, N2 28,
  (H2O)2 48) match the real basis; RHF energies are STO-3G-like
  (H2O -74.80, N2 -107.67, LiH -7.88 hartree), not cc-pVDZ's.

Occupied orbitals come from this package's RHF (``omegaqmc_b200.rhf``) by
default; ``seeded_mo_coeff`` gives reproducible non-SCF orbitals for parity
tests (an aufbau-like dominant AO per orbital plus a seeded admixture).
"""
from __future__ import annotations

import numpy as np

from .system import Mole, MeanField, ELEMENT_Z, build_shells, ANG_TO_BOHR

__all__ = ["sto3g_h", "ccpvdz_shaped", "named_system", "NAMED_SYSTEMS",
           "seeded_mo_coeff", "default_params_corr", "benchmark_params_corr",
           "synthetic_cusp_params", "make_mf"]


def sto3g_h():
    """STO-3G-shaped H 1s (the reference tests' primitive data)."""
    return [[0, [3.42525091, 0.15432897], [0.62391373, 0.53532814],
             [0.16885540, 0.44463454]]]


def _even_tempered(a_max, ratio, n):
    return a_max / ratio ** np.arange(n)


# Slater's-rules orbital exponents (zeta of the 1s and of the 2s/2p shells);
# hydrogen uses the molecular value 1.24.
_SLATER = {"H": (1.24, None), "He": (1.69, None), "Li": (2.69, 0.65), "Be": (3.69, 0.975),
           "B": (4.68, 1.3), "C": (5.67, 1.625), "N": (6.67, 1.95), "O": (7.66, 2.275),
           "F": (8.65, 2.6), "Ne": (9.64, 2.925)}
# polarisation exponents of the single d (first row) or p (H, He) function
_POL = {"H": 0.73, "He": 1.2, "Li": 0.2, "Be": 0.26, "B": 0.4, "C": 0.55, "N": 0.82,
        "O": 1.2, "F": 1.6, "Ne": 2.0}


def _sto_fit(alphas, zeta, n, l):
    """Least-squares Gaussian expansion of the Slater function r^(n-1) e^(-zeta r)
    with primitives r^l e^(-alpha r^2), in the r^2-weighted L2 norm; returns the
    coefficients of the unnormalised primitives (read_shell normalises)."""
    r = np.linspace(1e-4, 30.0 / zeta, 6000)
    w = r ** 2
    target = r ** (n - 1) * np.exp(-zeta * r)
    target = target / np.sqrt(np.sum(w * target * target))
    G = r[:, None] ** l * np.exp(-alphas[None, :] * r[:, None] ** 2)
    cn = (2 * alphas / np.pi) ** 0.75 * (4 * alphas) ** (l / 2)   # primitive norms
    A = (G * cn[None, :]) * np.sqrt(w)[:, None]
    c, *_ = np.linalg.lstsq(A, target * np.sqrt(w), rcond=None)
    return c


def ccpvdz_shaped(sym):
    """Synthetic basis with cc-pVDZ's shape for ``sym`` (PySCF format).

    Contractions are least-squares fits to Slater-type orbitals (1s; 2s, 2p
    with Slater's-rules exponents) over even-tempered primitives, the way
    STO-nG sets are built; the uncontracted diffuse and polarisation
    functions follow cc-pVDZ's layout."""
    z1, z2 = _SLATER[sym]
    if z2 is None:
        s_exp = _even_tempered(18.0 * z1 ** 2, 5.2, 3)
        s_cof = _sto_fit(s_exp, z1, 1, 0)
        return [
            [0] + [[float(a), float(c)] for a, c in zip(s_exp, s_cof)],
            [0, [float(0.08 * z1 ** 2), 1.0]],
            [1, [_POL[sym], 1.0]],
        ]
    n_s = 9 if ELEMENT_Z[sym] >= 5 else 8
    a_max = 220.0 * z1 ** 2
    a_min = 0.09 * z2 ** 2
    ratio = (a_max / a_min) ** (1.0 / (n_s - 1))
    s_exp = _even_tempered(a_max, ratio, n_s)
    c1 = _sto_fit(s_exp, z1, 1, 0)
    c2 = _sto_fit(s_exp, z2, 2, 0)
    s_entry = [0] + [[float(a), float(x), float(y)] for a, x, y in zip(s_exp, c1, c2)]
    p_exp = _even_tempered(6.0 * z2 ** 2, 4.2, 3)
    p_cof = _sto_fit(p_exp, z2, 2, 1)
    p_entry = [1] + [[float(a), float(c)] for a, c in zip(p_exp, p_cof)]
    return [
        s_entry,
        [0, [float(0.05 * z2 ** 2), 1.0]],
        p_entry,
        [1, [float(0.055 * z2 ** 2), 1.0]],
        [2, [_POL[sym], 1.0]],
    ]


def _water(origin, rot):
    """H2O at the reference geometry O-H 1.809 bohr, HOH 104.5 deg."""
    r = 1.809
    th = np.deg2rad(104.5) / 2
    loc = np.array([[0.0, 0.0, 0.0],
                    [r * np.sin(th), 0.0, r * np.cos(th)],
                    [-r * np.sin(th), 0.0, r * np.cos(th)]])
    return [("O", tuple(origin + rot @ loc[0])),
            ("H", tuple(origin + rot @ loc[1])),
            ("H", tuple(origin + rot @ loc[2]))]


def _rot(axis, deg):
    a = np.deg2rad(deg)
    c, s = np.cos(a), np.sin(a)
    if axis == "x":
        return np.array([[1, 0, 0], [0, c, -s], [0, s, c]])
    if axis == "y":
        return np.array([[c, 0, s], [0, 1, 0], [-s, 0, c]])
    return np.array([[c, -s, 0], [s, c, 0], [0, 0, 1]])


NAMED_SYSTEMS = ("H2", "LiH", "H2O", "N2", "H2O_dimer")


def named_system(name):
    """``Mole`` of a named system (bohr)."""
    if name == "H2":
        atoms = [("H", (0.0, 0.0, -0.7)), ("H", (0.0, 0.0, 0.7))]
        basis = {"H": sto3g_h()}
        label = "sto-3g"
    elif name == "LiH":
        atoms = [("Li", (0.0, 0.0, 0.0)), ("H", (0.0, 0.0, 3.015))]
        basis = {"Li": ccpvdz_shaped("Li"), "H": ccpvdz_shaped("H")}
        label = "cc-pvdz-shaped"
    elif name == "H2O":
        atoms = _water(np.zeros(3), np.eye(3))
        basis = {"O": ccpvdz_shaped("O"), "H": ccpvdz_shaped("H")}
        label = "cc-pvdz-shaped"
    elif name == "N2":
        atoms = [("N", (0.0, 0.0, -1.034)), ("N", (0.0, 0.0, 1.034))]
        basis = {"N": ccpvdz_shaped("N")}
        label = "cc-pvdz-shaped"
    elif name == "H2O_dimer":
        d = 3.0 * ANG_TO_BOHR
        w1 = _water(np.zeros(3), _rot("y", 90.0))
        w2 = _water(np.array([d, 0.0, 0.0]), _rot("x", 60.0) @ _rot("y", -55.0))
        atoms = w1 + w2
        basis = {"O": ccpvdz_shaped("O"), "H": ccpvdz_shaped("H")}
        label = "cc-pvdz-shaped"
    else:
        raise KeyError(f"unknown system {name!r}; known: {NAMED_SYSTEMS}")
    return Mole(atoms, basis, unit="Bohr", basis_name=label)


def seeded_mo_coeff(mol, seed=0, mix=0.08):
    """Seeded occupied MOs (nao, nocc) for ``mol`` (see module docstring)."""
    shells = build_shells(mol)
    nbf = shells[-1].isgs + shells[-1].nsgs
    nocc = mol.tot_electrons() // 2
    rng = np.random.default_rng(seed)
    if mol.natm == 2 and nbf == 2 and nocc == 1:
        return np.array([[1.0], [1.0]]) / np.sqrt(2.0)
    Z = mol.atom_charges()
    # candidate dominant AOs: (priority, ao index)
    cand = []
    for sh in shells:
        z = Z[sh.iat]
        if sh.am == 0:
            pri = (0 if (sh.entry == 0 and sh.column == 0 and z > 2) else
                   1 if sh.entry == 0 else 2) - 0.01 * z
            cand.append((pri, sh.isgs))
        elif sh.am == 1 and sh.entry <= 2:
            for k in range(3):
                cand.append((2.5 - 0.01 * z + 0.001 * k, sh.isgs + k))
    cand.sort()
    C = mix * rng.standard_normal((nbf, nocc))
    used = set()
    m = 0
    for _, ao in cand:
        if m == nocc:
            break
        if ao in used:
            continue
        used.add(ao)
        C[ao, m] += 1.0
        m += 1
    if m < nocc:
        raise ValueError("not enough candidate AOs for the occupied space")
    return C


def default_params_corr(mol, cusp=False, j1=True):
    """Padé Jastrow parameters.

    J2 satisfies the e-e cusp (like 0.25, unlike 0.5) with b = 1.0.  With
    ``j1``, J1 is ``b = 1.0`` per element (``a = -Z`` implied without cusp
    correction) or ``[-0.05, 1.0]`` with it."""
    out = {"J2_pade": {"like": np.array([0.25, 1.0]),
                       "unlike": np.array([0.5, 1.0])}}
    if j1:
        out["J1_pade"] = {s: (np.array([-0.05, 1.0]) if cusp else np.array(1.0))
                          for s in set(mol.elements)}
    return out


def benchmark_params_corr(mol):
    """Jastrow of the benchmark trial: Padé J2 (cusp a = 0.25 / 0.5, b = 3).

    With Gaussian orbitals that already fit the 1s shape, the cusp-free J1
    (a = -Z) counts the nuclear cusp twice and raises the local-energy
    variance of H2O from about 90 to several thousand hartree^2; among
    J2-only trials b = 3 gave the lowest variance (85 hartree^2)."""
    return {"J2_pade": {"like": np.array([0.25, 3.0]), "unlike": np.array([0.5, 3.0])}}


def synthetic_cusp_params(mol, seed=3):
    """Seeded cusp constants ``{sym: {"q0", "coeff"(8)}}``.

    The reference fits these per element and basis (``psi/cusp.py:25-93``);
    evaluation parity does not depend on their values, so tests use seeded
    ones of realistic size."""
    rng = np.random.default_rng(seed)
    out = {}
    for s in sorted(set(mol.elements)):
        coeff = np.concatenate([[1.0, 1.0], 0.3 * rng.standard_normal(6)])
        out[s] = {"q0": float(0.5 + rng.random()), "coeff": coeff}
    return out


_RHF_CACHE = {}


def make_mf(name, mos="rhf", seed=0):
    """Mean-field object of a named system: RHF orbitals (``mos="rhf"``)
    or seeded non-SCF orbitals (``mos="seeded"``)."""
    mol = named_system(name)
    if mos == "seeded":
        return MeanField(mol, seeded_mo_coeff(mol, seed=seed))
    if name not in _RHF_CACHE:
        from .rhf import run_rhf
        _RHF_CACHE[name] = run_rhf(mol)
    mf = _RHF_CACHE[name]
    return MeanField(mol, mf.mo_coeff, mf.mo_occ)
