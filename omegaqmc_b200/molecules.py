"""The named benchmark systems and their synthetic basis sets.

No quantum-chemistry package is available to this project, so the basis
sets of the named systems are generated here:

* ``sto3g_h`` uses the hydrogen STO-3G-shaped primitives that the
  reference's own tests carry (``tests/test_gto_kinetic_energy.py:677-683``).
* ``ccpvdz_shaped(sym)`` is a *shape-matched synthetic* basis: the same
  angular momenta, number of basis entries, contraction depths and general
  contraction layout as cc-pVDZ (H: 2s1p = 5 functions; Li-Ne: 3s2p1d = 14
  functions, the core s entry a two-column general contraction), with
  exponents and coefficients from a deterministic even-tempered rule.  The
  function counts (LiH 19, H2O 24, N2 28, (H2O)2 48) and the per-position
  exponential counts therefore match the real basis; absolute energies do
  not match literature values.

Occupied MO coefficients are seeded (``seeded_mo_coeff``): an aufbau-like
choice of one dominant AO per occupied orbital plus a seeded admixture of
all AOs, or, for H2, the symmetric bonding combination (which is the RHF
orbital of a two-function homonuclear basis).
"""
from __future__ import annotations

import numpy as np

from .system import Mole, MeanField, ELEMENT_Z, build_shells, ANG_TO_BOHR

__all__ = ["sto3g_h", "ccpvdz_shaped", "named_system", "NAMED_SYSTEMS",
           "seeded_mo_coeff", "default_params_corr", "synthetic_cusp_params"]


def sto3g_h():
    """STO-3G-shaped H 1s (the reference tests' primitive data)."""
    return [[0, [3.42525091, 0.15432897], [0.62391373, 0.53532814],
             [0.16885540, 0.44463454]]]


def _even_tempered(a_max, ratio, n):
    return a_max / ratio ** np.arange(n)


def ccpvdz_shaped(sym):
    """Synthetic basis with cc-pVDZ's shape for ``sym`` (PySCF format)."""
    Z = ELEMENT_Z[sym]
    if Z <= 2:
        s_exp = _even_tempered(10.0 * Z ** 2, 4.6, 3)
        s_cof = np.array([0.03, 0.20, 0.55])
        return [
            [0] + [[a, c] for a, c in zip(s_exp, s_cof)],
            [0, [0.14 * Z, 1.0]],
            [1, [0.8 * Z, 1.0]],
        ]
    # first row: 9-primitive s general contraction with two columns
    n_s = 9 if Z >= 5 else 8
    a_max = 1500.0 * Z ** 1.5
    s_exp = _even_tempered(a_max, 3.55, n_s)
    x = np.arange(n_s) / (n_s - 1)
    core = np.exp(-((x - 0.62) / 0.22) ** 2)
    core[-1] *= -0.1
    val = -0.45 * np.exp(-((x - 0.6) / 0.2) ** 2)
    val[-2:] = [0.55, 0.60]
    s_entry = [0] + [[a, c1, c2] for a, c1, c2 in zip(s_exp, core, val)]
    p_exp = _even_tempered(2.2 * Z, 4.3, 3)
    p_entry = [1] + [[a, c] for a, c in zip(p_exp, [0.05, 0.25, 0.55])]
    return [
        s_entry,
        [0, [0.038 * Z, 1.0]],
        p_entry,
        [1, [0.034 * Z, 1.0]],
        [2, [0.15 * Z, 1.0]],
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


def default_params_corr(mol, cusp=False):
    """Padé Jastrow parameters used by the benchmarks.

    J2 satisfies the e-e cusp (like 0.25, unlike 0.5) with b = 1.0; J1 is
    ``b = 1.0`` per element (``a = -Z`` implied without cusp correction)."""
    j1 = {}
    for s in set(mol.elements):
        j1[s] = np.array([-0.05, 1.0]) if cusp else np.array(1.0)
    return {"J1_pade": j1,
            "J2_pade": {"like": np.array([0.25, 1.0]),
                        "unlike": np.array([0.5, 1.0])}}


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


def make_mf(name, seed=0):
    mol = named_system(name)
    return MeanField(mol, seeded_mo_coeff(mol, seed=seed))
