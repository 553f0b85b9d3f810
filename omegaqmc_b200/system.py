"""Molecular system description for the GTO Slater–Jastrow wavefunction.

This module turns a PySCF-style mean-field object (or the light-weight
:class:`Mole` / :class:`MeanField` stand-ins defined here) into the flat
tables the CUDA kernels read: nuclei, contracted shells with normalised
primitive coefficients, occupied MO coefficients, Padé Jastrow parameters
and cusp-correction constants.

Conventions follow the reference trial wavefunction:

* Shell normalisation restates ``read_shell`` (``OmegaQMC/psi/shell.py:150-256``):
  s and p contractions are renormalised over the contraction, d/f/g shells
  carry primitive normalisation only.  A general contraction (several
  coefficient columns sharing one exponent list) becomes one shell per column.
* The cusp-corrected shell of each atom is the first coefficient column of
  the atom's first basis entry (``OmegaQMC/psi/gto.py:890-913``), with
  ``rc = 0.1`` for hydrogen and ``0.2`` otherwise (``gto.py:873-876``).
* Spherical AO order within a shell is that of ``_angular_cartesian``
  (``gto.py:607-671``); AOs are numbered atom by atom, entry by entry,
  column by column.
* Electrons alternate spin: up at even, down at odd positions
  (``OmegaQMC/spin_layout.py:56-80``); only closed shells (n_up == n_down)
  are supported, as in the reference's single-determinant path
  (``gto.py:846-888`` takes one ``mo_coeff[:, :nocc]`` for both spins).
* Padé J1 without cusp correction fixes ``a = -Z`` (``gto.py:1526-1560``).
"""
from __future__ import annotations

import math
import warnings
from dataclasses import dataclass, field

import numpy as np

__all__ = [
    "Mole", "MeanField", "Shell", "System", "read_shell", "build_system",
    "ELEMENT_Z", "parse_params_corr",
]

ELEMENT_Z = {
    "H": 1, "He": 2, "Li": 3, "Be": 4, "B": 5, "C": 6, "N": 7, "O": 8,
    "F": 9, "Ne": 10, "Na": 11, "Mg": 12, "Al": 13, "Si": 14, "P": 15,
    "S": 16, "Cl": 17, "Ar": 18,
}
ANG_TO_BOHR = 1.0 / 0.52917721092
PI32 = math.pi ** 1.5


# --------------------------------------------------------------------------
# Duck-typed PySCF objects
# --------------------------------------------------------------------------
class Mole:
    """Minimal stand-in for ``pyscf.gto.Mole`` as read by the GTO path.

    Only the attributes the reference's trial wavefunction touches are
    provided: ``_atom``, ``_basis``, ``atom_coords``, ``atom_charges``,
    ``atom_symbol``, ``natm``, ``tot_electrons``, ``nelec``, ``basis``,
    ``charge``, ``spin``, ``elements`` and ``groupname``.

    Args:
        atoms: ``[(symbol, (x, y, z)), ...]`` or a PySCF-style string
            ``"O 0 0 0; H 0 0 1.8"``.
        basis: ``{symbol: [[am, [alpha, c1, c2, ...], ...], ...]}`` in
            PySCF's internal (``mol._basis``) format.
        unit: ``"Bohr"`` (default) or ``"Angstrom"``.
        basis_name: label stored in ``mol.basis``.
    """

    def __init__(self, atoms, basis, unit="Bohr", charge=0, spin=0,
                 basis_name="gen"):
        if isinstance(atoms, str):
            atoms = _parse_atom_string(atoms)
        u = unit.lower()
        if u in ("bohr", "au", "a.u."):
            fac = 1.0
        elif u in ("angstrom", "ang", "a"):
            fac = ANG_TO_BOHR
        else:
            raise ValueError(f"unknown unit {unit!r}")
        self._atom = [(str(s), tuple(float(c) * fac for c in xyz))
                      for s, xyz in atoms]
        for s, _ in self._atom:
            if s not in ELEMENT_Z:
                raise ValueError(f"unknown element {s!r}")
            if s not in basis:
                raise ValueError(f"no basis given for element {s!r}")
        self._basis = {s: basis[s] for s, _ in self._atom}
        self.basis = basis_name
        self.charge = int(charge)
        self.spin = int(spin)
        self.unit = "Bohr"
        self.groupname = "C1"

    @property
    def natm(self):
        return len(self._atom)

    @property
    def elements(self):
        return [s for s, _ in self._atom]

    def atom_symbol(self, i):
        return self._atom[i][0]

    def atom_coords(self, unit="Bohr"):
        c = np.array([xyz for _, xyz in self._atom], dtype=np.float64)
        if unit.lower() in ("angstrom", "ang"):
            c = c / ANG_TO_BOHR
        return c

    def atom_charges(self):
        return np.array([ELEMENT_Z[s] for s, _ in self._atom], dtype=np.int64)

    def tot_electrons(self):
        return int(self.atom_charges().sum()) - self.charge

    @property
    def nelec(self):
        n = self.tot_electrons()
        nb = (n - self.spin) // 2
        return (n - nb, nb)

    @property
    def nao(self):
        return sum(s.nsgs for s in build_shells(self))


class MeanField:
    """Minimal stand-in for a converged ``pyscf.scf.RHF`` object.

    ``mo_coeff`` is ``(nao, nmo)`` over the spherical AOs in the order of
    :func:`build_shells`; ``mo_occ`` marks occupied columns with 2.
    """

    def __init__(self, mol, mo_coeff, mo_occ=None):
        self.mol = mol
        self.mo_coeff = np.asarray(mo_coeff, dtype=np.float64)
        if mo_occ is None:
            nocc = mol.tot_electrons() // 2
            mo_occ = np.zeros(self.mo_coeff.shape[1])
            mo_occ[:nocc] = 2.0
        self.mo_occ = np.asarray(mo_occ, dtype=np.float64)


def _parse_atom_string(s):
    out = []
    for line in s.replace(";", "\n").splitlines():
        line = line.strip()
        if not line:
            continue
        parts = line.split()
        out.append((parts[0], tuple(float(p) for p in parts[1:4])))
    return out


# --------------------------------------------------------------------------
# Shells
# --------------------------------------------------------------------------
@dataclass
class Shell:
    """One contracted shell (one coefficient column of a basis entry).

    Mirrors ``ShellType`` (``OmegaQMC/psi/shell.py:8-31``)."""
    am: int
    iat: int
    isgs: int
    nsgs: int
    alpha: np.ndarray
    norm: np.ndarray
    is_cusp: bool = False
    entry: int = 0          # index of the basis entry on its atom
    column: int = 0         # contraction column within the entry

    @property
    def nprim(self):
        return len(self.alpha)


_NSGS = {0: 1, 1: 3, 2: 5, 3: 7, 4: 9}


def read_shell(entry, iat, isgs):
    """Normalised shells of one PySCF basis entry ``[am, [a, c...], ...]``.

    Restates ``read_shell`` (``OmegaQMC/psi/shell.py:150-256``): primitive
    factor ``(2a/pi)^(3/4)`` times ``sqrt(4a)`` (p), ``4a/sqrt(3)`` (d),
    ``(4a)^(3/2)/sqrt(15)`` (f), ``(4a)^2/sqrt(105)`` (g); s and p shells are
    then renormalised over the contraction (``shell.py:180-218``).
    """
    am = int(entry[0])
    rows = entry[1:]
    if rows and not isinstance(rows[0], (list, tuple, np.ndarray)):
        # PySCF may carry a kappa scalar after am; it does not change
        # the non-relativistic shell.
        rows = rows[1:]
    prim = np.array(rows, dtype=np.float64)
    if prim.ndim != 2 or prim.shape[1] < 2:
        raise ValueError(f"bad basis entry {entry!r}")
    if am not in _NSGS:
        raise NotImplementedError(f"Angular momentum {am} not yet implemented")
    alphas = prim[:, 0]
    out = []
    cnorm0 = np.exp(0.75 * np.log(2.0 * alphas / np.pi))
    iu, ju = np.triu_indices(len(alphas), k=0)
    diag = iu == ju
    for ic in range(1, prim.shape[1]):
        c = prim[:, ic]
        if am == 0:
            norm = c * cnorm0
            asum = alphas[iu] + alphas[ju]
            terms = norm[iu] * norm[ju] / (asum * np.sqrt(asum))
            terms = np.where(diag, terms, 2.0 * terms)
            norm = norm * (1.0 / np.sqrt(np.sum(terms) * PI32))
        elif am == 1:
            norm = c * cnorm0 * np.sqrt(4.0 * alphas)
            asum = alphas[iu] + alphas[ju]
            terms = 0.5 * norm[iu] * norm[ju] / (asum * asum * np.sqrt(asum))
            terms = np.where(diag, terms, 2.0 * terms)
            norm = norm * (1.0 / np.sqrt(np.sum(terms) * PI32))
        elif am == 2:
            norm = c * cnorm0 * (4.0 * alphas) / np.sqrt(3.0)
        elif am == 3:
            norm = c * cnorm0 * (4.0 * alphas) ** 1.5 / np.sqrt(15.0)
        else:
            norm = c * cnorm0 * (4.0 * alphas) ** 2 / np.sqrt(105.0)
        out.append(Shell(am=am, iat=iat, isgs=isgs, nsgs=_NSGS[am],
                         alpha=alphas.copy(), norm=np.asarray(norm),
                         column=ic - 1))
        isgs += _NSGS[am]
    return out


def build_shells(mol, cusp=False):
    """All shells of ``mol`` in AO order (``gto.py:890-913``)."""
    shells = []
    isgs = 0
    for ia, (sym, _) in enumerate(mol._atom):
        for ish, entry in enumerate(mol._basis[sym]):
            for jsh, sh in enumerate(read_shell(entry, ia, isgs)):
                sh.entry = ish
                sh.is_cusp = bool(cusp and ish == 0 and jsh == 0)
                isgs = sh.isgs + sh.nsgs
                shells.append(sh)
    return shells


# --------------------------------------------------------------------------
# Jastrow parameters
# --------------------------------------------------------------------------
def parse_params_corr(params_corr, mol, cusp):
    """Per-atom Padé J1 ``(a, b)`` and J2 like/unlike ``(a, b)``.

    Returns ``(has_j1, j1_ab (natm, 2), has_j2, j2 (2, 2))`` where ``j2[0]``
    is the like-spin pair and ``j2[1]`` the unlike-spin pair.  Restates
    ``J1_ab`` (``gto.py:1526-1560``): with cusp-corrected orbitals each
    element carries ``[a, b]``; without them ``a = -Z`` and the entry is
    ``b`` (an ``[a, b]`` entry warns and its ``a`` is ignored; any other
    length raises ``ValueError``).  Keys other than ``J1_pade`` and
    ``J2_pade`` and the B-spline / J3_eeI terms (parsed by
    :func:`parse_bspline` and :func:`parse_j3`) raise
    ``NotImplementedError``.
    """
    params_corr = {} if params_corr is None else dict(params_corr)
    extra = [k for k in params_corr
             if k not in ("J1_pade", "J2_pade", "J1_bspline", "J2_bspline", "J3_eeI")]
    if extra:
        raise NotImplementedError(
            f"Jastrow terms {extra} are not supported; J1/J2 Padé, B-spline "
            "and J3_eeI terms are implemented on this path")
    natm = mol.natm
    Z = mol.atom_charges().astype(np.float64)
    j1 = np.zeros((natm, 2))
    has_j1 = "J1_pade" in params_corr and len(params_corr["J1_pade"]) > 0
    if has_j1:
        p1 = params_corr["J1_pade"]
        for ia in range(natm):
            sym = mol.atom_symbol(ia)
            if sym not in p1:
                raise KeyError(f"J1_pade has no entry for element {sym!r}")
            p = np.ravel(np.asarray(p1[sym], dtype=np.float64))
            if cusp:
                if p.shape[0] != 2:
                    raise ValueError(
                        f"J1_pade['{sym}'] must be [a, b] with cusp-"
                        "corrected orbitals")
                j1[ia] = p
            else:
                if p.shape[0] not in (1, 2):
                    raise ValueError(
                        f"J1_pade['{sym}'] has {p.shape[0]} entries; "
                        "expected b or [a, b].")
                if p.shape[0] == 2:
                    warnings.warn(
                        f"J1_pade['{sym}'] = [a, b] without cusp correction:"
                        " a is fixed at -Z and the given a is ignored.  "
                        "Pass b alone.", stacklevel=3)
                j1[ia] = (-Z[ia], p[-1])
    j2 = np.zeros((2, 2))
    has_j2 = "J2_pade" in params_corr
    if has_j2:
        p2 = params_corr["J2_pade"]
        if not isinstance(p2, dict):
            raise TypeError("J2_pade must be a dict with 'like' and 'unlike'")
        for k, key in enumerate(("like", "unlike")):
            v = np.ravel(np.asarray(p2[key], dtype=np.float64))
            if v.shape[0] < 2:
                raise ValueError(f"J2_pade['{key}'] needs [a, b]")
            j2[k] = v[:2]
    return has_j1, j1, has_j2, j2


# ---------------------------------------------------------------------------
# Three-body electron-electron-nucleus Jastrow (J3_eeI)
# ---------------------------------------------------------------------------
J3_DEFAULT = {"N_eI": 3, "N_ee": 3, "r_cut": 5.0}     # _parse_eeI_cfg, gto.py:970-984
J3_MAX_ORDER = 6


def eeI_num_params(n_eI, n_ee):
    """Free parameters of one J3_eeI polynomial block: unique gammas
    (symmetric in the two electron-nucleus orders) minus the no-cusp
    constraints (``_compute_eeI_num_params``, gto.py:243-251)."""
    n_gamma = (n_eI + 1) * (n_eI + 2) // 2 * (n_ee + 1)
    return n_gamma - ((2 * n_eI + 1) + (n_eI + n_ee + 1))


def eeI_constraint_map(n_eI, n_ee, r_cut):
    """Linear map from the free J3_eeI parameters to the unique gammas.

    Returns ``(A, lmn)``: ``gamma_unique = A @ free`` and ``lmn[k]`` the
    (l, m, n) powers of unique gamma k (l >= m; gamma(l, m, n) =
    gamma(m, l, n)).  The constraints make the polynomial cusp-free at
    r_ee = 0 and at r_eI = 0 given the (r_eI - L)^3 envelope; the free
    parameters are the columns left without a pivot when the constraint
    matrix is row-reduced with partial pivoting (QMCPACK
    PolynomialFunctor3D; the same rows, pivot rule and 1e-6 threshold as
    ``_build_eeI_constraint_map``, gto.py:321-463, so that the same
    parameter vector means the same gammas).
    """
    if n_ee < 1:
        raise ValueError("J3_eeI needs N_ee >= 1 (the e-e cusp row uses n = 1)")
    half = 0.5 * r_cut
    cont = 3.0                                  # envelope continuity order
    lmn = [(l, m, n) for m in range(n_eI + 1) for l in range(m, n_eI + 1)
           for n in range(n_ee + 1)]
    slot = {}
    for k, (l, m, n) in enumerate(lmn):
        slot[(l, m, n)] = k
        slot[(m, l, n)] = k
    ng = len(lmn)
    nrow = (2 * n_eI + 1) + (n_eI + n_ee + 1)
    K = np.zeros((nrow, ng))
    # r_ee cusp: the n = 1 gammas of each total order l + m
    for tot in range(2 * n_eI + 1):
        for m in range(tot + 1):
            l = tot - m
            if l <= n_eI and m <= n_eI and l >= m:
                K[tot, slot[(l, m, 1)]] = 2.0 if l > m else 1.0
    # r_eI cusp: one row per order l + n of the electron at the nucleus
    base = 2 * n_eI + 1
    for tot in range(n_eI + n_ee + 1):
        if tot <= n_ee:
            K[base + tot, slot[(0, 0, tot)]] = cont
            if n_eI >= 1:
                K[base + tot, slot[(0, 1, tot)]] = -half
        for l in range(1, tot + 1):
            n = tot - l
            if 0 <= n <= n_ee and l <= n_eI:
                K[base + tot, slot[(l, 0, n)]] = cont
                if n_eI >= 1:
                    K[base + tot, slot[(l, 1, n)]] = -half
    free = np.zeros(ng, dtype=bool)
    col = -1
    for row in range(nrow):
        col += 1
        while col < ng:
            piv = row + int(np.argmax(np.abs(K[row:, col])))
            if abs(K[piv, col]) >= 1e-6:
                break
            free[col] = True
            col += 1
        if col >= ng:
            break
        K[[row, piv]] = K[[piv, row]]
        K[row] /= K[row, col]
        f = K[:, col].copy()
        f[row] = 0.0
        K -= f[:, None] * K[row][None, :]
    free[col + 1:] = True
    fcols = np.flatnonzero(free)
    dcols = np.flatnonzero(~free)
    if fcols.size != eeI_num_params(n_eI, n_ee):
        raise ValueError("J3_eeI constraint system is rank deficient")
    A = np.zeros((ng, fcols.size))
    A[fcols, np.arange(fcols.size)] = 1.0
    for r, dc in enumerate(dcols):
        A[dc] = -K[r, fcols]
    return A, lmn


def eeI_gamma(params, n_eI, n_ee, r_cut):
    """Full symmetric gamma array (n_eI+1, n_eI+1, n_ee+1) of one block
    from its free parameters (``_vec_to_gamma_3d``, gto.py:466-478)."""
    A, lmn = eeI_constraint_map(n_eI, n_ee, r_cut)
    vec = A @ np.asarray(params, dtype=np.float64)
    g = np.zeros((n_eI + 1, n_eI + 1, n_ee + 1))
    for k, (l, m, n) in enumerate(lmn):
        g[l, m, n] = vec[k]
        g[m, l, n] = vec[k]
    return g


def parse_j3(params_corr, mol, jastrow_config=None):
    """J3_eeI tables, or None without a ``J3_eeI`` entry.

    ``params_corr["J3_eeI"]`` maps ``"like+<sym>"`` / ``"unlike+<sym>"`` to
    free-parameter vectors (same-spin and opposite-spin electron pairs
    around nuclei of element ``sym``).  Orders and cutoff come from
    ``jastrow_config["J3"]`` (``N_eI``, ``N_ee``, ``r_cut``; defaults 3, 3,
    5.0 bohr, gto.py:970-984).  Validation follows the driver
    (vmc_gto.py:595-611: a non-dict raises ``TypeError``, a key without the
    prefix ``ValueError``) and ``_sanitize_J3_eeI_params`` (gto.py:254-306:
    an entry that is not a 1-D vector of the right length warns and becomes
    zeros; the length is checked against the configured orders).  Keys of
    elements absent from the molecule are ignored, as in ``J3_eeI_fn``
    (gto.py:2011-2035), which sums over the molecule's elements.

    Returns ``{"n_eI", "n_ee", "r_cut", "types": per-atom type (-1 none),
    "elements": symbol per type, "gamma": (ntype, 2, n_eI+1, n_eI+1,
    n_ee+1) with block 0 like and 1 unlike, "on": (ntype, 2) flags,
    "params": the sanitised dict}``.
    """
    if not params_corr or "J3_eeI" not in params_corr:
        return None
    v = params_corr["J3_eeI"]
    if not isinstance(v, dict):
        raise TypeError(f"J3_eeI params must be a dict, got {type(v)}")
    for k in v:
        if not (k.startswith("like+") or k.startswith("unlike+")):
            raise ValueError(f"J3_eeI sub-key '{k}' must start with 'like+' or 'unlike+'")
    cfg = dict(J3_DEFAULT)
    if jastrow_config is not None and "J3" in jastrow_config:
        j = jastrow_config["J3"]
        for k in ("N_eI", "N_ee"):
            if k in j:
                cfg[k] = int(j[k])
        if "r_cut" in j:
            cfg["r_cut"] = float(j["r_cut"])
    n_eI, n_ee, r_cut = cfg["N_eI"], cfg["N_ee"], cfg["r_cut"]
    if not (0 <= n_eI <= J3_MAX_ORDER and 1 <= n_ee <= J3_MAX_ORDER):
        raise ValueError(f"J3 orders N_eI={n_eI}, N_ee={n_ee} out of range "
                         f"(0..{J3_MAX_ORDER}, 1..{J3_MAX_ORDER})")
    if not r_cut > 0.0:
        raise ValueError("J3 r_cut must be positive")
    npar = eeI_num_params(n_eI, n_ee)
    clean = {}
    for k, val in v.items():
        try:
            arr = np.asarray(val, dtype=np.float64)
        except Exception:
            warnings.warn(f"J3_eeI['{k}']: cannot convert to array; replacing with zeros",
                          stacklevel=3)
            clean[k] = np.zeros(npar)
            continue
        if arr.ndim != 1:
            warnings.warn(f"J3_eeI['{k}']: expected 1-D array, got ndim={arr.ndim}; "
                          "replacing with zeros", stacklevel=3)
            clean[k] = np.zeros(npar)
        elif arr.shape[0] != npar:
            warnings.warn(f"J3_eeI['{k}']: expected {npar} params (for N_eI={n_eI}, "
                          f"N_ee={n_ee}), got {arr.shape[0]}; replacing with zeros",
                          stacklevel=3)
            clean[k] = np.zeros(npar)
        else:
            clean[k] = arr.copy()
    elements = []
    for ia in range(mol.natm):
        sym = mol.atom_symbol(ia)
        if sym not in elements and ("like+" + sym in clean or "unlike+" + sym in clean):
            elements.append(sym)
    if not elements:
        return None
    types = [elements.index(mol.atom_symbol(ia)) if mol.atom_symbol(ia) in elements else -1
             for ia in range(mol.natm)]
    gamma = np.zeros((len(elements), 2, n_eI + 1, n_eI + 1, n_ee + 1))
    on = np.zeros((len(elements), 2), dtype=np.int32)
    for t, sym in enumerate(elements):
        for b, prefix in enumerate(("like+", "unlike+")):
            if prefix + sym in clean:
                gamma[t, b] = eeI_gamma(clean[prefix + sym], n_eI, n_ee, r_cut)
                on[t, b] = 1
    return {"n_eI": n_eI, "n_ee": n_ee, "r_cut": r_cut, "types": types,
            "elements": elements, "gamma": gamma, "on": on, "params": clean}


def bspline_coefs(params, delta_r, cusp_val):
    """Full coefficient vector (N + 4) of a cubic B-spline Jastrow term from
    its N parameters: c[1..N] = params, c[0] = params[1] - 2 dr cusp (the
    cusp condition u'(0) = cusp), c[N+1..N+3] = 0 (u, u', u'' vanish at the
    cutoff).  Restates _build_bspline_coefs (``gto.py:18-33``)."""
    p = np.ravel(np.asarray(params, dtype=np.float64))
    return np.concatenate([[p[1] - 2.0 * delta_r * cusp_val], p, np.zeros(3)])


def parse_bspline(params_corr, mol, cusp, jastrow_config=None):
    """B-spline J1/J2 tables ``(bs2, bs1)``.

    ``bs2``: None or ``{"like": coefs, "unlike": coefs, "r_cut": r}`` with the
    Kato cusps 1/4 (like) and 1/2 (unlike) built into the coefficients;
    ``bs1``: None or a per-atom list of ``(coefs, r_cut)`` (None for atoms
    whose element has no one-body spline), cusp value 0 with cusp-corrected
    orbitals and -Z without (``gto.py:1657-1931``).  Cutoffs come from
    ``jastrow_config`` (``{"J2": {"r_cut": r}, "J1": {sym: {"r_cut": r}}}``;
    10 bohr for every term when it is None, ``gto.py:948-968``).  Entries
    need at least 2 parameters (``ValueError``, ``vmc_gto.py:580-592``);
    Padé and B-spline terms of the same body are summed with a warning
    (``vmc_gto.py:609-617``)."""
    params_corr = {} if params_corr is None else params_corr
    for key in ("J1_bspline", "J2_bspline"):
        if key not in params_corr:
            continue
        v = params_corr[key]
        if not isinstance(v, dict):
            raise TypeError(f"{key} must be a dict, got {type(v)}")
        for sk, sv in v.items():
            if np.ravel(np.asarray(sv)).shape[0] < 2:
                raise ValueError(f"{key}['{sk}'] must have >= 2 coefficients")
    for body in ("J1", "J2"):
        if f"{body}_pade" in params_corr and f"{body}_bspline" in params_corr:
            warnings.warn(f"Both {body}_pade and {body}_bspline are present; "
                          "their contributions will be summed.", stacklevel=3)
    bs2 = None
    if "J2_bspline" in params_corr:
        if jastrow_config is None:
            rc2 = 10.0
        elif "J2" in jastrow_config:
            rc2 = float(jastrow_config["J2"]["r_cut"])
        else:
            raise ValueError("J2_bspline needs jastrow_config['J2']['r_cut']")
        p2 = params_corr["J2_bspline"]
        bs2 = {"r_cut": rc2}
        for key, cv in (("like", 0.25), ("unlike", 0.5)):
            p = np.ravel(np.asarray(p2[key], dtype=np.float64))
            bs2[key] = bspline_coefs(p, rc2 / (p.shape[0] + 1), cv)
    bs1 = None
    if "J1_bspline" in params_corr:
        p1 = params_corr["J1_bspline"]
        Z = mol.atom_charges().astype(np.float64)
        bs1 = []
        for ia in range(mol.natm):
            sym = mol.atom_symbol(ia)
            if jastrow_config is None:
                rc1 = 10.0
            elif "J1" in jastrow_config and sym in jastrow_config["J1"]:
                rc1 = float(jastrow_config["J1"][sym]["r_cut"])
            else:
                bs1.append(None)
                continue
            p = np.ravel(np.asarray(p1[sym], dtype=np.float64))
            cv = 0.0 if cusp else -Z[ia]
            bs1.append((bspline_coefs(p, rc1 / (p.shape[0] + 1), cv), rc1))
        if all(b is None for b in bs1):
            bs1 = None
    return bs2, bs1


# --------------------------------------------------------------------------
# Flattened system
# --------------------------------------------------------------------------
@dataclass
class System:
    """Flat, kernel-ready description of one molecule and its trial state.

    Exponent sharing: shells of the same atom and basis entry (the columns
    of a general contraction) share their exponential factors, so the
    kernels evaluate each distinct ``exp(-alpha r^2)`` once per electron
    position (``pgroup``).
    """
    nuc: np.ndarray            # (natm, 3) bohr
    Z: np.ndarray              # (natm,) float
    shells: list
    C: np.ndarray              # (nbf, nocc) occupied MO coefficients
    n_up: int
    n_dn: int
    has_j1: bool
    j1: np.ndarray             # (natm, 2)
    has_j2: bool
    j2: np.ndarray             # (2, 2) like, unlike
    cusp: bool
    cusp_rc: np.ndarray        # (natm,)
    cusp_q0: np.ndarray        # (natm,)
    cusp_coeff: np.ndarray     # (natm, 8)
    symbols: list = field(default_factory=list)
    bs2: object = None         # B-spline J2: {"like", "unlike": coefs, "r_cut"}
    bs1: object = None         # B-spline J1: per atom (coefs, r_cut) or None
    j3: object = None          # J3_eeI tables (see :func:`parse_j3`) or None
    md: object = None          # multi-determinant trial (see :func:`parse_trial`) or None
    spl: object = None         # quintic radial splines (see :func:`ao_spline_tables`) or None

    @property
    def natm(self):
        return self.nuc.shape[0]

    @property
    def nbf(self):
        return self.C.shape[0]

    @property
    def nocc(self):
        return self.C.shape[1]

    @property
    def n_e(self):
        return self.n_up + self.n_dn

    @property
    def e_nn(self):
        """Nuclear repulsion with the reference's eps-softened distance
        (``gto.py:2406-2430``)."""
        eps = np.finfo(np.float64).eps
        e = 0.0
        for i in range(self.natm):
            for j in range(i + 1, self.natm):
                d = self.nuc[i] - self.nuc[j]
                e += self.Z[i] * self.Z[j] / np.sqrt(np.dot(d, d) + eps)
        return float(e)

    def prim_groups(self):
        """Distinct exponent sets: list of (iat, alpha array, [shell ids])."""
        groups = {}
        order = []
        for i, sh in enumerate(self.shells):
            key = (sh.iat, sh.entry)
            if key not in groups:
                groups[key] = (sh.iat, sh.alpha, [])
                order.append(key)
            groups[key][2].append(i)
        return [groups[k] for k in order]

    def n_exp(self):
        """Distinct exponentials per electron position."""
        return sum(len(a) for _, a, _ in self.prim_groups())

    def n_prim_ref(self):
        """Exponentials per position as the reference evaluates them
        (one set per contraction column)."""
        return sum(sh.nprim for sh in self.shells)


def build_quintic_radial_spline(alpha, norm, smin=1.0e-6, tol=1.0e-7, npts=1001,
                                rmax_cap=100.0):
    """Quintic Hermite spline of a contracted radial g(s) = sum_p norm_p
    exp(-alpha_p s) in s = r^2 (QMCPACK's numerical-orbital transform,
    ``_build_quintic_radial_spline``, gto.py:141-198).

    Knots: s = 0 and a log grid from smin to smax = rmax^2, rmax the last
    radius on a 20001-point scan of [0, rmax_cap] where |g| > tol.  Each
    segment is the quintic matching (g, g', g'') at both ends (scipy
    ``BPoly.from_derivatives``, converted to power form ``PPoly``).
    Returns ``(knots (npts,), coefs (npts - 1, 6))``, coefficients of
    segment j in powers of (s - knots[j]), highest first."""
    from scipy.interpolate import BPoly, PPoly
    a = np.asarray(alpha, dtype=np.float64)
    c = np.asarray(norm, dtype=np.float64)

    def derivs(sv):
        sv = np.asarray(sv, dtype=np.float64)
        e = np.exp(-a[None, :] * sv[:, None])
        return np.stack([np.sum(c[None, :] * e, axis=1),
                         np.sum((-a * c)[None, :] * e, axis=1),
                         np.sum((a * a * c)[None, :] * e, axis=1)], axis=1)

    r_scan = np.linspace(0.0, rmax_cap, 20001)
    big = np.abs(derivs(r_scan ** 2)[:, 0]) > tol
    rmax = float(r_scan[np.max(np.nonzero(big))]) if big.any() else 1.0
    smax = max(rmax ** 2, 100.0 * smin)
    grid = np.concatenate([[0.0], np.logspace(np.log10(smin), np.log10(smax), npts - 1)])
    pp = PPoly.from_bernstein_basis(BPoly.from_derivatives(grid, derivs(grid)))
    return np.asarray(pp.x, dtype=np.float64), np.ascontiguousarray(np.asarray(pp.c).T)


def ao_spline_tables(shells, transform):
    """Spline tables of the shells the AO radial transform replaces (every
    shell but the cusp-corrected s ones, gto.py:905-936), or None when
    ``transform`` is falsy.  ``transform`` True uses the default grid; a
    dict overrides ``smin``, ``tol``, ``npts``, ``rmax_cap``.

    Returns ``{"npts", "smin", "tables": {shell index: (knots, coefs)}}``."""
    if not transform:
        return None
    kw = dict(transform) if isinstance(transform, dict) else {}
    unknown = set(kw) - {"smin", "tol", "npts", "rmax_cap"}
    if unknown:
        raise TypeError(f"unknown AO spline options {sorted(unknown)}")
    npts = int(kw.get("npts", 1001))
    if npts < 3:
        raise ValueError("AO spline npts must be at least 3")
    tables = {}
    for i, sh in enumerate(shells):
        if sh.is_cusp:
            continue
        tables[i] = build_quintic_radial_spline(sh.alpha, sh.norm, **kw)
    return {"npts": npts, "smin": float(kw.get("smin", 1.0e-6)), "tables": tables, "cfg": kw}


def parse_trial(trial, n_up, n_dn):
    """Multi-determinant expansion of a ``trial`` dict (``_parse_mol``,
    gto.py:846-863; format of ``OmegaQMC/psi/trial.py``): ``mo_coeff``
    (nao, nmo) for restricted orbitals or (2, nao, nmo) for UHF ones (alpha
    and beta columns side by side, the down occupations shifted by nmo),
    ``ci_coeffs`` (ndet,), ``occ_up`` (ndet, n_up), ``occ_dn`` (ndet, n_dn).

    Returns ``{"C": (nao, ncol), "ci", "occ_up", "occ_dn"}``."""
    def arr(x, dt):
        if torch_like(x):
            x = x.detach().cpu().numpy()
        return np.asarray(x, dtype=dt)

    mo = arr(trial["mo_coeff"], np.float64)
    ci = np.ravel(arr(trial["ci_coeffs"], np.float64))
    occ_up = np.atleast_2d(arr(trial["occ_up"], np.int64))
    occ_dn = np.atleast_2d(arr(trial["occ_dn"], np.int64))
    if mo.ndim == 3:
        if mo.shape[0] != 2:
            raise ValueError("UHF trial mo_coeff must have shape (2, nao, nmo)")
        occ_dn = occ_dn + mo.shape[2]
        mo = np.concatenate(list(mo), axis=1)
    if mo.ndim != 2:
        raise ValueError("trial mo_coeff must have shape (nao, nmo) or (2, nao, nmo)")
    if not (ci.shape[0] == occ_up.shape[0] == occ_dn.shape[0]) or ci.shape[0] < 1:
        raise ValueError("ci_coeffs, occ_up and occ_dn must list the same determinants")
    if occ_up.shape[1] != n_up or occ_dn.shape[1] != n_dn:
        raise ValueError(f"trial occupations have {occ_up.shape[1]} up and {occ_dn.shape[1]} "
                         f"down orbitals, the molecule {n_up} and {n_dn} electrons")
    if occ_up.min() < 0 or occ_dn.min() < 0 or max(occ_up.max(), occ_dn.max()) >= mo.shape[1]:
        raise ValueError("trial occupation index out of range of mo_coeff")
    return {"C": np.ascontiguousarray(mo), "ci": ci, "occ_up": occ_up, "occ_dn": occ_dn}


def torch_like(x):
    return hasattr(x, "detach") and hasattr(x, "cpu")


def build_system(mf, params_corr=None, params_cusp=None, jastrow_config=None, trial=None):
    """Build a :class:`System` from a PySCF-style mean-field object.

    Args:
        mf: object with ``mol`` (see :class:`Mole`), ``mo_coeff`` and
            ``mo_occ``.
        params_corr: Jastrow dict ``{"J1_pade": {sym: b or [a, b]},
            "J2_pade": {"like": [a, b], "unlike": [a, b]}}``.
        params_cusp: ``{sym: {"q0": float, "coeff": (8,)}}`` or None for no
            cusp correction (``gto.py:846-888``).
        jastrow_config: B-spline cutoffs (see :func:`parse_bspline`) and
            the J3_eeI orders and cutoff (see :func:`parse_j3`).
        trial: multi-determinant trial dict (see :func:`parse_trial`); the
            single-determinant orbitals are then the first determinant's up
            orbitals (``mo_occ_coeff``, gto.py:860-862).
    """
    mol = mf.mol
    n_e = mol.tot_electrons()
    n_up, n_dn = mol.nelec
    if n_up != n_dn:
        raise NotImplementedError(
            "only closed-shell single determinants are supported "
            f"(n_up={n_up}, n_dn={n_dn})")
    md = None
    if trial is not None:
        md = parse_trial(trial, n_up, n_dn)
        nocc = n_up
        C = np.ascontiguousarray(md["C"][:, md["occ_up"][0]])
    else:
        nocc = int(np.count_nonzero(np.asarray(mf.mo_occ) > 0))
        if nocc != n_up:
            raise ValueError(f"mo_occ marks {nocc} occupied orbitals, expected "
                             f"{n_up} for {n_e} electrons")
        C = np.ascontiguousarray(np.asarray(mf.mo_coeff, dtype=np.float64)[:, :nocc])
    cusp = params_cusp is not None
    shells = build_shells(mol, cusp=cusp)
    nbf = shells[-1].isgs + shells[-1].nsgs
    if C.shape[0] != nbf:
        raise ValueError(f"mo_coeff has {C.shape[0]} rows, basis has {nbf}")
    natm = mol.natm
    Z = mol.atom_charges().astype(np.float64)
    rc = np.zeros(natm)
    q0 = np.zeros(natm)
    coeff = np.zeros((natm, 8))
    if cusp:
        for ia in range(natm):
            sym = mol.atom_symbol(ia)
            rc[ia] = 0.1 if Z[ia] == 1 else 0.2
            q0[ia] = float(params_cusp[sym]["q0"])
            cf = np.ravel(np.asarray(params_cusp[sym]["coeff"], dtype=np.float64))
            if cf.shape[0] != 8:
                raise ValueError(f"cusp coeff for {sym} must have 8 entries")
            coeff[ia] = cf
    pc = {} if params_corr is None else params_corr
    has_j1, j1, has_j2, j2 = parse_params_corr(
        {k: v for k, v in pc.items() if not k.endswith("_bspline") and k != "J3_eeI"},
        mol, cusp)
    bs2, bs1 = parse_bspline(pc, mol, cusp, jastrow_config)
    j3 = parse_j3(pc, mol, jastrow_config)
    spl = ao_spline_tables(shells, getattr(mol, "ao_radial_transform", None))
    return System(nuc=mol.atom_coords(unit="Bohr"), Z=Z, shells=shells, C=C,
                  n_up=n_up, n_dn=n_dn, has_j1=has_j1, j1=j1, has_j2=has_j2,
                  j2=j2, cusp=cusp, cusp_rc=rc, cusp_q0=q0,
                  cusp_coeff=coeff, symbols=mol.elements, bs2=bs2, bs1=bs1, j3=j3, md=md,
                  spl=spl)
