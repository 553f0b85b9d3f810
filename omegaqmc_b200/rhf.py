"""Restricted Hartree-Fock front end (molecular orbitals without PySCF).

The reference obtains its occupied orbitals from a PySCF RHF calculation
(``OmegaQMC/vmc_gto.py:217-452``).  This module computes them for the same
basis conventions: every spherical AO of ``read_shell`` is expanded in
Cartesian Gaussian primitives (the solid-harmonic polynomials of
``_angular_cartesian`` times the normalised contraction), the one- and
two-electron integrals over those primitives come from
``csrc/mdints.c`` (McMurchie-Davidson), and a DIIS-accelerated SCF gives
``mo_coeff`` in the AO order the kernels use.

Usage::

    mf = run_rhf(mol)      # MeanField with mo_coeff, mo_occ, e_tot
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from .system import MeanField, build_shells

HERE = os.path.dirname(os.path.abspath(__file__))
_SRC = os.path.join(HERE, "csrc", "mdints.c")
_LIB = os.path.join(HERE, "libmdints.so")
_lib = None

# Real solid harmonics as monomials (the polynomials of _angular_cartesian,
# OmegaQMC/psi/gto.py:607-671): component -> [(coef, i, j, k)]
_s3 = np.sqrt(3.0)


def _harmonics():
    from math import sqrt
    cf1 = sqrt(2.5) * 0.5; cf2 = 3 * cf1; cf3 = sqrt(15.0); cf4 = sqrt(1.5) * 0.5
    cf5 = sqrt(6.0); cf6 = 1.5; cf7 = cf3 * 0.5
    g = [None, 2.9580398915498085, 6.2749501990055672, 2.0916500663351894,
         1.1180339887498949, 6.7082039324993694, 2.3717082451262845,
         3.1622776601683795, 0.55901699437494745, 3.3541019662496847,
         0.73950997288745213, 4.4370598373247132]
    return {
        0: [[(1.0, 0, 0, 0)]],
        1: [[(1.0, 1, 0, 0)], [(1.0, 0, 1, 0)], [(1.0, 0, 0, 1)]],
        2: [[(_s3, 1, 1, 0)], [(_s3, 0, 1, 1)],
            [(1.0, 0, 0, 2), (-0.5, 2, 0, 0), (-0.5, 0, 2, 0)],
            [(_s3, 1, 0, 1)], [(_s3 / 2, 2, 0, 0), (-_s3 / 2, 0, 2, 0)]],
        3: [[(cf2, 2, 1, 0), (-cf1, 0, 3, 0)], [(cf3, 1, 1, 1)],
            [(cf5, 0, 1, 2), (-cf4, 2, 1, 0), (-cf4, 0, 3, 0)],
            [(1.0, 0, 0, 3), (-cf6, 2, 0, 1), (-cf6, 0, 2, 1)],
            [(cf5, 1, 0, 2), (-cf4, 3, 0, 0), (-cf4, 1, 2, 0)],
            [(cf7, 2, 0, 1), (-cf7, 0, 2, 1)], [(-cf2, 1, 2, 0), (cf1, 3, 0, 0)]],
        4: [[(g[1], 3, 1, 0), (-g[1], 1, 3, 0)], [(g[2], 2, 1, 1), (-g[3], 0, 3, 1)],
            [(-g[4], 3, 1, 0), (-g[4], 1, 3, 0), (g[5], 1, 1, 2)],
            [(-g[6], 2, 1, 1), (-g[6], 0, 3, 1), (g[7], 0, 1, 3)],
            [(0.375, 4, 0, 0), (0.375, 0, 4, 0), (0.75, 2, 2, 0), (1.0, 0, 0, 4),
             (-3.0, 2, 0, 2), (-3.0, 0, 2, 2)],
            [(-g[6], 3, 0, 1), (-g[6], 1, 2, 1), (g[7], 1, 0, 3)],
            [(-g[8], 4, 0, 0), (g[8], 0, 4, 0), (g[9], 2, 0, 2), (-g[9], 0, 2, 2)],
            [(-g[2], 1, 2, 1), (g[3], 3, 0, 1)],
            [(g[10], 4, 0, 0), (g[10], 0, 4, 0), (-g[11], 2, 2, 0)]],
    }


HARM = _harmonics()


def _load():
    global _lib
    if _lib is not None:
        return _lib
    if (not os.path.exists(_LIB)) or os.path.getmtime(_LIB) < os.path.getmtime(_SRC):
        subprocess.run(["gcc", "-O3", "-fopenmp", "-fPIC", "-shared", "-o", _LIB + ".tmp",
                        _SRC, "-lm"], check=True)
        os.replace(_LIB + ".tmp", _LIB)
    lib = ctypes.CDLL(_LIB)
    P = ctypes.c_void_p
    lib.md_one_electron.argtypes = [ctypes.c_int, P, P, P, ctypes.c_int, P, P, P, P, P]
    lib.md_eri.argtypes = [ctypes.c_int, P, P, P, P]
    _lib = lib
    return lib


def cartesian_expansion(mol):
    """Primitive Cartesian functions and the AO expansion matrix.

    Returns (ctr (n,3), alpha (n,), pw (n,3) int, Tm (n, nbf)) with
    chi_ao(r) = sum_k Tm[k, ao] (x-A)^i (y-A)^j (z-A)^k exp(-alpha_k |r-A|^2)."""
    shells = build_shells(mol)
    nbf = shells[-1].isgs + shells[-1].nsgs
    nuc = mol.atom_coords()
    index = {}
    ctr, alpha, pw = [], [], []
    cols = []
    for sh in shells:
        for ic, terms in enumerate(HARM[sh.am]):
            ao = sh.isgs + ic
            for p, a in enumerate(sh.alpha):
                for coef, i, j, k in terms:
                    key = (sh.iat, float(a), i, j, k)
                    if key not in index:
                        index[key] = len(ctr)
                        ctr.append(nuc[sh.iat])
                        alpha.append(a)
                        pw.append((i, j, k))
                    cols.append((index[key], ao, coef * sh.norm[p]))
    n = len(ctr)
    Tm = np.zeros((n, nbf))
    for r, c, v in cols:
        Tm[r, c] += v
    return (np.ascontiguousarray(ctr, dtype=np.float64), np.asarray(alpha, dtype=np.float64),
            np.ascontiguousarray(pw, dtype=np.int32), Tm)


def integrals(mol):
    """(S, T, V, ERI) in the spherical AO basis of ``mol``."""
    lib = _load()
    ctr, alpha, pw, Tm = cartesian_expansion(mol)
    n = len(alpha)
    nuc = np.ascontiguousarray(mol.atom_coords(), dtype=np.float64)
    Z = mol.atom_charges().astype(np.float64)
    S = np.zeros((n, n)); T = np.zeros((n, n)); V = np.zeros((n, n))
    lib.md_one_electron(n, ctr.ctypes.data, alpha.ctypes.data, pw.ctypes.data, len(Z),
                        nuc.ctypes.data, Z.ctypes.data, S.ctypes.data, T.ctypes.data,
                        V.ctypes.data)
    eri = np.zeros((n, n, n, n))
    lib.md_eri(n, ctr.ctypes.data, alpha.ctypes.data, pw.ctypes.data, eri.ctypes.data)
    S = Tm.T @ S @ Tm
    T = Tm.T @ T @ Tm
    V = Tm.T @ V @ Tm
    # four quarter transformations
    g = np.tensordot(Tm, eri, axes=([0], [0]))            # a' b c d
    g = np.tensordot(g, Tm, axes=([1], [0]))               # a' c d b'
    g = np.tensordot(g, Tm, axes=([1], [0]))               # a' d b' c'
    g = np.tensordot(g, Tm, axes=([1], [0]))               # a' b' c' d'
    return S, T, V, g


def run_rhf(mol, max_iter=200, tol=1e-9, verbose=False):
    """Closed-shell RHF; returns a :class:`MeanField` with ``e_tot``."""
    S, T, V, eri = integrals(mol)
    H = T + V
    nocc = mol.tot_electrons() // 2
    e_nn = 0.0
    nuc = mol.atom_coords()
    Z = mol.atom_charges().astype(float)
    for i in range(len(Z)):
        for j in range(i + 1, len(Z)):
            e_nn += Z[i] * Z[j] / np.linalg.norm(nuc[i] - nuc[j])
    s, U = np.linalg.eigh(S)
    keep = s > 1e-9
    X = U[:, keep] / np.sqrt(s[keep])
    e, Cp = np.linalg.eigh(X.T @ H @ X)
    C = X @ Cp
    D = 2 * C[:, :nocc] @ C[:, :nocc].T
    diis_f, diis_e = [], []
    e_old = 0.0
    for it in range(max_iter):
        J = np.einsum("abcd,cd->ab", eri, D)
        K = np.einsum("acbd,cd->ab", eri, D)
        F = H + J - 0.5 * K
        err = F @ D @ S - S @ D @ F
        diis_f.append(F)
        diis_e.append(err)
        if len(diis_f) > 8:
            diis_f.pop(0)
            diis_e.pop(0)
        if len(diis_f) >= 2:
            m = len(diis_f)
            B = -np.ones((m + 1, m + 1))
            B[m, m] = 0.0
            for i in range(m):
                for j in range(m):
                    B[i, j] = np.vdot(diis_e[i], diis_e[j])
            rhs = np.zeros(m + 1)
            rhs[m] = -1.0
            try:
                c = np.linalg.solve(B, rhs)[:m]
                F = sum(ci * Fi for ci, Fi in zip(c, diis_f))
            except np.linalg.LinAlgError:
                pass
        e, Cp = np.linalg.eigh(X.T @ F @ X)
        C = X @ Cp
        D_new = 2 * C[:, :nocc] @ C[:, :nocc].T
        Fr = H + np.einsum("abcd,cd->ab", eri, D_new) - 0.5 * np.einsum("acbd,cd->ab", eri, D_new)
        e_el = 0.5 * np.sum(D_new * (H + Fr))
        if verbose:
            print(it, e_el + e_nn, np.max(np.abs(err)))
        if abs(e_el - e_old) < tol and np.max(np.abs(err)) < 1e-6:
            D = D_new
            break
        D = D_new
        e_old = e_el
    nbf = S.shape[0]
    mo_occ = np.zeros(C.shape[1])
    mo_occ[:nocc] = 2.0
    mf = MeanField(mol, C, mo_occ)
    mf.mo_energy = e
    mf.e_tot = float(e_el + e_nn)
    mf.converged = it < max_iter - 1
    mf.S = S
    return mf
