"""Cusp-correction parameters of the "Quady2025" scheme.

Restates ``get_cusp_params`` (``OmegaQMC/psi/cusp.py:25-93``) for a basis
given in PySCF's internal format:

1. the 1s contraction is the s entry with the most primitives, first
   coefficient column, normalised like ``read_shell`` (``cusp.py:340-372``);
2. inside the sphere r < rc (rc = 0.1 for H, 0.2 otherwise) eight radial
   functions are used: (1-b) X with X the 1s contraction, and
   b e^{-Zr} (r/rc)^k for k = 0, 2..7 (``cusp.py:285-300``); the overlap and
   Hamiltonian (-1/2 nabla^2 - Z/r) matrices over the sphere come from
   32-point Gauss-Legendre quadrature in r (the functions are spherical, so
   the angular integral is 4 pi) (``cusp.py:200-282``);
3. the lowest eigenvector of H c = E S c, scaled to c[0] = 1, is ``coeff``
   (``cusp.py:302-338``);
4. ``q0`` minimises (S_cusp - S_gto)^2 + (H_cusp - H_gto)^2 over the sphere
   (``cusp.py:390-457``; optax L-BFGS there, a bounded scalar search here).
"""
from __future__ import annotations

import numpy as np
from scipy.optimize import minimize_scalar

from .system import ELEMENT_Z

__all__ = ["get_cusp_params", "cusp_params_for_mol"]

PI32 = np.pi ** 1.5


def _one_s(basis):
    s_entries = [e for e in basis if e[0] == 0]
    entry = max(s_entries, key=lambda e: len(e) - 1)
    prim = np.array(entry[1:], dtype=np.float64)
    a, c = prim[:, 0], prim[:, 1]
    norm = c * np.exp(0.75 * np.log(2.0 * a / np.pi))
    asum = a[:, None] + a[None, :]
    S = np.sum(norm[:, None] * norm[None, :] / (asum * np.sqrt(asum)))
    return a, norm / np.sqrt(S * PI32)


def _b(r, rc):
    s = r / rc
    inside = r < rc
    b = np.where(inside, 1 - 10 * s ** 3 + 15 * s ** 4 - 6 * s ** 5, 0.0)
    b1 = np.where(inside, -(30 / rc) * s ** 2 * (1 - s) ** 2, 0.0)
    b2 = np.where(inside, -(60 / rc ** 2) * s * (1 - s) * (1 - 2 * s), 0.0)
    return b, b1, b2


def _funcs(r, a, n, Z, rc):
    """Values, first and second radial derivatives of the 8 functions."""
    b, b1, b2 = _b(r, rc)
    e = np.exp(-a[None, :] * (r * r)[:, None]) * n[None, :]
    X = e.sum(1)
    X1 = (-2 * a[None, :] * r[:, None] * e).sum(1)
    X2 = ((4 * a[None, :] ** 2 * (r * r)[:, None] - 2 * a[None, :]) * e).sum(1)
    vals, d1, d2 = [(1 - b) * X], [-b1 * X + (1 - b) * X1], [-b2 * X - 2 * b1 * X1 + (1 - b) * X2]
    S = np.exp(-Z * r)
    for k in (0, 2, 3, 4, 5, 6, 7):
        p = (r / rc) ** k
        p1 = k * r ** (k - 1) / rc ** k if k > 0 else 0 * r
        p2 = k * (k - 1) * r ** (k - 2) / rc ** k if k > 1 else 0 * r
        f = b * S * p
        f1 = b1 * S * p - Z * b * S * p + b * S * p1
        f2 = (b2 * S * p + Z * Z * b * S * p + b * S * p2
              + 2 * (-Z * b1 * S * p + b1 * S * p1 - Z * b * S * p1))
        vals.append(f)
        d1.append(f1)
        d2.append(f2)
    return np.array(vals), np.array(d1), np.array(d2)


def _quad(rc, n=32):
    x, w = np.polynomial.legendre.leggauss(n)
    return rc * 0.5 * (x + 1.0), rc * 0.5 * w


def _sh(f, f1, f2, r, w, Z):
    """Overlap and Hamiltonian matrices of functions f (m, nr) on the sphere."""
    dv = 4.0 * np.pi * r * r * w
    lap = f2 + 2.0 / r * f1
    S = (f * dv) @ f.T
    H = (f * dv) @ (-0.5 * lap - Z / r * f).T
    return S, 0.5 * (H + H.T)


def get_cusp_params(elem, basis):
    """``{elem: {"q0": float, "coeff": [8 floats]}}`` for ``elem`` in ``basis``
    (a PySCF-format list of entries for that element)."""
    Z = float(ELEMENT_Z[elem])
    rc = 0.1 if Z == 1 else 0.2
    a, n = _one_s(basis)
    r, w = _quad(rc)
    f, f1, f2 = _funcs(r, a, n, Z, rc)
    S, H = _sh(f, f1, f2, r, w, Z)
    L = np.linalg.cholesky(S + 1e-14 * np.eye(8) * np.max(np.abs(np.diag(S))))
    Li = np.linalg.inv(L)
    ev, y = np.linalg.eigh(Li @ H @ Li.T)
    c = Li.T @ y[:, np.argmin(ev)]
    coeff = c / c[0]
    # q0: match the GTO's overlap and energy over the sphere
    e = np.exp(-a[None, :] * (r * r)[:, None]) * n[None, :]
    X = e.sum(1)
    X1 = (-2 * a[None, :] * r[:, None] * e).sum(1)
    X2 = ((4 * a[None, :] ** 2 * (r * r)[:, None] - 2 * a[None, :]) * e).sum(1)
    Sg, Hg = _sh(X[None], X1[None], X2[None], r, w, Z)

    def obj(q0):
        cv = coeff.copy()
        cv[1:] *= q0
        g, g1, g2 = cv @ f, cv @ f1, cv @ f2
        Sc, Hc = _sh(g[None], g1[None], g2[None], r, w, Z)
        return (Sc[0, 0] - Sg[0, 0]) ** 2 + (Hc[0, 0] - Hg[0, 0]) ** 2

    res = minimize_scalar(obj, bounds=(1e-6, 1e3), method="bounded",
                          options={"xatol": 1e-12, "maxiter": 500})
    return {elem: {"q0": float(res.x), "coeff": [float(x) for x in coeff]}}


def cusp_params_for_mol(mol):
    """Cusp parameters for every element of ``mol``."""
    out = {}
    for sym in mol.elements:
        if sym not in out:
            out.update(get_cusp_params(sym, mol._basis[sym]))
    return out
