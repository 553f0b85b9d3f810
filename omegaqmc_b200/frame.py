"""Canonical molecular frame of ``generate_molecular_orbitals``
(``OmegaQMC/vmc_gto.py:314-352`` with ``symmetrization_level >= 1``).

The reference moves a molecule without point-group symmetry (C1) to the
centre of nuclear charge and rotates it onto the principal axes of the
charge-weighted inertia tensor, ordered by ascending moment and signed by a
rule that depends only on the geometry (``charge_inertia_axes``,
``OmegaQMC/symm/point_groups.py:439-568``).  This module restates that
transformation.  Molecules with symmetry keep, in the reference, the axes
PySCF's ``symm.geom.detect_symm`` assigns (re-signed); PySCF is not part of
this package, so here they keep their input frame.  Energies and every other
sampled quantity are invariant under the rotation; only the coordinates
written to the checkpoint differ.
"""
from __future__ import annotations

import numpy as np

__all__ = ["charge_inertia_axes", "has_point_symmetry", "canonical_coordinates"]


def _reference_atom(proj, tol_rel=1e-6):
    """Atom with the largest |projection|, near-ties (to tol_rel of the
    largest) going to the lowest index (``point_groups.py:439-454``)."""
    a = np.abs(np.asarray(proj, dtype=float))
    scale = max(1.0, float(a.max()))
    bucket = np.round(a / (tol_rel * scale))
    best = bucket.max()
    return int(np.flatnonzero(bucket == best)[0])


def _charge_inertia(coords, charges):
    """Centre of nuclear charge, centred coordinates and the ascending
    eigen-decomposition of sum_i q_i (|x_i|^2 1 - x_i x_i^T)
    (``point_groups.py:457-476``)."""
    c = np.asarray(coords, dtype=float)
    q = np.asarray(charges, dtype=float)
    centre = q @ c / q.sum()
    x = c - centre
    r2 = np.einsum("ij,ij->i", x, x)
    tensor = np.einsum("i,i->", q, r2) * np.eye(3) - np.einsum("i,ij,ik->jk", q, x, x)
    evals, evecs = np.linalg.eigh(tensor)
    return centre, x, evals, evecs


def _degenerate(evals, rtol):
    scale = max(1.0, float(np.abs(evals).max()))
    return bool(np.any(np.diff(evals) < rtol * scale))


def _signed_frame(dirs, x, tol_rel=1e-8):
    """Rows of ``dirs`` signed so that each axis's most strongly projected
    atom sits at a positive coordinate, then made a proper rotation by
    flipping an undetermined axis (or the least-determined one)
    (``point_groups.py:490-521``)."""
    A = np.array(dirs, dtype=float)
    tol = tol_rel * max(1.0, float(np.abs(x).max()))
    score = np.empty(3)
    for k in range(3):
        p = x @ A[k]
        score[k] = p[_reference_atom(p)]
        if score[k] < -tol:
            A[k] *= -1.0
            score[k] = -score[k]
    if np.linalg.det(A) < 0.0:
        free = [k for k in range(3) if abs(score[k]) <= tol]
        k = free[0] if free else int(np.argmin(score))
        A[k] *= -1.0
    return A


def charge_inertia_axes(coords, charges, degen_rtol=1e-3):
    """(centre, axes) of the canonical frame: centre of nuclear charge and the
    charge-inertia principal axes as rows (ascending moment, proper
    rotation); None when two moments coincide to ``degen_rtol``."""
    centre, x, evals, evecs = _charge_inertia(coords, charges)
    if _degenerate(evals, degen_rtol):
        return None
    return centre, _signed_frame(evecs.T, x)


def has_point_symmetry(coords, charges, tol=1e-5, degen_rtol=1e-3):
    """Whether the nuclei have a symmetry operation besides the identity.

    A degenerate charge-inertia tensor (linear molecules, groups with a
    three-fold or higher axis) counts as symmetric.  Otherwise every
    operation of the molecule's point group maps the principal axes onto
    themselves, so the candidates are the inversion, the two-fold rotations
    about the axes and the reflections through the planes normal to them;
    each is tested on the nuclei (same charge within ``tol`` bohr)."""
    centre, x, evals, evecs = _charge_inertia(coords, charges)
    if _degenerate(evals, degen_rtol):
        return True
    q = np.asarray(charges, dtype=float)
    y = x @ evecs                       # coordinates in the principal frame
    ops = [np.diag(d) for d in ((-1, -1, -1), (1, -1, -1), (-1, 1, -1), (-1, -1, 1),
                                (-1, 1, 1), (1, -1, 1), (1, 1, -1))]
    for R in ops:
        z = y @ R
        d = np.linalg.norm(z[:, None, :] - y[None, :, :], axis=-1)
        same = np.abs(q[:, None] - q[None, :]) < 1e-9
        if np.all(np.any((d < tol) & same, axis=1)):
            return True
    return False


def canonical_coordinates(coords, charges):
    """Coordinates in the reference's canonical frame for a molecule
    without point-group symmetry; the input coordinates otherwise."""
    c = np.asarray(coords, dtype=float)
    if len(c) < 2 or has_point_symmetry(c, charges):
        return c.copy()
    frame = charge_inertia_axes(c, charges)
    if frame is None:
        return c.copy()
    centre, axes = frame
    return (c - centre) @ axes.T
