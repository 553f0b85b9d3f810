"""CPU FP64 oracle for the GTO Slater–Jastrow evaluation (TEST INFRASTRUCTURE).

This module is the checker, never the product: only ``tests/``, the smoke
entry point and the CPU-baseline leg of the benchmark may import it.  It
restates the reference's per-walker evaluation in numpy, vectorised over
walkers, line by line from:

* ``OmegaQMC/psi/shell.py:37-148``   cusp-corrected s orbital (value, VGL)
* ``OmegaQMC/psi/gto.py:607-725``    real solid harmonics and their gradients
* ``OmegaQMC/psi/gto.py:781-811``    contracted radial value, R'/r, Laplacian
* ``OmegaQMC/psi/gto.py:1012-1056``  AO values (``cgs_sph_get``)
* ``OmegaQMC/psi/gto.py:1101-1214``  AO/MO value-gradient-Laplacian
* ``OmegaQMC/psi/gto.py:728-778``    Slater assembly (inverse, Gamma, lap)
* ``OmegaQMC/psi/gto.py:1278-1290``  log|det| of the up and down blocks
* ``OmegaQMC/psi/gto.py:1319-1480``  multi-determinant Slater part
* ``OmegaQMC/psi/gto.py:141-240``    quintic radial splines of the AO transform
* ``OmegaQMC/psi/gto.py:1493-1649``  Padé J1/J2 value and VGL
* ``OmegaQMC/psi/gto.py:243-604, 1933-2196``  J3_eeI three-body Jastrow
* ``OmegaQMC/psi/gto.py:2220-2254``  log|psi| = log|det| + J
* ``OmegaQMC/psi/gto.py:2406-2451``  eps-softened Coulomb terms
* ``OmegaQMC/psi/gto.py:2506-2579``  analytic kinetic energy

It is pinned against outputs of the reference's own source (run under a
numpy/torch stand-in for JAX, ``tests/golden/make_golden.py``) and against
the relations the reference's tests check (closed-form J1, the ``np.dot``
cusp form, analytic versus autodiff-Hessian kinetic energy).
"""
from __future__ import annotations

import math

import numpy as np

EPS = float(np.finfo(np.float64).eps)
MIN_DIST_THRESHOLD = 1e-4   # OmegaQMC/constants.py:23

# ---------------------------------------------------------------------------
# Real solid harmonics as monomial tables: Y_c = sum coef * x^i y^j z^k.
# The polynomials are those of _angular_cartesian (gto.py:607-671).
# ---------------------------------------------------------------------------
_cd1 = math.sqrt(3.0)
_cd2 = _cd1 * 0.5
_cf1 = math.sqrt(2.5) * 0.5
_cf2 = 3.0 * _cf1
_cf3 = math.sqrt(15.0)
_cf4 = math.sqrt(1.5) * 0.5
_cf5 = math.sqrt(6.0)
_cf6 = 1.5
_cf7 = _cf3 * 0.5
_cg = [None, 2.9580398915498085, 6.2749501990055672, 2.0916500663351894,
       1.1180339887498949, 6.7082039324993694, 2.3717082451262845,
       3.1622776601683795, 0.55901699437494745, 3.3541019662496847,
       0.73950997288745213, 4.4370598373247132]

HARMONICS = {
    0: [[(1.0, 0, 0, 0)]],
    1: [[(1.0, 1, 0, 0)], [(1.0, 0, 1, 0)], [(1.0, 0, 0, 1)]],
    2: [[(_cd1, 1, 1, 0)],
        [(_cd1, 0, 1, 1)],
        [(1.0, 0, 0, 2), (-0.5, 2, 0, 0), (-0.5, 0, 2, 0)],
        [(_cd1, 1, 0, 1)],
        [(_cd2, 2, 0, 0), (-_cd2, 0, 2, 0)]],
    3: [[(_cf2, 2, 1, 0), (-_cf1, 0, 3, 0)],
        [(_cf3, 1, 1, 1)],
        [(_cf5, 0, 1, 2), (-_cf4, 2, 1, 0), (-_cf4, 0, 3, 0)],
        [(1.0, 0, 0, 3), (-_cf6, 2, 0, 1), (-_cf6, 0, 2, 1)],
        [(_cf5, 1, 0, 2), (-_cf4, 3, 0, 0), (-_cf4, 1, 2, 0)],
        [(_cf7, 2, 0, 1), (-_cf7, 0, 2, 1)],
        [(-_cf2, 1, 2, 0), (_cf1, 3, 0, 0)]],
    4: [[(_cg[1], 3, 1, 0), (-_cg[1], 1, 3, 0)],
        [(_cg[2], 2, 1, 1), (-_cg[3], 0, 3, 1)],
        [(-_cg[4], 3, 1, 0), (-_cg[4], 1, 3, 0), (_cg[5], 1, 1, 2)],
        [(-_cg[6], 2, 1, 1), (-_cg[6], 0, 3, 1), (_cg[7], 0, 1, 3)],
        [(0.375, 4, 0, 0), (0.375, 0, 4, 0), (0.75, 2, 2, 0), (1.0, 0, 0, 4),
         (-3.0, 2, 0, 2), (-3.0, 0, 2, 2)],
        [(-_cg[6], 3, 0, 1), (-_cg[6], 1, 2, 1), (_cg[7], 1, 0, 3)],
        [(-_cg[8], 4, 0, 0), (_cg[8], 0, 4, 0), (_cg[9], 2, 0, 2),
         (-_cg[9], 0, 2, 2)],
        [(-_cg[2], 1, 2, 1), (_cg[3], 3, 0, 1)],
        [(_cg[10], 4, 0, 0), (_cg[10], 0, 4, 0), (-_cg[11], 2, 2, 0)]],
}


def _pow(x, n):
    return np.ones_like(x) if n == 0 else x ** n


def harmonics(am, dr):
    """Y (..., 2am+1) and grad Y (..., 2am+1, 3) at displacements dr (..., 3)."""
    x, y, z = dr[..., 0], dr[..., 1], dr[..., 2]
    comps = HARMONICS[am]
    Y = np.zeros(dr.shape[:-1] + (len(comps),))
    G = np.zeros(dr.shape[:-1] + (len(comps), 3))
    for c, terms in enumerate(comps):
        for coef, i, j, k in terms:
            Y[..., c] += coef * _pow(x, i) * _pow(y, j) * _pow(z, k)
            if i:
                G[..., c, 0] += coef * i * _pow(x, i - 1) * _pow(y, j) * _pow(z, k)
            if j:
                G[..., c, 1] += coef * j * _pow(x, i) * _pow(y, j - 1) * _pow(z, k)
            if k:
                G[..., c, 2] += coef * k * _pow(x, i) * _pow(y, j) * _pow(z, k - 1)
    return Y, G


# ---------------------------------------------------------------------------
# Cusp-corrected s orbital (shell.py:37-148)
# ---------------------------------------------------------------------------
def cusp_b(r, rc):
    s = r / rc
    return np.where(r < rc, 1.0 - 10.0 * s ** 3 + 15.0 * s ** 4 - 6.0 * s ** 5, 0.0)


def cusp_s(r, rc, Z, rad_s, q0, coeff):
    """f = c0 (1-b) R + b q0 e^{-Zr} (c1 + sum_{k=2..7} c_k (r/rc)^k)."""
    b = cusp_b(r, rc)
    sl = q0 * np.exp(-Z * r)
    s = r / rc
    poly = coeff[1] + sum(coeff[k] * s ** k for k in range(2, 8))
    return coeff[0] * (1.0 - b) * rad_s + b * sl * poly


def cusp_s_vgl(r, rc, Z, R, Rp_r, Rlap, q0, coeff):
    """(f, f'/r, f'' + 2 f'/r) of the cusp-corrected s orbital.

    The (1-b) R part is division free as in ``shell.py:107-130``; the
    polynomial part Q = b q0 e^{-Zr} P(r) is differentiated analytically
    (the reference uses scalar autodiff, ``shell.py:132-147``) and keeps the
    plain ``Q'/r`` division."""
    s = r / rc
    oms = 1.0 - s
    inside = r < rc
    b = np.where(inside, 1.0 - 10.0 * s ** 3 + 15.0 * s ** 4 - 6.0 * s ** 5, 0.0)
    bp = np.where(inside, -(30.0 / rc) * s ** 2 * oms ** 2, 0.0)
    bp_r = np.where(inside, -(30.0 / rc ** 3) * r * oms ** 2, 0.0)
    bpp = np.where(inside, -(60.0 / rc ** 2) * s * oms * (1.0 - 2.0 * s), 0.0)
    BL = bpp + 2.0 * bp_r
    c0 = coeff[0]
    A_val = c0 * (1.0 - b) * R
    A_gr = c0 * (-bp_r * R + (1.0 - b) * Rp_r)
    A_lap = c0 * (-BL * R + (1.0 - b) * Rlap - 2.0 * r * bp * Rp_r)
    S = q0 * np.exp(-Z * r)
    P = coeff[1] + sum(coeff[k] * s ** k for k in range(2, 8))
    P1 = sum(k * coeff[k] * s ** (k - 1) for k in range(2, 8)) / rc
    P2 = sum(k * (k - 1) * coeff[k] * s ** (k - 2) for k in range(2, 8)) / rc ** 2
    Q = b * S * P
    Qp = bp * S * P - Z * b * S * P + b * S * P1
    Qpp = (bpp * S * P + Z * Z * b * S * P + b * S * P2
           + 2.0 * (-Z * bp * S * P + bp * S * P1 - Z * b * S * P1))
    Qp = np.where(inside, Qp, 0.0)
    Qpp = np.where(inside, Qpp, 0.0)
    Q_gr = Qp / r
    return A_val + Q, A_gr + Q_gr, A_lap + Qpp + 2.0 * Q_gr


# ---------------------------------------------------------------------------
# AO evaluation
# ---------------------------------------------------------------------------
# ---------------------------------------------------------------------------
# Quintic radial splines of the AO transform (gto.py:141-240)
# ---------------------------------------------------------------------------
def quintic_radial_spline(alpha, norm, smin=1.0e-6, tol=1.0e-7, npts=1001, rmax_cap=100.0):
    """(knots, coefs) of ``_build_quintic_radial_spline`` (gto.py:141-198):
    Hermite quintics matching g, g', g'' of g(s) = sum_p norm_p
    exp(-alpha_p s) at s = 0 and on a log grid up to the tol cutoff."""
    from scipy.interpolate import BPoly, PPoly
    a = np.asarray(alpha, dtype=np.float64)
    c = np.asarray(norm, dtype=np.float64)

    def ders(sv):
        e = np.exp(-a[None, :] * np.asarray(sv, dtype=np.float64)[:, None])
        return np.stack([(c * e).sum(1), (-a * c * e).sum(1), (a * a * c * e).sum(1)], axis=1)

    rs = np.linspace(0.0, rmax_cap, 20001)
    big = np.abs(ders(rs ** 2)[:, 0]) > tol
    rmax = float(rs[np.max(np.nonzero(big))]) if big.any() else 1.0
    smax = max(rmax ** 2, 100.0 * smin)
    sg = np.concatenate([[0.0], np.logspace(np.log10(smin), np.log10(smax), npts - 1)])
    pp = PPoly.from_bernstein_basis(BPoly.from_derivatives(sg, ders(sg)))
    return np.asarray(pp.x), np.asarray(pp.c).T


def spline_gdd(knots, coefs, s):
    """(g, g', g'') at s and the inside mask (``_locate_and_horner``,
    gto.py:200-217)."""
    seg = np.clip(np.searchsorted(knots, s, side="right") - 1, 0, coefs.shape[0] - 1)
    d = s - knots[seg]
    c = coefs[seg]
    g = ((((c[..., 0] * d + c[..., 1]) * d + c[..., 2]) * d + c[..., 3]) * d + c[..., 4]) * d \
        + c[..., 5]
    gp = (((5 * c[..., 0] * d + 4 * c[..., 1]) * d + 3 * c[..., 2]) * d + 2 * c[..., 3]) * d \
        + c[..., 4]
    gpp = ((20 * c[..., 0] * d + 12 * c[..., 1]) * d + 6 * c[..., 2]) * d + 2 * c[..., 3]
    inside = s < knots[-1]
    return np.where(inside, g, 0.0), np.where(inside, gp, 0.0), np.where(inside, gpp, 0.0)


_SPL_CACHE = {}


def _shell_spline(system, i, sh):
    """The spline of shell i when the system's AO transform splines it."""
    spl = getattr(system, "spl", None)
    if spl is None or i not in spl["tables"]:
        return None
    key = (tuple(sh.alpha), tuple(sh.norm), tuple(sorted(spl["cfg"].items())))
    if key not in _SPL_CACHE:
        _SPL_CACHE[key] = quintic_radial_spline(sh.alpha, sh.norm, **spl["cfg"])
    return _SPL_CACHE[key]


def _shell_disp(system, sh, x):
    dr = x - system.nuc[sh.iat]
    r2 = np.sum(dr * dr, axis=-1)
    return dr, r2, np.sqrt(r2)


def ao_value(system, x):
    """AO values (..., nbf) at positions x (..., 3) (``gto.py:1012-1056``)."""
    out = np.zeros(x.shape[:-1] + (system.nbf,))
    for i, sh in enumerate(system.shells):
        dr, r2, r = _shell_disp(system, sh, x)
        R = np.sum(np.exp(-sh.alpha * r2[..., None]) * sh.norm, axis=-1)
        sp = _shell_spline(system, i, sh)
        if sp is not None:
            R = spline_gdd(sp[0], sp[1], r2)[0]                    # _radial_val_spline
        if sh.am == 0 and sh.is_cusp:
            ia = sh.iat
            v = cusp_s(r, system.cusp_rc[ia], system.Z[ia], R,
                       system.cusp_q0[ia], system.cusp_coeff[ia])[..., None]
        else:
            Y, _ = harmonics(sh.am, dr)
            v = R[..., None] * Y
        out[..., sh.isgs:sh.isgs + sh.nsgs] = v
    return out


def ao_vgl(system, x):
    """AO value (..., nbf), gradient (..., nbf, 3), Laplacian (..., nbf)
    (``gto.py:781-811, 1101-1186``)."""
    shp = x.shape[:-1]
    val = np.zeros(shp + (system.nbf,))
    grad = np.zeros(shp + (system.nbf, 3))
    lap = np.zeros(shp + (system.nbf,))
    for i, sh in enumerate(system.shells):
        dr, r2, r = _shell_disp(system, sh, x)
        e = np.exp(-sh.alpha * r2[..., None]) * sh.norm
        R = np.sum(e, axis=-1)
        Rp = np.sum(-2.0 * sh.alpha * e, axis=-1)
        Rl = np.sum((4.0 * sh.alpha ** 2 * r2[..., None] - 6.0 * sh.alpha) * e, axis=-1)
        sp = _shell_spline(system, i, sh)
        if sp is not None:                                          # _radial_vgl_spline
            g, gp, gpp = spline_gdd(sp[0], sp[1], r2)
            R, Rp, Rl = g, 2.0 * gp, 6.0 * gp + 4.0 * r2 * gpp
        sl = slice(sh.isgs, sh.isgs + sh.nsgs)
        if sh.am == 0:
            if sh.is_cusp:
                ia = sh.iat
                R, Rp, Rl = cusp_s_vgl(r, system.cusp_rc[ia], system.Z[ia], R, Rp,
                                       Rl, system.cusp_q0[ia], system.cusp_coeff[ia])
            val[..., sl] = R[..., None]
            grad[..., sl, :] = (Rp[..., None] * dr)[..., None, :]
            lap[..., sl] = Rl[..., None]
        else:
            Y, gY = harmonics(sh.am, dr)
            val[..., sl] = R[..., None] * Y
            grad[..., sl, :] = (Rp[..., None, None] * dr[..., None, :] * Y[..., None]
                                + R[..., None, None] * gY)
            lap[..., sl] = (Rl + 2.0 * sh.am * Rp)[..., None] * Y
    return val, grad, lap


def mo_value(system, X):
    """MO values (W, n_e, nocc) (``gto.py:1058-1070``)."""
    return ao_value(system, X) @ system.C


def mo_vgl(system, X):
    """MO value/gradient/Laplacian (``gto.py:1188-1214``)."""
    v, g, l = ao_vgl(system, X)
    return (v @ system.C, np.einsum("...ax,am->...mx", g, system.C),
            l @ system.C)


# ---------------------------------------------------------------------------
# Slater determinant
# ---------------------------------------------------------------------------
def log_slater(system, X):
    """log|det up| + log|det down| (``gto.py:1278-1290``), or the
    multi-determinant log|sum_d c_d D_up D_dn| with a trial."""
    if getattr(system, "md", None) is not None:
        return multidet_assemble(system, X)[0]
    mo = mo_value(system, X)
    _, la = np.linalg.slogdet(mo[:, 0::2, :])
    _, lb = np.linalg.slogdet(mo[:, 1::2, :])
    return la + lb


def slater_assemble(mo_val, mo_grad, mo_lap):
    """(log|det|, grad_e (W,n_e,3), lap_e (W,n_e)) (``gto.py:728-778``)."""
    W, n_e, _ = mo_val.shape
    grad = np.zeros((W, n_e, 3))
    lap = np.zeros((W, n_e))
    logv = np.zeros(W)
    for off in (0, 1):
        S = mo_val[:, off::2, :]
        G = mo_grad[:, off::2, :, :]
        L = mo_lap[:, off::2, :]
        A = np.linalg.inv(S)
        Gam = np.einsum("wji,wijx->wix", A, G)
        lp = np.einsum("wji,wij->wi", A, L) - np.sum(Gam * Gam, axis=-1)
        _, ld = np.linalg.slogdet(S)
        logv += ld
        grad[:, off::2] = Gam
        lap[:, off::2] = lp
    return logv, grad, lap


def multidet_assemble(system, X):
    """(log|psi_S|, grad_e, lap_e) of a multi-determinant Slater part,
    restating ``log_slater_multidet`` and ``log_slater_multidet_analytic``
    (gto.py:1319-1480): per term the up and down slogdet, inverses, Gamma
    and ell; signed log-sum-exp weights w_d summing to 1; grad = sum_d w_d
    Gamma_d, lap = sum_d w_d (|Gamma_d|^2 + ell_d) - |grad|^2."""
    md = system.md
    C = md["C"]
    v, g, l = ao_vgl(system, X)
    mv = v @ C
    mg = np.einsum("...ax,am->...mx", g, C)
    ml = l @ C
    W, n_e, _ = X.shape
    nd = len(md["ci"])
    logs = np.zeros((W, nd))
    phase = np.zeros((W, nd))
    gam = np.zeros((W, nd, n_e, 3))
    sec = np.zeros((W, nd, n_e))
    for d in range(nd):
        for off, occ in ((0, md["occ_up"][d]), (1, md["occ_dn"][d])):
            S = mv[:, off::2][:, :, occ]
            G = mg[:, off::2][:, :, occ, :]
            L = ml[:, off::2][:, :, occ]
            sgn, ld = np.linalg.slogdet(S)
            A = np.linalg.inv(S)
            Gam = np.einsum("wji,wijx->wix", A, G)
            ell = np.einsum("wji,wij->wi", A, L) - np.sum(Gam * Gam, axis=-1)
            logs[:, d] += ld
            phase[:, d] = (sgn if off == 0 else phase[:, d] * sgn)
            gam[:, d, off::2] = Gam
            sec[:, d, off::2] = np.sum(Gam * Gam, axis=-1) + ell
        phase[:, d] *= np.sign(md["ci"][d])
    contrib = np.log(np.abs(md["ci"]))[None, :] + logs
    lmax = np.max(contrib, axis=1)
    shifted = phase * np.exp(contrib - lmax[:, None])
    total = np.sum(shifted, axis=1)
    w = shifted / total[:, None]
    grad = np.einsum("wd,wdix->wix", w, gam)
    lap = np.einsum("wd,wdi->wi", w, sec) - np.sum(grad * grad, axis=-1)
    return np.log(np.abs(total)) + lmax, grad, lap


# ---------------------------------------------------------------------------
# Padé Jastrow
# ---------------------------------------------------------------------------
def _pairs(n_e):
    return np.triu_indices(n_e, k=1)


def bspline_vgl(c, r, r_cut):
    """Uniform-knot cubic B-spline u(r), u'(r), u''(r) with coefficients
    c[0..N+3] on knots k * dr, dr = r_cut / (N + 1), zero for r >= r_cut
    (``_bspline_eval_vgl``, ``gto.py:67-119``, with the callers' cutoff
    mask)."""
    c = np.asarray(c, dtype=np.float64)
    n = c.shape[0] - 4
    dinv = (n + 1) / r_cut
    x = r * dinv
    i = np.clip(np.floor(x).astype(np.int64), 0, n)
    t = x - i
    t2, t3 = t * t, t * t * t
    w = [(-t3 + 3 * t2 - 3 * t + 1) / 6, (3 * t3 - 6 * t2 + 4) / 6,
         (-3 * t3 + 3 * t2 + 3 * t + 1) / 6, t3 / 6]
    w1 = [(-3 * t2 + 6 * t - 3) / 6, (9 * t2 - 12 * t) / 6, (-9 * t2 + 6 * t + 3) / 6,
          3 * t2 / 6]
    w2 = [(-6 * t + 6) / 6, (18 * t - 12) / 6, (-18 * t + 6) / 6, 6 * t / 6]
    cs = [c[i + k] for k in range(4)]
    val = sum(w[k] * cs[k] for k in range(4))
    d1 = sum(w1[k] * cs[k] for k in range(4)) * dinv
    d2 = sum(w2[k] * cs[k] for k in range(4)) * dinv * dinv
    m = (r < r_cut).astype(np.float64)
    return val * m, d1 * m, d2 * m


# ---------------------------------------------------------------------------
# J3_eeI (gto.py:243-604, 1933-2196)
# ---------------------------------------------------------------------------
def eeI_constraint_map(N_eI, N_ee, r_cut):
    """gamma_unique = A @ free and the (l, m, n) of each unique gamma,
    restating ``_build_eeI_constraint_map`` (gto.py:321-463) loop by loop."""
    L = 0.5 * r_cut
    index = {}
    lmn = []
    for m in range(N_eI + 1):
        for l in range(m, N_eI + 1):
            for n in range(N_ee + 1):
                index[(l, m, n)] = index[(m, l, n)] = len(lmn)
                lmn.append((l, m, n))
    NG = len(lmn)
    NC = (2 * N_eI + 1) + (N_eI + N_ee + 1)
    Cm = np.zeros((NC, NG))
    for k in range(2 * N_eI + 1):
        for mi in range(k + 1):
            li = k - mi
            if li <= N_eI and mi <= N_eI:
                if li > mi:
                    Cm[k, index[(li, mi, 1)]] = 2.0
                elif li == mi:
                    Cm[k, index[(li, mi, 1)]] = 1.0
    ro = 2 * N_eI + 1
    for kp in range(N_eI + N_ee + 1):
        if kp <= N_ee:
            Cm[ro + kp, index[(0, 0, kp)]] = 3.0
            if N_eI >= 1:
                Cm[ro + kp, index[(0, 1, kp)]] = -L
        for li in range(1, kp + 1):
            ni = kp - li
            if 0 <= ni <= N_ee and li <= N_eI:
                Cm[ro + kp, index[(li, 0, ni)]] = 3.0
                if N_eI >= 1:
                    Cm[ro + kp, index[(li, 1, ni)]] = -L
    indep = np.zeros(NG, dtype=bool)
    col = -1
    for row in range(NC):
        while True:
            col += 1
            if col >= NG:
                break
            best, big = row, abs(Cm[row, col])
            for ri in range(row + 1, NC):
                if abs(Cm[ri, col]) > big:
                    best, big = ri, abs(Cm[ri, col])
            if big < 1e-6:
                indep[col] = True
                continue
            break
        if col >= NG:
            break
        Cm[[row, best]] = Cm[[best, row]]
        Cm[row] /= Cm[row, col]
        for ri in range(NC):
            if ri != row:
                Cm[ri] -= Cm[ri, col] * Cm[row]
    for c in range(col + 1, NG):
        indep[c] = True
    ic = np.where(indep)[0]
    dc = np.where(~indep)[0]
    A = np.zeros((NG, len(ic)))
    for p, j in enumerate(ic):
        A[j, p] = 1.0
    for c, i in enumerate(dc):
        for p, j in enumerate(ic):
            A[i, p] = -Cm[c, j]
    return A, lmn


def eeI_gamma3d(free, N_eI, N_ee, r_cut):
    """Symmetric gamma(l, m, n) of one block (``_vec_to_gamma_3d``)."""
    A, lmn = eeI_constraint_map(N_eI, N_ee, r_cut)
    vec = A @ np.asarray(free, dtype=np.float64)
    g = np.zeros((N_eI + 1, N_eI + 1, N_ee + 1))
    for k, (l, m, n) in enumerate(lmn):
        g[l, m, n] = g[m, l, n] = vec[k]
    return g


def _j3_blocks(system):
    """(atom index, same-spin flag, gamma) for every populated block."""
    j3 = getattr(system, "j3", None)
    if j3 is None:
        return []
    syms = list(system.symbols)
    out = []
    for I in range(system.natm):
        for prefix, same in (("like+", True), ("unlike+", False)):
            key = prefix + syms[I]
            if key in j3["params"]:
                out.append((I, same, eeI_gamma3d(j3["params"][key], j3["n_eI"], j3["n_ee"],
                                                 j3["r_cut"])))
    return out


def _eeI_poly_derivs(g, r12, r1, r2, L):
    """u = P (r1-L)^3 (r2-L)^3 and its partials for particle 1
    (``_eval_eeI_poly_vgl``, gto.py:508-604): u, u_1, u_12, u_11, u_1212,
    u_1_12."""
    nI, _, nE = g.shape
    P = P1 = P11 = P12 = P112 = P1212 = 0.0
    for l in range(nI):
        for m in range(nI):
            for n in range(nE):
                c = g[l, m, n]
                if c == 0.0:
                    continue
                a = r1 ** l
                a1 = l * r1 ** (l - 1) if l >= 1 else 0.0
                a2 = l * (l - 1) * r1 ** (l - 2) if l >= 2 else 0.0
                b = r2 ** m
                e = r12 ** n
                e1 = n * r12 ** (n - 1) if n >= 1 else 0.0
                e2 = n * (n - 1) * r12 ** (n - 2) if n >= 2 else 0.0
                P = P + c * a * b * e
                P1 = P1 + c * a1 * b * e
                P11 = P11 + c * a2 * b * e
                P12 = P12 + c * a * b * e1
                P112 = P112 + c * a1 * b * e1
                P1212 = P1212 + c * a * b * e2
    s1, s2 = r1 - L, r2 - L
    E = s1 ** 3 * s2 ** 3
    E1 = 3.0 * s1 ** 2 * s2 ** 3
    E11 = 6.0 * s1 * s2 ** 3
    return (P * E, P1 * E + P * E1, P12 * E, P11 * E + 2.0 * P1 * E1 + P * E11, P1212 * E,
            P112 * E + P12 * E1)


def j3_value(system, X, blocks=None):
    """J3_eeI = -sum over nuclei I and pairs i<j of the block's u, for
    r_iI, r_jI < L (``J3_eeI_fn``, gto.py:1951-2040).  ``blocks`` replaces
    the system's (atom, same-spin, gamma) blocks when given."""
    W, n_e, _ = X.shape
    J = np.zeros(W)
    blocks = _j3_blocks(system) if blocks is None else blocks
    if not blocks:
        return J
    L = 0.5 * system.j3["r_cut"]
    i, j = _pairs(n_e)
    for I, same, g in blocks:
        sel = ((i % 2) == (j % 2)) == same
        a, b = i[sel], j[sel]
        r12 = np.linalg.norm(X[:, a] - X[:, b], axis=-1)          # (W, pairs)
        r1 = np.linalg.norm(X[:, a] - system.nuc[I], axis=-1)
        r2 = np.linalg.norm(X[:, b] - system.nuc[I], axis=-1)
        # power tables and the einsum of _eval_eeI_poly (gto.py:474-488)
        p1 = np.stack([r1 ** k for k in range(g.shape[0])], axis=-1)
        p2 = np.stack([r2 ** k for k in range(g.shape[0])], axis=-1)
        p12 = np.stack([r12 ** k for k in range(g.shape[2])], axis=-1)
        P = np.einsum("lmn,wpl,wpm,wpn->wp", g, p1, p2, p12)
        u = P * ((r1 - L) * (r2 - L)) ** 3
        J -= np.sum(np.where((r1 < L) & (r2 < L), u, 0.0), axis=-1)
    return J


def j3_vgl(system, X, blocks=None):
    """Per-electron gradient and Laplacian of J3_eeI (``J3_eeI_vgl``,
    gto.py:2042-2196): each electron of a triplet takes the partials with
    itself as particle 1 (u is symmetric in the two electrons)."""
    W, n_e, _ = X.shape
    grad = np.zeros((W, n_e, 3))
    lap = np.zeros((W, n_e))
    blocks = _j3_blocks(system) if blocks is None else blocks
    if not blocks:
        return grad, lap
    L = 0.5 * system.j3["r_cut"]
    for I, same, g in blocks:
        for a in range(n_e):
            for b in range(n_e):
                if a == b or ((a % 2) == (b % 2)) != same:
                    continue
                d12 = X[:, a] - X[:, b]
                d1 = X[:, a] - system.nuc[I]
                r12 = np.linalg.norm(d12, axis=-1)
                r1 = np.linalg.norm(d1, axis=-1)
                r2 = np.linalg.norm(X[:, b] - system.nuc[I], axis=-1)
                m = ((r1 < L) & (r2 < L)).astype(np.float64)
                _, u1, u12, u11, u1212, u112 = _eeI_poly_derivs(g, r12, r1, r2, L)
                e1 = d1 / r1[:, None]
                e12 = d12 / r12[:, None]
                cos = np.sum(e1 * e12, axis=-1)
                grad[:, a] -= m[:, None] * (u1[:, None] * e1 + u12[:, None] * e12)
                lap[:, a] -= m * (u11 + 2.0 * u1 / r1 + u1212 + 2.0 * u12 / r12
                                  + 2.0 * u112 * cos)
    return grad, lap


def jastrow_value(system, X):
    """J1 + J2 (``gto.py:1500-1573``, Padé; ``1684-1780``, B-spline) + J3_eeI."""
    W, n_e, _ = X.shape
    J = np.zeros(W)
    if system.has_j2:
        i, j = _pairs(n_e)
        d = X[:, i] - X[:, j]
        r = np.sqrt(np.sum(d * d, axis=-1))
        same = (i % 2) == (j % 2)
        a = np.where(same, system.j2[0, 0], system.j2[1, 0])
        b = np.where(same, system.j2[0, 1], system.j2[1, 1])
        # like and unlike sums are separate in the reference
        u = a * r / (1.0 + b * r)
        J += np.sum(u * same, axis=-1) + np.sum(u * (~same), axis=-1)
    if system.has_j1:
        d = X[:, None, :, :] - system.nuc[None, :, None, :]
        r = np.sqrt(np.sum(d * d, axis=-1))            # (W, natm, n_e)
        a = system.j1[:, 0][None, :, None]
        b = system.j1[:, 1][None, :, None]
        J += np.sum(a * r / (1.0 + b * r), axis=(1, 2))
    bs2 = getattr(system, "bs2", None)
    if bs2 is not None:
        i, j = _pairs(n_e)
        d = X[:, i] - X[:, j]
        r = np.sqrt(np.sum(d * d, axis=-1))
        same = (i % 2) == (j % 2)
        u_l = bspline_vgl(bs2["like"], r, bs2["r_cut"])[0]
        u_u = bspline_vgl(bs2["unlike"], r, bs2["r_cut"])[0]
        J += np.sum(u_l * same, axis=-1) + np.sum(u_u * (~same), axis=-1)
    bs1 = getattr(system, "bs1", None)
    if bs1 is not None:
        for I, entry in enumerate(bs1):
            if entry is None:
                continue
            c, rc = entry
            d = X - system.nuc[I][None, None, :]
            r = np.sqrt(np.sum(d * d, axis=-1))
            J += np.sum(bspline_vgl(c, r, rc)[0], axis=-1)
    J += j3_value(system, X)
    return J


def jastrow_vgl(system, X):
    """Per-electron gradient and Laplacian of J1 + J2 (``gto.py:1575-1649``)."""
    W, n_e, _ = X.shape
    grad = np.zeros((W, n_e, 3))
    lap = np.zeros((W, n_e))
    if system.has_j2:
        i, j = _pairs(n_e)
        d = X[:, i] - X[:, j]
        r = np.sqrt(np.sum(d * d, axis=-1))
        same = (i % 2) == (j % 2)
        a = np.where(same, system.j2[0, 0], system.j2[1, 0])
        b = np.where(same, system.j2[0, 1], system.j2[1, 1])
        den = 1.0 + b * r
        up = a / (den * den)
        upp = -2.0 * a * b / (den * den * den)
        gp = (up / r)[..., None] * d
        lp = upp + 2.0 * up / r
        for k in range(len(i)):
            grad[:, i[k]] += gp[:, k]
            grad[:, j[k]] -= gp[:, k]
            lap[:, i[k]] += lp[:, k]
            lap[:, j[k]] += lp[:, k]
    if system.has_j1:
        d = X[:, :, None, :] - system.nuc[None, None, :, :]
        r = np.sqrt(np.sum(d * d, axis=-1))            # (W, n_e, natm)
        a = system.j1[:, 0][None, None, :]
        b = system.j1[:, 1][None, None, :]
        den = 1.0 + b * r
        up = a / (den * den)
        upp = -2.0 * a * b / (den * den * den)
        grad += np.sum((up / r)[..., None] * d, axis=2)
        lap += np.sum(upp + 2.0 * up / r, axis=2)
    bs2 = getattr(system, "bs2", None)
    if bs2 is not None:
        i, j = _pairs(n_e)
        d = X[:, i] - X[:, j]
        r = np.sqrt(np.sum(d * d, axis=-1))
        same = (i % 2) == (j % 2)
        _, ul, ull = bspline_vgl(bs2["like"], r, bs2["r_cut"])
        _, uu, uuu = bspline_vgl(bs2["unlike"], r, bs2["r_cut"])
        up = np.where(same, ul, uu)
        upp = np.where(same, ull, uuu)
        gp = (up / r)[..., None] * d
        lp = upp + 2.0 * up / r
        for k in range(len(i)):
            grad[:, i[k]] += gp[:, k]
            grad[:, j[k]] -= gp[:, k]
            lap[:, i[k]] += lp[:, k]
            lap[:, j[k]] += lp[:, k]
    bs1 = getattr(system, "bs1", None)
    if bs1 is not None:
        for I, entry in enumerate(bs1):
            if entry is None:
                continue
            c, rc = entry
            d = X - system.nuc[I][None, None, :]
            r = np.sqrt(np.sum(d * d, axis=-1))
            _, up, upp = bspline_vgl(c, r, rc)
            grad += (up / r)[..., None] * d
            lap += upp + 2.0 * up / r
    g3, l3 = j3_vgl(system, X)
    return grad + g3, lap + l3


# ---------------------------------------------------------------------------
# Energies
# ---------------------------------------------------------------------------
def e_ee(X):
    """sum_{i<j} 1/sqrt(r^2 + eps) (``gto.py:2406-2440``)."""
    n_e = X.shape[1]
    i, j = _pairs(n_e)
    d = X[:, i] - X[:, j]
    return np.sum(1.0 / np.sqrt(np.sum(d * d, axis=-1) + EPS), axis=-1)


def e_en(system, X):
    """-sum Z / sqrt(r^2 + eps) (``gto.py:2445-2451``)."""
    d = X[:, :, None, :] - system.nuc[None, None, :, :]
    return np.sum(-system.Z[None, None, :] / np.sqrt(np.sum(d * d, axis=-1) + EPS),
                  axis=(1, 2))


def log_psi(system, X):
    """log|psi| (``gto.py:2220-2254``)."""
    X = np.asarray(X, dtype=np.float64)
    return log_slater(system, X) + jastrow_value(system, X)


def evaluate(system, X):
    """Full per-walker evaluation.

    Returns a dict with ``logpsi`` (W,), ``grad`` (W, n_e, 3) =
    grad log|psi|, ``lap`` (W, n_e) = per-electron Laplacian of log|psi|,
    ``e_ee``, ``e_en``, ``e_ke`` and ``e_loc`` = ee + en + ke + nn, following
    ``local_energy_ke`` (``gto.py:2506-2579``) and ``_local_energy_batch``
    (``OmegaQMC/vmc_gto.py:801-812``)."""
    X = np.asarray(X, dtype=np.float64)
    if getattr(system, "md", None) is not None:
        _, gs, ls = multidet_assemble(system, X)
    else:
        mv, mg, ml = mo_vgl(system, X)
        _, gs, ls = slater_assemble(mv, mg, ml)
    gj, lj = jastrow_vgl(system, X)
    grad = gs + gj
    lap = ls + lj
    ke = -0.5 * (np.sum(lap, axis=-1) + np.sum(grad * grad, axis=(1, 2)))
    ee = e_ee(X)
    en = e_en(system, X)
    return {"logpsi": log_psi(system, X), "grad": grad, "lap": lap,
            "e_ee": ee, "e_en": en, "e_ke": ke,
            "e_loc": ee + en + ke + system.e_nn}


def local_energy(system, X):
    return evaluate(system, X)["e_loc"]


# ---------------------------------------------------------------------------
# Statistics: do_binning_analysis (OmegaQMC/utils.py:86-150)
# ---------------------------------------------------------------------------
def binning_analysis(a):
    """(mean, serr, sdev, kappa); kappa = 1 + 2 sum_{k>=1} ac_k summed until
    the first negative normalised autocorrelation."""
    a = np.asarray(a, dtype=np.float64)
    n = a.shape[0]
    xbar = a.mean()
    sdev = a.std()
    x = a - xbar
    nfft = 1 << int(math.ceil(math.log2(max(2 * n - 1, 1))))
    fx = np.fft.rfft(x, nfft)
    ac = np.fft.irfft(fx * np.conj(fx), nfft)[:n]
    if ac[0] == 0:
        return xbar, 0.0, sdev, 1.0
    ac = ac / ac[0]
    kappa = 1.0
    for k in range(1, n):
        if ac[k] < 0:
            break
        kappa += 2.0 * ac[k]
    serr = sdev * math.sqrt(kappa / n)
    return float(xbar), float(serr), float(sdev), float(kappa)


# ---------------------------------------------------------------------------
# Jastrow-parameter derivatives (the per-walker inputs of the linear-method
# optimiser, compute_walker_derivs, OmegaQMC/vmcopt_gto_linear.py:686-703)
# ---------------------------------------------------------------------------
def _pade_param_terms(a, b, r):
    """d/da, d/db of u = a r/(1+b r), of u' and of L = u'' + 2u'/r."""
    den = 1.0 + b * r
    du = (r / den, -a * r * r / den ** 2)
    dup = (1.0 / den ** 2, -2.0 * a * r / den ** 3)
    dupp = (-2.0 * b / den ** 3, -2.0 * a / den ** 3 + 6.0 * a * b * r / den ** 4)
    dL = tuple(dupp[k] + 2.0 * dup[k] / r for k in range(2))
    return du, dup, dL


def bspline_types(system):
    """Element symbols with a one-body B-spline, in order of first atom: the
    element types of the device tables and of the raw parameter layout."""
    out = []
    for ia, e in enumerate(getattr(system, "bs1", None) or []):
        if e is not None and system.symbols[ia] not in out:
            out.append(system.symbols[ia])
    return out


def _bspline_param_terms(c, r, r_cut):
    """Coefficient indices (i..i+3) and the weights of u, u', u'' on them."""
    n = len(c) - 4
    dinv = (n + 1) / r_cut
    x = r * dinv
    i = np.clip(np.floor(x).astype(np.int64), 0, n)
    t = x - i
    t2, t3 = t * t, t * t * t
    w = [(-t3 + 3 * t2 - 3 * t + 1) / 6, (3 * t3 - 6 * t2 + 4) / 6,
         (-3 * t3 + 3 * t2 + 3 * t + 1) / 6, t3 / 6]
    w1 = [v * dinv for v in ((-3 * t2 + 6 * t - 3) / 6, (9 * t2 - 12 * t) / 6,
                             (-9 * t2 + 6 * t + 3) / 6, 3 * t2 / 6)]
    w2 = [v * dinv * dinv for v in ((-6 * t + 6) / 6, (18 * t - 12) / 6, (-18 * t + 6) / 6,
                                    6 * t / 6)]
    m = r < r_cut
    return i, w, w1, w2, m, n


def _scatter_bspline(dl, de, base, n, i, w, w1, w2, m, r, gd, half):
    """Add the parameter derivatives of spline terms at distances r
    (flattened over walkers x terms, walker index wi) into dl/de rows.
    Parameter P_q is coefficient q+1; coefficient 0 = P_1 - 2 dr cusp."""
    W = dl.shape[0]
    for k in range(4):
        idx = i + k
        dL = w2[k] + 2.0 * w1[k] / r
        ce = (0.5 * (dL + 2.0 * w1[k] * gd)) if half else (dL + w1[k] * gd)
        for q in range(n):
            sel = ((idx == q + 1) | ((q == 1) & (idx == 0))) & m
            dl[:, base + q] += np.sum(np.where(sel, w[k], 0.0), axis=-1)
            de[:, base + q] -= np.sum(np.where(sel, ce, 0.0), axis=-1)


def param_count(system):
    """Raw parameters: Padé (4 + 2 natm), then the J2 B-spline like and
    unlike parameters, then the J1 B-spline parameters per element type,
    then the J3_eeI unique gammas per element type (like, unlike)."""
    n = 4 + 2 * system.natm
    bs2 = getattr(system, "bs2", None)
    if bs2 is not None:
        n += len(bs2["like"]) - 4 + len(bs2["unlike"]) - 4
    for sym in bspline_types(system):
        ia = system.symbols.index(sym)
        n += len(system.bs1[ia][0]) - 4
    n += sum(len(lmn) for _, _, lmn in _j3_raw_blocks(system))
    return n


def _j3_raw_blocks(system):
    """(element, same-spin flag, unique (l, m, n) list) of the J3 raw
    parameter blocks: element types in order of first atom, like then
    unlike, present blocks only."""
    j3 = getattr(system, "j3", None)
    if j3 is None:
        return []
    syms = list(system.symbols)
    elements = []
    for sym in syms:
        if sym not in elements and ("like+" + sym in j3["params"]
                                    or "unlike+" + sym in j3["params"]):
            elements.append(sym)
    _, lmn = eeI_constraint_map(j3["n_eI"], j3["n_ee"], j3["r_cut"])
    out = []
    for sym in elements:
        for prefix, same in (("like+", True), ("unlike+", False)):
            if prefix + sym in j3["params"]:
                out.append((sym, same, lmn))
    return out


def param_derivatives(system, X, grad=None):
    """Per-walker d log|psi| / dp and d E_L / dp for the raw parameters
    (``param_count``): Padé p = (J2 like a, like b, unlike a, unlike b, then J1
    a_I, b_I per atom), then the B-spline parameters.

    lnpsi depends on p only through J; E_L only through its kinetic part
    -1/2 sum_e (lap_e + |G_e|^2) with G_e the full gradient of ln|psi|
    (from ``evaluate`` unless given), so dE_L/dp = -1/2 sum_e (d lap_e/dp +
    2 G_e . dG_e/dp).  Terms absent from the system give zero columns."""
    X = np.asarray(X, dtype=np.float64)
    W, n_e, _ = X.shape
    if grad is None:
        grad = evaluate(system, X)["grad"]
    n_raw = param_count(system)
    dl = np.zeros((W, n_raw))
    de = np.zeros((W, n_raw))
    if system.has_j2:
        i, j = _pairs(n_e)
        d = X[:, i] - X[:, j]
        r = np.sqrt(np.sum(d * d, axis=-1))
        rhat = d / r[..., None]
        gdot = np.sum((grad[:, i] - grad[:, j]) * rhat, axis=-1)
        same = (i % 2) == (j % 2)
        for k, mask in ((0, same), (1, ~same)):
            a, b = system.j2[k]
            du, dup, dL = _pade_param_terms(a, b, r)
            for q in range(2):
                dl[:, 2 * k + q] = np.sum(du[q] * mask, axis=-1)
                de[:, 2 * k + q] = -np.sum((dL[q] + dup[q] * gdot) * mask, axis=-1)
    if system.has_j1:
        for I in range(system.natm):
            d = X - system.nuc[I][None, None, :]
            r = np.sqrt(np.sum(d * d, axis=-1))                 # (W, n_e)
            gdot = np.sum(grad * d, axis=-1) / r
            a, b = system.j1[I]
            du, dup, dL = _pade_param_terms(a, b, r)
            for q in range(2):
                dl[:, 4 + 2 * I + q] = np.sum(du[q], axis=-1)
                de[:, 4 + 2 * I + q] = -0.5 * np.sum(dL[q] + 2.0 * dup[q] * gdot, axis=-1)
    base = 4 + 2 * system.natm
    bs2 = getattr(system, "bs2", None)
    if bs2 is not None:
        i, j = _pairs(n_e)
        d = X[:, i] - X[:, j]
        r = np.sqrt(np.sum(d * d, axis=-1))
        gd = np.sum((grad[:, i] - grad[:, j]) * d, axis=-1) / r
        same = (i % 2) == (j % 2)
        for key, mask in (("like", same), ("unlike", ~same)):
            ii, w, w1, w2, m, n = _bspline_param_terms(bs2[key], r, bs2["r_cut"])
            _scatter_bspline(dl, de, base, n, ii, w, w1, w2, m & mask[None, :], r, gd, False)
            base += n
    for sym in bspline_types(system):
        for I, entry in enumerate(system.bs1):
            if entry is None or system.symbols[I] != sym:
                continue
            c, rc = entry
            d = X - system.nuc[I][None, None, :]
            r = np.sqrt(np.sum(d * d, axis=-1))
            gd = np.sum(grad * d, axis=-1) / r
            ii, w, w1, w2, m, n = _bspline_param_terms(c, r, rc)
            _scatter_bspline(dl, de, base, n, ii, w, w1, w2, m, r, gd, True)
        base += len(system.bs1[system.symbols.index(sym)][0]) - 4
    # J3 is linear in the gammas: the derivative by one unique gamma is the
    # J3 value / VGL with that gamma (and its (m, l, n) mirror) set to 1
    j3 = getattr(system, "j3", None)
    for sym, same, lmn in _j3_raw_blocks(system):
        atoms = [I for I in range(system.natm) if system.symbols[I] == sym]
        for (l, m, n) in lmn:
            g = np.zeros((j3["n_eI"] + 1, j3["n_eI"] + 1, j3["n_ee"] + 1))
            g[l, m, n] = g[m, l, n] = 1.0
            blocks = [(I, same, g) for I in atoms]
            dl[:, base] = j3_value(system, X, blocks)
            dg, dlap = j3_vgl(system, X, blocks)
            de[:, base] = -0.5 * np.sum(dlap + 2.0 * np.sum(grad * dg, axis=-1), axis=-1)
            base += 1
    return dl, de
