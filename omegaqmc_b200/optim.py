"""Inputs of the linear-method Jastrow optimiser, on the GPU.

The reference's optimiser (``_VMCOptDriverGTO_Linear``,
OmegaQMC/vmcopt_gto_linear.py) samples walkers, then for every walker needs
E_L, d ln|psi| / dp and d E_L / dp with respect to the flattened Jastrow
parameters (``compute_walker_derivs``, vmcopt_gto_linear.py:686-703, by
``jax.grad``), and builds the overlap and Hamiltonian matrices of the
linear method from them (``_build_matrices``, vmcopt_gto_linear.py:466-520).
Here the per-walker quantities come from the library (``oqmc_eval`` for E_L
and the gradient of ln|psi|, ``oqmc_param_derivs`` for the analytic Padé
parameter derivatives) and the matrices are formed on the host.

Parameter order: ``flatten_params`` follows the reference's pytree
flattening (``_flatten_params``, vmcopt_gto_linear.py:37-52): dictionary keys
in sorted order ("J1_pade" before "J2_pade", element symbols sorted, "like"
before "unlike"), each entry flattened in place ([a, b] -> a, b; a bare b ->
b).  A J1 entry [a, b] without cusp correction keeps a = -Z, so its a
derivative is 0, as in the reference where that a is ignored.
"""
from __future__ import annotations

import numpy as np
import torch

from .context import GTOContext, _dptr, _stream_ptr
from .system import eeI_constraint_map

__all__ = ["flatten_params", "raw_to_flat", "walker_derivatives", "build_matrices"]


def flatten_params(params_corr):
    """(flat parameter vector, layout) of a ``params_corr`` dict; layout is a
    list of (term, key, length) in flattening order."""
    flat, layout = [], []
    for term in sorted(params_corr):
        sub = params_corr[term]
        for key in sorted(sub):
            v = np.ravel(np.asarray(sub[key], dtype=np.float64))
            layout.append((term, key, int(v.size)))
            flat.extend(v.tolist())
    return np.array(flat, dtype=np.float64), layout


def raw_to_flat(raw, params_corr, system):
    """Map per-walker derivatives of the library's raw parameters (J2 like a,
    like b, unlike a, unlike b, then J1 a_I, b_I per atom; then the B-spline
    parameters: J2 like, J2 unlike, J1 per element in order of first atom;
    then the J3_eeI unique gammas per element type, like then unlike block)
    onto the flat parameter order; Padé J1 entries collect the atoms of
    their element, and J3 blocks go through the constraint matrix
    (d/dp = A^T d/dgamma, gamma_unique = A p)."""
    raw = np.asarray(raw)
    atom_symbols, cusp = list(system.symbols), system.cusp
    _, layout = flatten_params(params_corr)
    out = np.zeros((raw.shape[0], sum(n for _, _, n in layout)))
    # offsets of the B-spline blocks in the raw layout
    bs_off = {}
    b = 4 + 2 * system.natm
    if getattr(system, "bs2", None) is not None:
        nl, nu = len(system.bs2["like"]) - 4, len(system.bs2["unlike"]) - 4
        bs_off[("J2_bspline", "like")] = b
        bs_off[("J2_bspline", "unlike")] = b + nl
        b += nl + nu
    seen = []
    for ia, e in enumerate(getattr(system, "bs1", None) or []):
        if e is not None and atom_symbols[ia] not in seen:
            seen.append(atom_symbols[ia])
            bs_off[("J1_bspline", atom_symbols[ia])] = b
            b += len(e[0]) - 4
    j3 = getattr(system, "j3", None)
    j3_off, A3 = {}, None
    if j3 is not None:
        A3, lmn = eeI_constraint_map(j3["n_eI"], j3["n_ee"], j3["r_cut"])
        for t, sym in enumerate(j3["elements"]):
            for blk, prefix in enumerate(("like+", "unlike+")):
                if j3["on"][t][blk]:
                    j3_off[prefix + sym] = b
                    b += len(lmn)
    o = 0
    for term, key, n in layout:
        if term == "J3_eeI":
            if key in j3_off:
                ng = A3.shape[0]
                out[:, o:o + n] = raw[:, j3_off[key]:j3_off[key] + ng] @ A3
            o += n
            continue
        if term.endswith("_bspline"):
            if (term, key) in bs_off:
                out[:, o:o + n] = raw[:, bs_off[(term, key)]:bs_off[(term, key)] + n]
            o += n
            continue
        if term == "J2_pade":
            k = 0 if key == "like" else 2
            out[:, o] = raw[:, k]
            if n > 1:
                out[:, o + 1] = raw[:, k + 1]
        elif term == "J1_pade":
            atoms = [i for i, s in enumerate(atom_symbols) if s == key]
            da = sum(raw[:, 4 + 2 * i] for i in atoms) if atoms else 0.0
            db = sum(raw[:, 5 + 2 * i] for i in atoms) if atoms else 0.0
            if n == 1:
                out[:, o] = db
            else:
                out[:, o] = da if cusp else 0.0
                out[:, o + 1] = db
        o += n
    return out


def walker_derivatives(ctx: GTOContext, X, params_corr, stream=None):
    """(E_L (W,), d ln|psi|/dp (W, P), dE_L/dp (W, P)) in the flat parameter
    order, for walkers X (W, n_e, 3), evaluated in FP64 on the GPU."""
    X = ctx.walkers_tensor(X)
    W = X.shape[0]
    ev = ctx.evaluate(X, want_grad=True, want_lap=False, stream=stream)
    n_raw = int(ctx.lib.oqmc_param_count(ctx._h))
    ctx._check(min(n_raw, 0))
    dl = torch.empty(W, n_raw, dtype=torch.float64, device=ctx.device)
    de = torch.empty(W, n_raw, dtype=torch.float64, device=ctx.device)
    ctx._check(ctx.lib.oqmc_param_derivs(ctx._h, _dptr(X), W, _dptr(ev["grad"]), _dptr(dl),
                                         _dptr(de), _stream_ptr(stream)))
    dl_f = raw_to_flat(dl.cpu().numpy(), params_corr, ctx.system)
    de_f = raw_to_flat(de.cpu().numpy(), params_corr, ctx.system)
    return ev["e_loc"].cpu().numpy(), dl_f, de_f


def build_matrices(E_L, dlogpsi, dEL):
    """Overlap S and Hamiltonian H of the linear method for pure energy
    minimisation, (num_opt + 1) x (num_opt + 1), from per-walker samples
    (restates _build_matrices, OmegaQMC/vmcopt_gto_linear.py:466-520)."""
    E_L = np.asarray(E_L, dtype=np.float64)
    dlogpsi = np.asarray(dlogpsi, dtype=np.float64)
    dEL = np.asarray(dEL, dtype=np.float64)
    nw, n = dlogpsi.shape
    dD = dlogpsi - dlogpsi.mean(axis=0)[None, :]
    S = np.zeros((n + 1, n + 1))
    S[0, 0] = 1.0
    S[1:, 1:] = dD.T @ dD / nw
    H = np.zeros((n + 1, n + 1))
    H[0, 0] = E_L.mean()
    rhs = dEL + dD * E_L[:, None]
    H[0, 1:] = rhs.mean(axis=0)
    H[1:, 0] = (dD * E_L[:, None]).mean(axis=0)
    H[1:, 1:] = dD.T @ rhs / nw
    return H, S
