"""``get_psi_fun``: the reference's per-walker wavefunction surface on the GPU.

Mirrors ``OmegaQMC.psi.get_psi_fun`` (``OmegaQMC/psi/gto.py:2601-2621``):
it returns

    (log_psi, (E_ee, E_nn, E_en, E_ke), (get_psi_mo, get_psi_mo_partition_vg),
     (log_psi_C, ke_C))

with the reference's call signatures.  Each function accepts one walker
``(n_e, 3)`` or a batch ``(W, n_e, 3)`` as numpy arrays or torch tensors and
evaluates on the current CUDA device through the library's FP64 kernels;
numpy in gives numpy out (a float for a single walker), torch in gives CUDA
tensors.  Jastrow parameters (``curr_params``) and nuclear coordinates are
call-time arguments as in the reference; a device context is built (and
cached) for each distinct set.

Multi-determinant ``trial`` dicts evaluate through the library's FP64
multi-determinant kernels.  Not on this path: the MO-coefficient
(CPHF/force) variants, which raise ``NotImplementedError``.
"""
from __future__ import annotations

import copy
import hashlib
from typing import Any, Callable, NamedTuple

import numpy as np
import torch

from .context import GTOContext
from .system import build_system, Mole

__all__ = ["get_psi_fun", "VMCTrialState", "PsiGTO"]


class VMCTrialState(NamedTuple):
    """Container of a VMC trial wavefunction (``OmegaQMC/psi/__init__.py:24-44``)."""
    log_psi: Callable
    log_psi_C: Callable = None
    energy_fns: Any = None
    get_psi_mo: Callable = None
    ke_C: Callable = None


def _key(params, nuc):
    h = hashlib.sha1()
    for k in sorted(params or {}):
        v = params[k]
        h.update(k.encode())
        if isinstance(v, dict):
            for kk in sorted(v):
                h.update(kk.encode())
                h.update(np.ascontiguousarray(np.asarray(_np(v[kk]), dtype=np.float64)).tobytes())
        else:
            h.update(np.ascontiguousarray(np.asarray(_np(v), dtype=np.float64)).tobytes())
    h.update(np.ascontiguousarray(nuc, dtype=np.float64).tobytes())
    return h.hexdigest()


def _np(x):
    if torch.is_tensor(x):
        return x.detach().cpu().numpy()
    return np.asarray(x)


class _MolAt:
    """``mol`` with nuclei moved to given coordinates (bohr)."""

    def __init__(self, mol, nuc):
        self.__dict__.update(mol.__dict__)
        self._atom = [(s, tuple(float(c) for c in xyz))
                      for (s, _), xyz in zip(mol._atom, np.asarray(nuc))]


class PsiGTO:
    """Per-walker GTO Slater-Jastrow functions backed by the CUDA kernels."""

    def __init__(self, mf, params_cusp=None, trial=None, jastrow_config=None):
        self.trial = trial
        self.mf = mf
        self.params_cusp = params_cusp
        self.jastrow_config = jastrow_config
        self.nuc0 = np.asarray(mf.mol.atom_coords(unit="Bohr"), dtype=np.float64)
        self._ctx = {}

    # -- contexts -----------------------------------------------------------
    def context(self, params, nuc=None):
        nuc = self.nuc0 if nuc is None else np.asarray(_np(nuc), dtype=np.float64)
        k = _key(params, nuc)
        ctx = self._ctx.get(k)
        if ctx is None:
            mf = self.mf
            if not np.array_equal(nuc, self.nuc0):
                mf = copy.copy(self.mf)
                mf.mol = _MolAt(self.mf.mol, nuc)
            p = {kk: (dict(v) if isinstance(v, dict) else v) for kk, v in (params or {}).items()}
            for kk, v in p.items():
                if isinstance(v, dict):
                    p[kk] = {a: _np(b) for a, b in v.items()}
            system = build_system(mf, p, self.params_cusp, self.jastrow_config, self.trial)
            ctx = GTOContext(system)
            if len(self._ctx) > 16:
                self._ctx.clear()
            self._ctx[k] = ctx
        return ctx

    @staticmethod
    def _prep(elec):
        single = elec.ndim == 2
        return single, (elec[None] if single else elec)

    @staticmethod
    def _out(t, single, as_torch):
        if as_torch:
            return t[0] if single else t
        a = t.detach().cpu().numpy()
        return float(a[0]) if single and a.ndim == 1 else (a[0] if single else a)

    def _run(self, elec, nuc, params, key):
        as_torch = torch.is_tensor(elec)
        single, X = self._prep(elec)
        ctx = self.context(params, nuc)
        if key == "logpsi":
            r = ctx.log_psi(X)
        else:
            r = ctx.evaluate(X, want_grad=key == "grad", want_lap=False)[key]
        return self._out(r, single, as_torch)

    # -- the reference's functions -----------------------------------------
    def log_trial_wavefunction(self, elec_crds, nuc_crds, curr_params):
        """log|psi| (``gto.py:2220-2254``)."""
        return self._run(elec_crds, nuc_crds, curr_params, "logpsi")

    def local_energy_ee(self, elec_crds):
        """Electron-electron repulsion (``gto.py:2432-2437``)."""
        return self._run(elec_crds, None, {}, "e_ee")

    def local_energy_en(self, elec_crds, nuc_crds):
        """Electron-nucleus attraction (``gto.py:2445-2451``)."""
        return self._run(elec_crds, nuc_crds, {}, "e_en")

    def local_energy_ke(self, elec_crds, nuc_crds, curr_params):
        """Analytic kinetic energy (``gto.py:2506-2579``)."""
        return self._run(elec_crds, nuc_crds, curr_params, "e_ke")

    def local_energy_nn(self, nuc_crds):
        """Nuclear repulsion (``gto.py:2439-2443``), a setup-time constant."""
        nuc = np.asarray(_np(nuc_crds), dtype=np.float64)
        Z = self.mf.mol.atom_charges().astype(np.float64)
        eps = np.finfo(np.float64).eps
        e = 0.0
        for i in range(len(Z)):
            for j in range(i + 1, len(Z)):
                d = nuc[i] - nuc[j]
                e += Z[i] * Z[j] / np.sqrt(np.dot(d, d) + eps)
        return e

    def grad_log_psi(self, elec_crds, nuc_crds, curr_params):
        """grad log|psi| per electron (the ``grad_flat`` that ``local_energy_ke``
        builds, ``gto.py:2513-2575``), shape (…, n_e, 3)."""
        return self._run(elec_crds, nuc_crds, curr_params, "grad")

    def get_psi_mo(self, elec_crds, nuc_crds):
        """Occupied MO values (n_e, nocc) (``gto.py:1058-1070``); the second
        element (the per-atom s-shell partition used by forces) is None."""
        as_torch = torch.is_tensor(elec_crds)
        single, X = self._prep(elec_crds)
        mv = self.context({}, nuc_crds).mo_values(X)
        return self._out(mv, single, as_torch), None

    def get_psi_mo_partition_vg(self, elec_crds, nuc_crds):
        raise NotImplementedError("MO partitions are used only by the force "
                                  "estimators, which are not on this path")

    def log_trial_wavefunction_C(self, *a, **k):
        raise NotImplementedError("explicit-MO (CPHF) variants are not on this path")

    def local_energy_ke_C(self, *a, **k):
        raise NotImplementedError("explicit-MO (CPHF) variants are not on this path")


def get_psi_fun(mf, params_cusp=None, trial=None, jastrow_config=None):
    """Wavefunction and local-energy functions (``gto.py:2601-2621``)."""
    obj = PsiGTO(mf, params_cusp=params_cusp, trial=trial,
                 jastrow_config=jastrow_config)
    return (
        obj.log_trial_wavefunction,
        (obj.local_energy_ee, obj.local_energy_nn, obj.local_energy_en,
         obj.local_energy_ke),
        (obj.get_psi_mo, obj.get_psi_mo_partition_vg),
        (obj.log_trial_wavefunction_C, obj.local_energy_ke_C),
    )
