"""Device context: a :class:`~omegaqmc_b200.system.System` uploaded to one GPU.

``GTOContext`` packs the system into the C ABI's ``oqmc_system_desc`` and
wraps every entry point with torch CUDA tensors as the buffers.  torch only
allocates device memory and provides streams; all arithmetic runs in the
library's kernels.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib as L
from .system import System

__all__ = ["GTOContext", "require_cuda"]


def require_cuda():
    if not torch.cuda.is_available():
        raise RuntimeError(
            "omegaqmc_b200 needs a CUDA device (sm_100a); there is no CPU path")


def _dptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)


def _stream_ptr(stream):
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def pack_system(system: System):
    """Arrays of the C descriptor (kept alive by the returned dict)."""
    groups = system.prim_groups()
    g_atom, g_am, g_np, g_nc, alpha, norm, cusp = [], [], [], [], [], [], []
    order = []
    for iat, a, shell_ids in groups:
        shs = [system.shells[i] for i in shell_ids]
        am = shs[0].am
        if any(s.am != am for s in shs):
            raise ValueError("mixed angular momenta in one basis entry")
        g_atom.append(iat)
        g_am.append(am)
        g_np.append(len(a))
        g_nc.append(len(shs))
        alpha.extend(a.tolist())
        for s in shs:
            norm.extend(s.norm.tolist())
            cusp.append(int(s.is_cusp))
            order.append(s)
    # the library numbers AOs group by group; check it matches the system
    ao = 0
    for s in order:
        if s.isgs != ao:
            raise ValueError("shell AO order does not follow exponent groups")
        ao += s.nsgs
    arr = {
        "nuc": np.ascontiguousarray(system.nuc, dtype=np.float64).ravel(),
        "Z": np.ascontiguousarray(system.Z, dtype=np.float64),
        "group_atom": np.array(g_atom, dtype=np.int32),
        "group_am": np.array(g_am, dtype=np.int32),
        "group_nprim": np.array(g_np, dtype=np.int32),
        "group_ncol": np.array(g_nc, dtype=np.int32),
        "alpha": np.array(alpha, dtype=np.float64),
        "norm": np.array(norm, dtype=np.float64),
        "shell_cusp": np.array(cusp, dtype=np.int32),
        "C": np.ascontiguousarray(system.C, dtype=np.float64).ravel(),
        "j1": np.ascontiguousarray(system.j1, dtype=np.float64).ravel(),
        "j2": np.ascontiguousarray(system.j2, dtype=np.float64).ravel(),
        "cusp_rc": np.ascontiguousarray(system.cusp_rc, dtype=np.float64),
        "cusp_q0": np.ascontiguousarray(system.cusp_q0, dtype=np.float64),
        "cusp_coeff": np.ascontiguousarray(system.cusp_coeff, dtype=np.float64).ravel(),
    }
    d = L.SystemDesc()
    d.natm = system.natm
    d.nbf = system.nbf
    d.nocc = system.nocc
    d.n_e = system.n_e
    d.ngroup = len(groups)
    d.has_j1 = int(system.has_j1)
    d.has_j2 = int(system.has_j2)
    d.cusp = int(system.cusp)
    d.e_nn = system.e_nn
    bs2 = getattr(system, "bs2", None)
    if bs2 is not None:
        arr["bs2_coef_like"] = np.ascontiguousarray(bs2["like"], dtype=np.float64)
        arr["bs2_coef_unlike"] = np.ascontiguousarray(bs2["unlike"], dtype=np.float64)
        d.has_bs2 = 1
        d.bs2_ncoef_like = arr["bs2_coef_like"].shape[0]
        d.bs2_ncoef_unlike = arr["bs2_coef_unlike"].shape[0]
        d.bs2_rcut = float(bs2["r_cut"])
    bs1 = getattr(system, "bs1", None)
    if bs1 is not None:
        # one table per element, in order of the element's first atom (the
        # raw parameter order of oqmc_param_derivs)
        syms = []
        for ia, entry in enumerate(bs1):
            if entry is not None and system.symbols[ia] not in syms:
                syms.append(system.symbols[ia])
        tables = [bs1[system.symbols.index(sym)] for sym in syms]
        arr["bs1_type"] = np.array([syms.index(system.symbols[ia]) if e is not None else -1
                                    for ia, e in enumerate(bs1)], dtype=np.int32)
        arr["bs1_ncoef"] = np.array([len(t[0]) for t in tables], dtype=np.int32)
        arr["bs1_rcut"] = np.array([t[1] for t in tables], dtype=np.float64)
        arr["bs1_coef"] = np.concatenate([np.asarray(t[0], dtype=np.float64) for t in tables])
        types = tables
        d.has_bs1 = 1
        d.bs1_ntype = len(types)
    j3 = getattr(system, "j3", None)
    if j3 is not None:
        arr["j3_type"] = np.array(j3["types"], dtype=np.int32)
        arr["j3_on"] = np.ascontiguousarray(j3["on"], dtype=np.int32).ravel()
        arr["j3_gamma"] = np.ascontiguousarray(j3["gamma"], dtype=np.float64).ravel()
        d.has_j3 = 1
        d.j3_n_ei = int(j3["n_eI"])
        d.j3_n_ee = int(j3["n_ee"])
        d.j3_ntype = len(j3["elements"])
        d.j3_rcut = float(j3["r_cut"])
    spl = getattr(system, "spl", None)
    if spl is not None and spl["tables"]:
        index = {id(sh): i for i, sh in enumerate(system.shells)}
        ids = sorted(spl["tables"])
        tab_of = {i: t for t, i in enumerate(ids)}
        arr["spl_shell"] = np.array([tab_of.get(index[id(sh)], -1) for sh in order],
                                    dtype=np.int32)
        arr["spl_knots"] = np.ascontiguousarray(
            np.stack([spl["tables"][i][0] for i in ids]), dtype=np.float64).ravel()
        arr["spl_coef"] = np.ascontiguousarray(
            np.stack([spl["tables"][i][1] for i in ids]), dtype=np.float64).ravel()
        d.has_spl = 1
        d.spl_npts = int(spl["npts"])
        d.spl_ntab = len(ids)
        d.spl_smin = float(spl["smin"])
    for k, v in arr.items():
        ct = ctypes.c_int if v.dtype == np.int32 else ctypes.c_double
        setattr(d, k, v.ctypes.data_as(ctypes.POINTER(ct)))
    return d, arr


class GTOContext:
    """One system on one CUDA device (the current one at construction)."""

    def __init__(self, system: System, device=None):
        require_cuda()
        self.lib = L.load()
        self.system = system
        self.device = torch.device("cuda", torch.cuda.current_device()
                                   if device is None else torch.device(device).index)
        self.n_e = system.n_e
        self.nocc = system.nocc
        desc, self._keep = pack_system(system)
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            code = self.lib.oqmc_create(ctypes.byref(h), ctypes.byref(desc))
        L.check(code, None)
        self._h = h
        if getattr(system, "md", None) is not None:
            self.set_multidet(system.md)

    # -- lifetime --------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self.lib.oqmc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, code):
        L.check(code, self._h)

    # -- helpers ----------------------------------------------------------
    def walkers_tensor(self, X):
        """(W, n_e, 3) float64 contiguous CUDA tensor on this device."""
        t = torch.as_tensor(X, dtype=torch.float64)
        if t.ndim == 2:
            t = t.unsqueeze(0)
        if t.ndim != 3 or t.shape[1] != self.n_e or t.shape[2] != 3:
            raise ValueError(f"walkers must be (W, {self.n_e}, 3), got {tuple(t.shape)}")
        return t.to(self.device).contiguous()

    def flags(self, clear=True, stream=None):
        f = ctypes.c_uint(0)
        self._check(self.lib.oqmc_get_flags(self._h, ctypes.byref(f), int(clear),
                                            _stream_ptr(stream)))
        return f.value

    # -- evaluation -----------------------------------------------------
    def evaluate(self, X, want_grad=True, want_lap=True, stream=None):
        """Full FP64 evaluation; returns a dict of CUDA tensors."""
        X = self.walkers_tensor(X)
        W = X.shape[0]
        opt = dict(dtype=torch.float64, device=self.device)
        logpsi = torch.empty(W, **opt)
        grad = torch.empty(W, self.n_e, 3, **opt) if want_grad else None
        lap = torch.empty(W, self.n_e, **opt) if want_lap else None
        ep = torch.empty(W, 4, **opt)
        self._check(self.lib.oqmc_eval(self._h, _dptr(X), W, _dptr(logpsi), _dptr(grad),
                                       _dptr(lap), _dptr(ep), _stream_ptr(stream)))
        out = {"logpsi": logpsi, "e_ee": ep[:, 0], "e_en": ep[:, 1], "e_ke": ep[:, 2],
               "e_loc": ep[:, 3]}
        if want_grad:
            out["grad"] = grad
        if want_lap:
            out["lap"] = lap
        return out

    def log_psi(self, X, stream=None):
        X = self.walkers_tensor(X)
        out = torch.empty(X.shape[0], dtype=torch.float64, device=self.device)
        self._check(self.lib.oqmc_log_psi(self._h, _dptr(X), X.shape[0], _dptr(out),
                                          _stream_ptr(stream)))
        return out

    def mo_values(self, X, stream=None):
        X = self.walkers_tensor(X)
        out = torch.empty(X.shape[0], self.n_e, self.nocc, dtype=torch.float64,
                          device=self.device)
        self._check(self.lib.oqmc_mo_values(self._h, _dptr(X), X.shape[0], _dptr(out),
                                            _stream_ptr(stream)))
        return out

    # -- sampler ------------------------------------------------------------
    def state_evaluate(self, state, W, precision, stream=None):
        """Outputs of a sampler state in its own precision (``oqmc_state_eval``):
        the tracked log|det| plus the Jastrow, the gradient and per-electron
        Laplacian of log|psi| from the state's inverse, and the local-energy
        parts; a dict of CUDA tensors keyed like :meth:`evaluate`."""
        opt = dict(dtype=torch.float64, device=self.device)
        W = int(W)
        logpsi = torch.empty(W, **opt)
        grad = torch.empty(W, self.n_e, 3, **opt)
        lap = torch.empty(W, self.n_e, **opt)
        ep = torch.empty(W, 4, **opt)
        self._check(self.lib.oqmc_state_eval(self._h, _dptr(state), W, int(precision),
                                             _dptr(logpsi), _dptr(grad), _dptr(lap),
                                             _dptr(ep), _stream_ptr(stream)))
        return {"logpsi": logpsi, "grad": grad, "lap": lap, "e_ee": ep[:, 0],
                "e_en": ep[:, 1], "e_ke": ep[:, 2], "e_loc": ep[:, 3]}

    def state_bytes(self, W, precision):
        return int(self.lib.oqmc_state_bytes(self._h, int(W), int(precision)))

    def new_state(self, W, precision):
        return torch.empty(self.state_bytes(W, precision), dtype=torch.uint8,
                           device=self.device)

    def refresh(self, X, state, precision, stream=None):
        self._check(self.lib.oqmc_refresh(self._h, _dptr(X), X.shape[0], _dptr(state),
                                          int(precision), _stream_ptr(stream)))

    def sweeps(self, X, state, precision, n_sweeps, step, seed, step_base, sums,
               measure_every=1, el_trace=None, eparts_last=None, walkers_per_block=0,
               stream=None):
        self._check(self.lib.oqmc_sweeps(
            self._h, _dptr(X), X.shape[0], _dptr(state), int(precision), int(n_sweeps),
            int(measure_every), float(step), ctypes.c_uint64(seed & (2**64 - 1)),
            ctypes.c_uint64(step_base), _dptr(sums), _dptr(el_trace), _dptr(eparts_last),
            int(walkers_per_block), _stream_ptr(stream)))

    def equilibrate(self, X, state, precision, n_steps, step, target, rate, seed, step_base,
                    refresh_every, since_refresh, acc_trace, step_trace=None, stream=None):
        """``oqmc_equilibrate``: n_steps sweeps with the step width (the
        one-element CUDA tensor ``step``) adapted on the device after each."""
        self._check(self.lib.oqmc_equilibrate(
            self._h, _dptr(X), X.shape[0], _dptr(state), int(precision), int(n_steps),
            _dptr(step), float(target), float(rate), ctypes.c_uint64(seed & (2**64 - 1)),
            ctypes.c_uint64(step_base), int(refresh_every), int(since_refresh),
            _dptr(acc_trace), _dptr(step_trace), _stream_ptr(stream)))

    def basin(self, X, state, precision, n_steps, sigma, seed, step_base, acc_sum=None,
              stream=None):
        self._check(self.lib.oqmc_basin(
            self._h, _dptr(X), X.shape[0], _dptr(state), int(precision), int(n_steps),
            float(sigma), ctypes.c_uint64(seed & (2**64 - 1)), ctypes.c_uint64(step_base),
            _dptr(acc_sum), _stream_ptr(stream)))

    def specialize(self, enable=True):
        """Compile (NVRTC) and use kernels specialised to this system's basis
        and orbitals; raises NotImplementedError where NVRTC is unavailable."""
        self._check(self.lib.oqmc_specialize(self._h, int(enable)))

    def use_tensor_cores(self, enable=True):
        """Mixed-precision local energy with the MO contraction on tcgen05."""
        self._check(self.lib.oqmc_use_tensor_cores(self._h, int(enable)))

    def set_multidet(self, md):
        """Use a multi-determinant Slater part (``md`` from
        :func:`~omegaqmc_b200.system.parse_trial`, or None for the single
        determinant).  Evaluation and FP64 sampling follow the expansion."""
        if md is None:
            self._check(self.lib.oqmc_set_multidet(self._h, 0, 0, None, None, None, None))
            self._md_keep = None
            return
        C = np.ascontiguousarray(md["C"], dtype=np.float64)
        ci = np.ascontiguousarray(md["ci"], dtype=np.float64)
        up = np.ascontiguousarray(md["occ_up"], dtype=np.int32)
        dn = np.ascontiguousarray(md["occ_dn"], dtype=np.int32)
        pd, pi = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
        self._md_keep = (C, ci, up, dn)
        self._check(self.lib.oqmc_set_multidet(
            self._h, ci.shape[0], C.shape[1], C.ctypes.data_as(pd), ci.ctypes.data_as(pd),
            up.ctypes.data_as(pi), dn.ctypes.data_as(pi)))

    def multidet_info(self):
        """(terms, distinct up determinants, distinct down determinants,
        padded orbital columns); zeros for a single determinant."""
        v = [ctypes.c_int() for _ in range(4)]
        self._check(self.lib.oqmc_multidet_info(self._h, *[ctypes.byref(x) for x in v]))
        return tuple(x.value for x in v)

    def set_move_kind(self, kind):
        """0: single-electron sweeps (default); 1: the reference's all-electron
        steps (``metropolis_move_alle``), one proposal per sweep."""
        self._check(self.lib.oqmc_set_move_kind(self._h, int(kind)))

    def set_proposal(self, kind, r0=1.0, fmin_frac=0.05):
        """0: fixed-width Gaussian (reference); 1: nucleus-scaled width."""
        self._check(self.lib.oqmc_set_proposal(self._h, int(kind), float(r0), float(fmin_frac)))

    def set_mlp_proposal(self, mlp):
        """Propose moves with a trained :class:`~omegaqmc_b200.learned.MLPProposal`
        (``None`` restores the previous proposal).  Needs ``specialize()``;
        sweeps then run in mixed precision only."""
        self._mlp = mlp
        self._check(self.lib.oqmc_set_mlp_proposal(self._h, mlp._h if mlp is not None else None))

    def set_mlp_groups(self, groups):
        """128-walker groups per CTA of the learned-proposal sweep (2 or 4)."""
        self._check(self.lib.oqmc_set_mlp_groups(self._h, int(groups)))

    def set_split(self, tight_alpha):
        self._check(self.lib.oqmc_set_split(self._h, float(tight_alpha)))
