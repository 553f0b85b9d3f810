"""Generate golden vectors by running the reference's own wavefunction code.

Run where the reference checkout is available, naming it with ``--ref`` or
the ``OMEGAQMC_REF`` environment variable::

    python tests/golden/make_golden.py --ref <checkout> [--cases ...] [--verify]

A case whose fixture already exists is recomputed from the inputs stored in
that fixture (atoms, basis, cusp and Jastrow parameters, orbitals, trial,
walkers), so re-running the script reproduces every committed fixture
whatever the package's molecule builders do today; ``--fresh`` rebuilds the
inputs from the builders instead.  ``--verify`` recomputes and compares with
the stored outputs without writing.  The ``bench_*`` cases are the exact
trials the benchmark runs: the synthetic cc-pVDZ-shaped basis, RHF orbitals
from this package's SCF and the benchmark Jastrow (``h2o``, ``n2``), the
H2/STO-3G plain-method trial (Padé J2) and the LiH trial (Padé J1 + J2).

JAX and PySCF are not installed, so the reference modules
``OmegaQMC/psi/shell.py``, ``OmegaQMC/psi/gto.py`` and ``OmegaQMC/utils.py``
are imported unmodified from the checkout with ``jax_standin`` registered as
``jax`` (torch float64 underneath) and empty stand-ins for PySCF/h5py module
imports that the evaluation never calls.  The molecule is passed as a
duck-typed mean-field object built from this package's :class:`Mole`.

For each case the script stores the system specification (atoms, basis,
occupied MOs, Jastrow and cusp parameters), seeded walker configurations and
the reference's per-walker outputs: ``log_trial_wavefunction``,
``local_energy_ee/en/ke``, ``local_energy_nn``, the analytic gradient of
log|psi| (the ``grad_flat`` that ``local_energy_ke`` builds,
``gto.py:2513-2575``) and the per-electron Laplacian.  It also stores one
``do_binning_analysis`` result (``utils.py:86-150``) on a seeded series.
"""
from __future__ import annotations

import importlib
import json
import os
import sys
import types
import warnings

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

import jax_standin  # noqa: E402

jax_standin.install()
import torch  # noqa: E402

from omegaqmc_b200.system import Mole, MeanField, ELEMENT_Z  # noqa: E402
from omegaqmc_b200 import molecules as M  # noqa: E402

REF = os.environ.get("OMEGAQMC_REF")


def _stub(name, **attrs):
    m = types.ModuleType(name)
    for k, v in attrs.items():
        setattr(m, k, v)
    sys.modules[name] = m
    return m


def load_reference():
    """Import the reference's shell/gto/utils modules from the checkout."""
    if not REF or not os.path.isdir(os.path.join(REF, "OmegaQMC")):
        raise SystemExit("name the reference checkout with --ref or OMEGAQMC_REF")
    _stub("h5py")
    _stub("pyscf", __config__=types.SimpleNamespace(),
          gto=types.SimpleNamespace(Mole=type("Mole", (), {})))
    _stub("pyscf.gto", Mole=type("Mole", (), {}))
    _stub("pyscf.gto.basis", _format_basis_name=lambda s: s)
    _stub("pyscf.lib", logger=types.SimpleNamespace(), param=types.SimpleNamespace())
    _stub("pyscf.data")
    _stub("pyscf.data.elements", MASSES=[0.0] * 120, ELEMENTS_PROTON={},
          _atom_symbol=lambda s: s)
    pkg = types.ModuleType("OmegaQMC")
    pkg.__path__ = [os.path.join(REF, "OmegaQMC")]
    sys.modules["OmegaQMC"] = pkg
    psi = types.ModuleType("OmegaQMC.psi")
    psi.__path__ = [os.path.join(REF, "OmegaQMC", "psi")]
    sys.modules["OmegaQMC.psi"] = psi
    utils = importlib.import_module("OmegaQMC.utils")
    shell = importlib.import_module("OmegaQMC.psi.shell")
    gto = importlib.import_module("OmegaQMC.psi.gto")
    return gto, shell, utils


def load_point_groups():
    """The reference's OmegaQMC/symm/point_groups.py (numpy only)."""
    symm = types.ModuleType("OmegaQMC.symm")
    symm.__path__ = [os.path.join(REF, "OmegaQMC", "symm")]
    sys.modules["OmegaQMC.symm"] = symm
    return importlib.import_module("OmegaQMC.symm.point_groups")


# geometries (bohr) and charges for the canonical-frame fixture: asymmetric
# molecules, one already near its frame, one with a planar fragment, and a
# degenerate (linear) case
FRAME_CASES = [
    ([[0.1, -0.3, 0.2], [1.9, 0.4, -0.5], [-0.7, 1.6, 0.9], [0.3, -1.2, 2.4]], [8, 1, 9, 1]),
    ([[0.0, 0.0, 0.0], [2.1, 0.3, 0.0], [-0.6, 1.9, 0.4]], [6, 1, 8]),
    ([[1.0, 2.0, 3.0], [3.2, 2.4, 2.1], [0.2, 4.1, 3.3], [1.5, 0.2, 4.4], [2.5, 3.5, 0.9]],
     [6, 1, 1, 9, 17]),
    ([[0.0, 0.0, 0.0], [0.0, 0.0, 2.0], [0.0, 0.0, -3.1]], [1, 6, 7]),
]


def frame_fixture(pg):
    """Reference outputs of charge_inertia_axes for FRAME_CASES, each
    geometry also rotated and shifted."""
    rng = np.random.default_rng(5)
    out = {}
    for k, (xyz, q) in enumerate(FRAME_CASES):
        xyz = np.array(xyz, dtype=float)
        A = np.linalg.qr(rng.normal(size=(3, 3)))[0]
        if np.linalg.det(A) < 0:
            A[:, 0] *= -1
        for tag, c in (("a", xyz), ("b", xyz @ A.T + rng.normal(size=3))):
            r = pg.charge_inertia_axes(c, np.array(q))
            out[f"coords_{k}{tag}"] = c
            out[f"charges_{k}{tag}"] = np.array(q)
            if r is None:
                out[f"none_{k}{tag}"] = np.array(1)
            else:
                out[f"centre_{k}{tag}"] = np.asarray(r[0])
                out[f"axes_{k}{tag}"] = np.asarray(r[1])
    return out


class _RefMole:
    """Adapter exposing this package's Mole with tensor charges."""

    def __init__(self, mol):
        self._m = mol
        self._atom = mol._atom
        self._basis = mol._basis
        self.natm = mol.natm
        self.basis = mol.basis
        self.elements = mol.elements
        self.charge = mol.charge
        self.ao_radial_transform = getattr(mol, "ao_radial_transform", None)

    def atom_charges(self):
        return torch.tensor(self._m.atom_charges(), dtype=torch.int64)

    def tot_electrons(self):
        return self._m.tot_electrons()

    def atom_symbol(self, i):
        return self._m.atom_symbol(i)

    def atom_coords(self, unit="Bohr"):
        return self._m.atom_coords(unit)


class _RefMF:
    def __init__(self, mf):
        self.mol = _RefMole(mf.mol)
        self.mo_coeff = torch.tensor(mf.mo_coeff)
        self.mo_occ = mf.mo_occ


def _walkers(mol, n, sigma, seed):
    rng = np.random.default_rng(seed)
    Z = mol.atom_charges()
    idx = np.repeat(np.arange(mol.natm), Z)
    nuc = mol.atom_coords()
    return nuc[idx][None] + sigma * rng.standard_normal((n, len(idx), 3))


def _to_json(obj):
    if isinstance(obj, dict):
        return {k: _to_json(v) for k, v in obj.items()}
    if isinstance(obj, (list, tuple)):
        return [_to_json(v) for v in obj]
    if isinstance(obj, np.ndarray):
        return obj.tolist()
    if isinstance(obj, (np.floating, np.integer)):
        return obj.item()
    return obj


def _with_splines(mol, transform):
    mol.ao_radial_transform = transform
    return mol


def _j3_params(syms, npar, seed):
    """Seeded J3_eeI free parameters (scale 0.05, as the reference's test
    ``_eeI_params``, tests/test_gto_jastrow.py:374-381)."""
    rng = np.random.default_rng(seed)
    return {p + s: rng.normal(size=npar) * 0.05 for s in syms for p in ("like+", "unlike+")}


def fg_test_system():
    """Small system whose basis has f and g shells (am 3, 4)."""
    basis = {
        "Be": [[0, [40.0, 0.3, -0.1], [8.0, 0.6, -0.2], [1.5, 0.3, 0.7]],
               [1, [3.0, 0.4], [0.7, 0.7]],
               [2, [1.1, 1.0]],
               [3, [0.9, 1.0]],
               [4, [0.8, 1.0]]],
        "H": [[0, [5.0, 0.2], [0.9, 0.6], [0.25, 0.4]], [1, [0.7, 1.0]]],
    }
    atoms = [("Be", (0.0, 0.1, -0.3)), ("H", (0.2, -0.1, 2.4)),
             ("H", (-0.3, 0.2, -2.9))]
    return Mole(atoms, basis)


CASES = {
    # name: (mol builder, use cusp, params builder, sigma, n walkers)
    "h2_sto3g": (lambda: M.named_system("H2"), False,
                 lambda mol: {"J2_pade": {"like": np.array([0.25, 1.0]),
                                          "unlike": np.array([0.5, 1.0])}},
                 0.5, 24),
    "h2o_nocusp": (lambda: M.named_system("H2O"), False,
                   lambda mol: {"J1_pade": {"O": np.array(0.9), "H": np.array(0.4)},
                                "J2_pade": {"like": np.array([0.25, 0.6]),
                                            "unlike": np.array([0.5, 0.4])}},
                   0.6, 24),
    "h2o_cusp": (lambda: M.named_system("H2O"), True,
                 lambda mol: {"J1_pade": {"O": np.array([-0.4, 0.9]),
                                          "H": np.array([-0.1, 0.5])},
                              "J2_pade": {"like": np.array([0.25, 1.0]),
                                          "unlike": np.array([0.5, 1.0])}},
                 0.6, 24),
    "lih_cusp": (lambda: M.named_system("LiH"), True,
                 lambda mol: {"J2_pade": {"like": np.array([0.25, 0.8]),
                                          "unlike": np.array([0.5, 0.8])}},
                 1.0, 16),
    "n2_nocusp": (lambda: M.named_system("N2"), False,
                  lambda mol: {"J1_pade": {"N": np.array(1.1)},
                               "J2_pade": {"like": np.array([0.25, 1.0]),
                                           "unlike": np.array([0.5, 1.0])}},
                  0.7, 8),
    "fg_shells": (fg_test_system, True,
                  lambda mol: {"J1_pade": {"Be": np.array([-0.3, 0.8]),
                                           "H": np.array([-0.05, 0.6])},
                               "J2_pade": {"like": np.array([0.25, 0.7]),
                                           "unlike": np.array([0.5, 0.7])}},
                  0.8, 12),
    "nojastrow": (lambda: M.named_system("LiH"), False, lambda mol: {}, 1.0, 8),
    # B-spline one- and two-body Jastrows with short cutoffs (walkers cross
    # them), and B-spline summed with Padé at the default 10-bohr cutoff
    "h2o_bspline": (lambda: M.named_system("H2O"), False,
                    lambda mol: {"J1_bspline": {"O": np.array([0.3, -0.2, 0.1, 0.05, -0.02, 0.01]),
                                                "H": np.array([0.1, 0.05, -0.03, 0.02])},
                                 "J2_bspline": {"like": np.array([0.2, 0.1, 0.05, 0.02, 0.01]),
                                                "unlike": np.array([0.4, 0.25, 0.1, 0.05, 0.02,
                                                                    0.01])}},
                    1.1, 24),
    "lih_bspline_pade": (lambda: M.named_system("LiH"), True,
                         lambda mol: {"J2_pade": {"like": np.array([0.25, 1.0]),
                                                  "unlike": np.array([0.5, 1.0])},
                                      "J2_bspline": {"like": np.array([0.1, 0.05, 0.02, 0.01]),
                                                     "unlike": np.array([0.2, 0.1, 0.03])},
                                      "J1_bspline": {"Li": np.array([-0.3, -0.1, 0.05]),
                                                     "H": np.array([-0.1, 0.02])}},
                         1.0, 16),
    # J3_eeI three-body terms: default orders and cutoff (3, 3, 5 bohr) on
    # H2O with both spin blocks of both elements; orders 2, 2 and a 4-bohr
    # cutoff with only some blocks, on cusp-corrected LiH with Padé J1/J2
    "h2o_j3": (lambda: M.named_system("H2O"), False,
               lambda mol: {"J2_pade": {"like": np.array([0.25, 1.0]),
                                        "unlike": np.array([0.5, 1.0])},
                            "J3_eeI": _j3_params(("O", "H"), 26, seed=13)},
               0.7, 24),
    "lih_j3": (lambda: M.named_system("LiH"), True,
               lambda mol: {"J1_pade": {"Li": np.array([-0.3, 0.8]),
                                        "H": np.array([-0.1, 0.6])},
                            "J2_pade": {"like": np.array([0.25, 0.8]),
                                        "unlike": np.array([0.5, 0.8])},
                            "J3_eeI": {k: v for k, v in
                                       _j3_params(("Li", "H"), 8, seed=17).items()
                                       if k != "unlike+H"}},
               1.0, 16),
    # the quintic radial-spline AO transform (gto.py:141-240, 905-936):
    # default grid without cusp correction (every shell splined), and a
    # coarser grid with cusp-corrected s shells kept analytic
    "h2o_spline": (lambda: _with_splines(M.named_system("H2O"), True), False,
                   lambda mol: {"J1_pade": {"O": np.array(0.9), "H": np.array(0.4)},
                                "J2_pade": {"like": np.array([0.25, 0.6]),
                                            "unlike": np.array([0.5, 0.4])}},
                   0.6, 24),
    "lih_spline_cusp": (lambda: _with_splines(M.named_system("LiH"),
                                              {"npts": 401, "tol": 1e-8}), True,
                        lambda mol: {"J2_pade": {"like": np.array([0.25, 0.8]),
                                                 "unlike": np.array([0.5, 0.8])}},
                        1.0, 16),
    "h2o_md": (lambda: M.named_system("H2O"), False,
               lambda mol: {"J1_pade": {"O": np.array(0.9), "H": np.array(0.4)},
                            "J2_pade": {"like": np.array([0.25, 0.6]),
                                        "unlike": np.array([0.5, 0.4])}},
               0.6, 24),
    "lih_md_uhf": (lambda: M.named_system("LiH"), True,
                   lambda mol: {"J2_pade": {"like": np.array([0.25, 0.8]),
                                            "unlike": np.array([0.5, 0.8])}},
                   1.0, 16),
    # the benchmark's own trials (RHF orbitals, see RHF_CASES): H2O and N2
    # with the benchmark Jastrow (Padé J2, b = 3, no J1); the H2/STO-3G
    # plain-method trial (J2 b = 1); the LiH trial (Padé J1 with a = -Z and
    # J2, b = 1)
    "bench_h2o": (lambda: M.named_system("H2O"), False, M.benchmark_params_corr, 1.0, 24),
    "bench_n2": (lambda: M.named_system("N2"), False, M.benchmark_params_corr, 1.0, 16),
    "bench_h2": (lambda: M.named_system("H2"), False,
                 lambda mol: M.default_params_corr(mol, j1=False), 0.5, 24),
    "bench_lih": (lambda: M.named_system("LiH"), False, M.default_params_corr, 1.0, 24),
}

# cases whose orbitals come from this package's RHF (the others use seeded
# orbitals)
RHF_CASES = {"bench_h2o": "H2O", "bench_n2": "N2", "bench_h2": "H2", "bench_lih": "LiH"}

# B-spline cutoffs and J3 orders per case (jastrow_config of _PsiGTO,
# gto.py:948-984)
JASTROW_CONFIG = {
    "h2o_bspline": {"J2": {"r_cut": 4.0},
                    "J1": {"O": {"r_cut": 3.5}, "H": {"r_cut": 3.0}}},
    "lih_j3": {"J3": {"N_eI": 2, "N_ee": 2, "r_cut": 4.0}},
}

# multi-determinant trials (trial dicts of OmegaQMC/psi/trial.py): a
# restricted expansion on H2O (6 terms, 8 orbitals) and a UHF expansion on
# cusp-corrected LiH (alpha and beta orbitals differ)
def _trial_h2o(mf, seed):
    rng = np.random.default_rng(seed)
    C = np.asarray(mf.mo_coeff)
    mo = np.concatenate([C, rng.normal(size=(C.shape[0], 3)) * 0.3], axis=1)
    g, s1, s2, s3 = [0, 1, 2, 3, 4], [0, 1, 2, 3, 5], [0, 1, 2, 4, 6], [0, 1, 2, 3, 7]
    up = [g, s1, g, s2, s1, g]
    dn = [g, g, s1, s2, s2, s3]
    ci = [0.95, -0.12, -0.12, 0.08, 0.05, 0.03]
    return {"mo_coeff": mo, "ci_coeffs": np.array(ci), "occ_up": np.array(up),
            "occ_dn": np.array(dn), "ndet": len(ci)}


def _trial_lih_uhf(mf, seed):
    rng = np.random.default_rng(seed)
    C = np.asarray(mf.mo_coeff)
    n = C.shape[0]
    a = np.concatenate([C, rng.normal(size=(n, 2)) * 0.3], axis=1)
    b = np.concatenate([C + rng.normal(size=C.shape) * 0.02, rng.normal(size=(n, 2)) * 0.3],
                       axis=1)
    up = [[0, 1], [0, 2], [0, 3], [0, 1]]
    dn = [[0, 1], [0, 1], [0, 2], [1, 3]]
    ci = [0.9, 0.2, -0.15, 0.1]
    return {"mo_coeff": np.stack([a, b]), "ci_coeffs": np.array(ci), "occ_up": np.array(up),
            "occ_dn": np.array(dn), "ndet": len(ci)}


TRIALS = {"h2o_md": _trial_h2o, "lih_md_uhf": _trial_lih_uhf}

# (N_eI, N_ee, r_cut) of the stored J3_eeI constraint maps
EEI_MAPS = [(3, 3, 5.0), (2, 2, 4.0), (2, 3, 6.0), (4, 3, 5.0), (1, 2, 3.0)]


def _json_params(d):
    if d is None:
        return None
    out = {}
    for k, v in d.items():
        if isinstance(v, dict):
            out[k] = {kk: np.asarray(vv, dtype=np.float64) for kk, vv in v.items()}
        else:
            out[k] = np.asarray(v, dtype=np.float64)
    return out


def stored_inputs(name):
    """The inputs stored in an existing fixture, or None."""
    path = os.path.join(HERE, f"golden_{name}.npz")
    if not os.path.exists(path):
        return None
    d = dict(np.load(path))
    spec = json.loads(str(d["spec"]))
    mol = Mole([(a[0], tuple(a[1])) for a in spec["atoms"]], spec["basis"], unit="Bohr")
    if spec.get("ao_splines") is not None:
        mol.ao_radial_transform = spec["ao_splines"]
    mf = M.MeanField(mol, d["mo_coeff"], d["mo_occ"])
    pcusp = spec["cusp"]
    if pcusp is not None:
        pcusp = {k: {"q0": v["q0"], "coeff": np.asarray(v["coeff"])} for k, v in pcusp.items()}
    trial = None
    if "trial_ci" in d:
        trial = {"mo_coeff": d["trial_mo_coeff"], "ci_coeffs": d["trial_ci"],
                 "occ_up": d["trial_occ_up"], "occ_dn": d["trial_occ_dn"],
                 "ndet": len(d["trial_ci"])}
    return (mol, mf, _json_params(spec["params_corr"]), pcusp, d["X"],
            spec.get("jastrow_config"), trial), d


def built_inputs(name, seed):
    """Inputs of a case from the package's builders."""
    mk, cusp, mkp, sigma, nw = CASES[name]
    mol = mk()
    if name in RHF_CASES:
        ref = M.make_mf(RHF_CASES[name])
        mf = M.MeanField(mol, ref.mo_coeff, ref.mo_occ)
    else:
        mf = M.MeanField(mol, M.seeded_mo_coeff(mol, seed=seed))
    params = mkp(mol)
    pcusp = M.synthetic_cusp_params(mol, seed=seed + 11) if cusp else None
    X = _walkers(mol, nw, sigma, seed + 101)
    jcfg = JASTROW_CONFIG.get(name)
    trial = TRIALS[name](mf, seed + 31) if name in TRIALS else None
    return mol, mf, params, pcusp, X, jcfg, trial


def run_case(gto, inputs):
    mol, mf, params, pcusp, X, jcfg, trial = inputs
    cusp = pcusp is not None
    nw = len(X)
    rmf = _RefMF(mf)
    ref_trial = None
    if trial is not None:
        ref_trial = {"mo_coeff": trial["mo_coeff"],
                     "ci_coeffs": torch.tensor(trial["ci_coeffs"]),
                     "occ_up": torch.tensor(trial["occ_up"], dtype=torch.int64),
                     "occ_dn": torch.tensor(trial["occ_dn"], dtype=torch.int64),
                     "ndet": trial["ndet"]}
    obj = gto._PsiGTO(rmf, params_cusp=(
        {s: {"q0": torch.tensor(v["q0"]), "coeff": torch.tensor(v["coeff"])}
         for s, v in pcusp.items()} if cusp else None), trial=ref_trial, jastrow_config=jcfg)
    nuc = torch.tensor(mol.atom_coords())
    tp = {}
    for k, v in params.items():
        if isinstance(v, dict):
            tp[k] = {kk: torch.tensor(np.asarray(vv, dtype=np.float64))
                     for kk, vv in v.items()}
    out = {k: [] for k in ("logpsi", "e_ee", "e_en", "e_ke", "grad", "lap")}
    for w in range(nw):
        x = torch.tensor(X[w])
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")
            lp = obj.log_trial_wavefunction(x, nuc, tp)
            ke = obj.local_energy_ke(x, nuc, tp)
            _, gs, ls = obj._log_slater_analytic(x, nuc)
            grad = gs.reshape(-1)
            lap = ls
            if "J1_pade" in tp:
                g, L = obj._J1_pade_vgl(x, nuc, tp["J1_pade"])
                grad = grad + g.reshape(-1)
                lap = lap + L
            if "J2_pade" in tp:
                g, L = obj._J2_pade_vgl(x, tp["J2_pade"])
                grad = grad + g.reshape(-1)
                lap = lap + L
            if "J1_bspline" in tp:
                g, L = obj._J1_bspline_vgl(x, nuc, tp["J1_bspline"])
                grad = grad + g.reshape(-1)
                lap = lap + L
            if "J2_bspline" in tp:
                for fn in (obj._J2_bspline_aa_vgl, obj._J2_bspline_ab_vgl):
                    g, L = fn(x, tp["J2_bspline"])
                    grad = grad + g.reshape(-1)
                    lap = lap + L
            if "J3_eeI" in tp:
                g, L = obj._J3_eeI_vgl(x, nuc, tp["J3_eeI"])
                grad = grad + g.reshape(-1)
                lap = lap + L
        out["logpsi"].append(float(lp))
        out["e_ke"].append(float(ke))
        out["e_ee"].append(float(obj.local_energy_ee(x)))
        out["e_en"].append(float(obj.local_energy_en(x, nuc)))
        out["grad"].append(grad.detach().numpy().reshape(-1, 3))
        out["lap"].append(lap.detach().numpy())
    e_nn = float(obj.local_energy_nn(nuc))
    # the autodiff-Hessian kinetic energy on the first walkers
    ke_h = []
    for w in range(min(3, nw)):
        x = torch.tensor(X[w])
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")
            ke_h.append(float(obj._local_energy_ke_hessian(x, nuc, tp)))
    spec = {"atoms": mol._atom, "basis": mol._basis, "cusp": pcusp,
            "params_corr": params, "jastrow_config": jcfg,
            "ao_splines": getattr(mol, "ao_radial_transform", None)}
    res = {k: np.array(v) for k, v in out.items()}
    res.update(X=X, mo_coeff=mf.mo_coeff, mo_occ=mf.mo_occ, e_nn=e_nn,
               e_ke_hessian=np.array(ke_h),
               spec=np.array(json.dumps(_to_json(spec))))
    if trial is not None:
        res.update(trial_mo_coeff=trial["mo_coeff"], trial_ci=trial["ci_coeffs"],
                   trial_occ_up=trial["occ_up"], trial_occ_dn=trial["occ_dn"])
    return res


def main():
    import argparse
    ap = argparse.ArgumentParser()
    ap.add_argument("--cases", nargs="*", default=None,
                    help="generate only these cases (default: all, plus binning and cusp)")
    ap.add_argument("--ref", default=None, help="the reference checkout (or OMEGAQMC_REF)")
    ap.add_argument("--fresh", action="store_true",
                    help="build inputs from the package's builders even where a fixture exists")
    ap.add_argument("--verify", action="store_true",
                    help="recompute from the stored inputs and compare; write nothing")
    args = ap.parse_args()
    global REF
    REF = args.ref or REF
    gto, shell, utils = load_reference()
    os.makedirs(HERE, exist_ok=True)
    worst = 0.0
    for k, name in enumerate(CASES):
        if args.cases is not None and name not in args.cases:
            continue
        stored = None if args.fresh else stored_inputs(name)
        if args.verify and stored is None:
            print(f"{name}: no fixture to verify")
            continue
        inputs = stored[0] if stored is not None else built_inputs(name, seed=k)
        res = run_case(gto, inputs)
        if args.verify:
            d = stored[1]
            diff = max(float(np.max(np.abs(res[q] - d[q]) / (np.abs(d[q]) + 1.0)))
                       for q in ("logpsi", "e_ee", "e_en", "e_ke", "grad", "lap"))
            worst = max(worst, diff)
            print(f"{name}: max relative difference to the fixture {diff:.3e}")
            continue
        np.savez_compressed(os.path.join(HERE, f"golden_{name}.npz"), **res)
        print(f"{name}: {len(res['logpsi'])} walkers, logpsi[0]={res['logpsi'][0]:.12f}")
    if args.verify:
        print(f"worst {worst:.3e}")
        return
    if args.cases is None or "frame" in args.cases:
        np.savez_compressed(os.path.join(HERE, "golden_frame.npz"),
                            **frame_fixture(load_point_groups()))
        print("frame fixture:", len(FRAME_CASES), "geometries")
    if args.cases is None or "eeI_map" in args.cases:
        maps = {}
        for n_ei, n_ee, rc in EEI_MAPS:
            A, ls, ms, ns = gto._build_eeI_constraint_map(n_ei, n_ee, rc)
            key = f"{n_ei}_{n_ee}_{rc:g}"
            maps["A_" + key] = np.asarray(A)
            maps["lmn_" + key] = np.stack([np.asarray(ls), np.asarray(ms), np.asarray(ns)], 1)
        np.savez_compressed(os.path.join(HERE, "golden_eeI_map.npz"), **maps)
        print("eeI maps:", ", ".join(sorted(k for k in maps if k.startswith("A_"))))
    if args.cases is not None:
        return
    # binning analysis on a seeded AR(1) series
    rng = np.random.default_rng(42)
    x = np.zeros(2000)
    for i in range(1, 2000):
        x[i] = 0.8 * x[i - 1] + rng.standard_normal()
    xbar, serr, sdev, kappa = utils.do_binning_analysis(torch.tensor(x))
    np.savez_compressed(os.path.join(HERE, "golden_binning.npz"), series=x,
                        result=np.array([float(xbar), float(serr), float(sdev),
                                         float(kappa)]))
    # the cusp-s value at the radii the reference's sharding test uses
    rng = np.random.default_rng(0)
    coeff = rng.normal(size=8)
    rs = np.array([0.0, 0.03, 0.11, 0.2, 0.5])
    vals = [float(shell.evaluate_cusp_s(torch.tensor(r), 0.25, 8.0, 0.7, 1.3,
                                        torch.tensor(coeff))) for r in rs]
    # VGL at radii inside and outside rc
    rv = np.array([0.013, 0.05, 0.12, 0.19, 0.31])
    vgl = []
    for r in rv:
        f, fp, fl = shell.evaluate_cusp_s_vgl(torch.tensor(r), 0.2, 8.0, 0.7, -1.1,
                                              3.3, 1.3, torch.tensor(coeff))
        vgl.append([float(f), float(fp), float(fl)])
    np.savez_compressed(os.path.join(HERE, "golden_cusp.npz"), coeff=coeff,
                        r=rs, val=np.array(vals), r_vgl=rv, vgl=np.array(vgl))
    print("binning kappa", float(kappa))


if __name__ == "__main__":
    main()
