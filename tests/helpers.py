"""Shared test helpers: load golden fixtures and build systems from them."""
from __future__ import annotations

import glob
import json
import os

import numpy as np

from omegaqmc_b200.system import Mole, MeanField, build_system

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden_cases():
    out = []
    for p in sorted(glob.glob(os.path.join(GOLDEN, "golden_*.npz"))):
        name = os.path.basename(p)[len("golden_"):-4]
        if name in ("binning", "cusp", "eeI_map", "frame"):
            continue
        out.append(name)
    return out


def _params(d):
    if d is None:
        return None
    out = {}
    for k, v in d.items():
        if isinstance(v, dict):
            out[k] = {kk: np.asarray(vv, dtype=np.float64) for kk, vv in v.items()}
        else:
            out[k] = np.asarray(v, dtype=np.float64)
    return out


def load_golden(name):
    """(mf, params_corr, params_cusp, data) of a golden case."""
    d = dict(np.load(os.path.join(GOLDEN, f"golden_{name}.npz")))
    spec = json.loads(str(d["spec"]))
    atoms = [(a[0], tuple(a[1])) for a in spec["atoms"]]
    mol = Mole(atoms, spec["basis"], unit="Bohr")
    mol.ao_radial_transform = spec.get("ao_splines")
    mf = MeanField(mol, d["mo_coeff"], d["mo_occ"])
    params = _params(spec["params_corr"])
    cusp = spec["cusp"]
    if cusp is not None:
        cusp = {s: {"q0": v["q0"], "coeff": np.asarray(v["coeff"])}
                for s, v in cusp.items()}
    return mf, params, cusp, d


def golden_trial(d):
    """The multi-determinant trial dict stored with a golden case, or None."""
    if "trial_ci" not in d:
        return None
    return {"mo_coeff": d["trial_mo_coeff"], "ci_coeffs": d["trial_ci"],
            "occ_up": d["trial_occ_up"], "occ_dn": d["trial_occ_dn"]}


def golden_system(name):
    mf, params, cusp, d = load_golden(name)
    spec = json.loads(str(d["spec"]))
    return build_system(mf, params, cusp, spec.get("jastrow_config"), golden_trial(d)), d


def seeded_walkers(system, n, sigma, seed):
    """Walkers with electrons assigned to nuclei by charge, N(nucleus, sigma)."""
    rng = np.random.default_rng(seed)
    idx = np.repeat(np.arange(system.natm), system.Z.astype(int))
    return system.nuc[idx][None] + sigma * rng.standard_normal((n, len(idx), 3))
