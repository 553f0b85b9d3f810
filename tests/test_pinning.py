"""CPU pins of the pieces that stand between the kernels and the reported
numbers: the C restatement (the CPU baseline and the reference arm of the
benchmark) against the reference's own outputs, the benchmark's exact
trials against their golden cases, the driver's copy of the reference's
binning analysis, and the driver's initial walkers.

The golden cases are reference outputs (``tests/golden/make_golden.py``
imports the reference's ``psi/gto.py`` unmodified); ``bench_h2o``,
``bench_n2``, ``bench_h2`` and ``bench_lih`` are the trials the benchmark
samples, built by the same package functions the benchmark calls.
"""
import json

import numpy as np
import pytest

from helpers import GOLDEN, golden_cases, golden_system
from oracle import cref
from oracle import gto_oracle as O
from omegaqmc_b200 import molecules as M
from omegaqmc_b200 import vmc
from omegaqmc_b200.sampler import init_walkers_ball
from omegaqmc_b200.system import Mole, MeanField, build_system

REL = 1e-10


def _ke_scale(d):
    """Scale of the kinetic-energy terms: near a node E_ke is a small
    difference of large terms, defined to FP64 only at this scale (as in the
    reference)."""
    return 0.5 * (np.sum(np.abs(d["lap"]), axis=1) + np.sum(d["grad"] ** 2, axis=(1, 2))) + 1.0


def _cref_cases():
    out = []
    for name in golden_cases():
        s, _ = golden_system(name)
        out.append(pytest.param(name, marks=() if cref.supports(s) else
                                pytest.mark.skip(reason="outside the C restatement")))
    return out


@pytest.mark.parametrize("name", _cref_cases())
def test_c_restatement_matches_reference_outputs(name):
    s, d = golden_system(name)
    lp, ep = cref.evaluate(s, d["X"], nthreads=2)
    assert np.max(np.abs(lp - d["logpsi"]) / (np.abs(d["logpsi"]) + 1)) < REL
    for k, key in enumerate(("e_ee", "e_en")):
        assert np.max(np.abs(ep[:, k] - d[key]) / (np.abs(d[key]) + 1)) < REL, key
    sc = _ke_scale(d)
    assert np.max(np.abs(ep[:, 2] - d["e_ke"]) / sc) < REL
    e_l = d["e_ee"] + d["e_en"] + d["e_ke"] + float(d["e_nn"])
    assert np.max(np.abs(ep[:, 3] - e_l) / sc) < REL


def test_c_restatement_refuses_terms_it_does_not_cover():
    s, d = golden_system("h2o_bspline")
    with pytest.raises(ValueError):
        cref.evaluate(s, d["X"])
    s, d = golden_system("h2o_md")
    with pytest.raises(ValueError):
        cref.run(s, np.ascontiguousarray(d["X"][:2]), 1, 0.1)


BENCH = {"bench_h2o": ("H2O", M.benchmark_params_corr),
         "bench_n2": ("N2", M.benchmark_params_corr),
         "bench_h2": ("H2", lambda mol: M.default_params_corr(mol, j1=False)),
         "bench_lih": ("LiH", M.default_params_corr)}


@pytest.mark.parametrize("name", sorted(BENCH))
def test_benchmark_trial_is_the_golden_case(name):
    """The system the benchmark builds (molecule, basis, RHF orbitals,
    Jastrow) is the one the reference evaluated for the golden case."""
    mol_name, params = BENCH[name]
    mf = M.make_mf(mol_name)
    s = build_system(mf, params(mf.mol))
    g, d = golden_system(name)
    np.testing.assert_allclose(s.nuc, g.nuc, rtol=0, atol=1e-14)
    np.testing.assert_allclose(s.C, g.C, rtol=0, atol=1e-10)
    assert (s.has_j1, s.has_j2) == (g.has_j1, g.has_j2)
    np.testing.assert_array_equal(s.j2, g.j2)
    np.testing.assert_array_equal(s.j1, g.j1)
    assert len(s.shells) == len(g.shells)
    for a, b in zip(s.shells, g.shells):
        assert (a.am, a.iat) == (b.am, b.iat)
        np.testing.assert_allclose(a.alpha, b.alpha, rtol=1e-15)
    # and the oracle evaluates the benchmark's system as the reference did
    o = O.evaluate(s, d["X"])
    assert np.max(np.abs(o["logpsi"] - d["logpsi"]) / (np.abs(d["logpsi"]) + 1)) < REL
    assert np.max(np.abs(o["e_loc"] - (d["e_ee"] + d["e_en"] + d["e_ke"] + float(d["e_nn"])))
                  / _ke_scale(d)) < REL


def test_driver_binning_analysis_matches_reference():
    """The driver's final mean, error bar and kappa come from
    ``vmc.binning_analysis``; the reference's do_binning_analysis
    (OmegaQMC/utils.py:86-150) gave the stored result on the stored series."""
    g = np.load(f"{GOLDEN}/golden_binning.npz")
    ours = np.array(vmc.binning_analysis(g["series"]))
    np.testing.assert_allclose(ours, g["result"], rtol=1e-12, atol=0)
    assert vmc.binning_analysis(np.full(16, 2.5)) == (2.5, 0.0, 0.0, 1.0)


def _mol(atoms, charge=0):
    basis = {"H": [[0, [1.0, 1.0]]], "O": [[0, [5.0, 1.0]], [1, [1.0, 1.0]]],
             "Li": [[0, [3.0, 1.0]], [0, [0.5, 1.0]]], "Ne": [[0, [9.0, 1.0]], [0, [2.5, 1.0]], [1, [2.0, 1.0]], [1, [0.6, 1.0]]]}
    return Mole(atoms, basis, unit="Bohr", charge=charge)


def _system(mol):
    n = (mol.tot_electrons()) // 2
    C = np.zeros((mol.nao, n))
    for k in range(n):
        C[k, k] = 1.0
    return build_system(MeanField(mol, C), {})


def _centres(system, charge):
    """Electron-to-atom assignment of _initialize_walkers
    (OmegaQMC/vmc_gto.py:86-96): Z electrons per atom in atom order; an
    anion's extra electrons on atom 0; a cation drops the last ones."""
    idx = [ia for ia, z in enumerate(system.Z.astype(int)) for _ in range(z)]
    if charge < 0:
        idx += [0] * (-charge)
    elif charge > 0:
        idx = idx[:-charge]
    return system.nuc[np.array(idx)]


@pytest.mark.parametrize("charge", [0, 2, -2])
def test_initial_walkers_follow_reference_rule_molecule(charge):
    """Molecules: offsets uniform in a ball of radius 0.4 x the shortest
    internuclear distance about the assigned centre
    (OmegaQMC/vmc_gto.py:100-110)."""
    atoms = [("O", (0.0, 0.0, 0.0)), ("H", (0.0, 1.43, 1.11)), ("H", (0.0, -1.43, 1.11))]
    s = _system(_mol(atoms, charge))
    W = 20000
    X = init_walkers_ball(s, W, seed=5)
    cen = _centres(s, charge)
    assert X.shape == (W, s.n_e, 3) == (W, len(cen), 3)
    off = X - cen[None]
    r = np.linalg.norm(off, axis=-1)
    sep = 0.4 * min(np.linalg.norm(s.nuc[i] - s.nuc[j])
                    for i in range(3) for j in range(i + 1, 3))
    assert r.max() <= sep * (1 + 1e-12)
    # uniform in the ball: (r / sep)^3 ~ U(0, 1); isotropic directions
    u = np.sort((r / sep).ravel() ** 3)
    ks = np.max(np.abs(u - np.arange(1, u.size + 1) / u.size))
    assert ks < 1.63 / np.sqrt(u.size)          # Kolmogorov-Smirnov, alpha = 0.01
    d = off / r[..., None]
    assert np.all(np.abs(d.reshape(-1, 3).mean(0)) < 0.01)
    assert np.allclose(np.cov(d.reshape(-1, 3).T), np.eye(3) / 3, atol=0.01)


def test_initial_walkers_follow_reference_rule_atom():
    """Atoms: N(0, (0.5 sqrt(n_e))^2) about the nucleus
    (OmegaQMC/vmc_gto.py:111-115)."""
    s = _system(_mol([("Ne", (0.1, -0.2, 0.3))]))
    W = 20000
    X = init_walkers_ball(s, W, seed=9)
    off = X - s.nuc[0]
    sig = 0.5 * np.sqrt(s.n_e)
    assert abs(off.std() / sig - 1) < 0.01
    assert np.all(np.abs(off.reshape(-1, 3).mean(0)) < 0.02 * sig)
    # Gaussian tails, not a ball
    assert np.abs(off).max() > 3 * sig


def test_initial_walkers_are_seeded():
    atoms = [("Li", (0.0, 0.0, 0.0)), ("H", (0.0, 0.0, 3.015))]
    s = _system(_mol(atoms))
    assert np.array_equal(init_walkers_ball(s, 8, 3), init_walkers_ball(s, 8, 3))
    assert not np.array_equal(init_walkers_ball(s, 8, 3), init_walkers_ball(s, 8, 4))
