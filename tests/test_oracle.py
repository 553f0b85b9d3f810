"""The CPU oracle against the reference's own outputs and relations.

* golden vectors produced by running the reference's ``gto.py`` /
  ``shell.py`` / ``utils.py`` (``tests/golden/make_golden.py``);
* the relations the reference's tests check: the ``np.dot`` cusp form
  (tests/test_multi_gpu_sharding.py:47-68), the closed-form Padé J1
  (tests/test_gto_jastrow.py:495-505), analytic versus autodiff-Hessian
  kinetic energy (tests/test_gto_kinetic_energy.py:182-200), hand-written
  versus autodiff angular gradients (tests/test_gto_kinetic_energy.py:611-644)
  and finite-difference gradients (tests/test_gto_kinetic_energy.py:79-108).
"""
import warnings

import numpy as np
import pytest
import torch

from helpers import golden_cases, golden_system, load_golden, seeded_walkers, GOLDEN
from oracle import gto_oracle as O
from omegaqmc_b200 import molecules as M
from omegaqmc_b200.system import build_system, read_shell, MeanField

CASES = golden_cases()


def _rel(a, b, floor=1.0):
    return np.max(np.abs(np.asarray(a) - np.asarray(b)) / (np.abs(b) + floor))


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference_outputs(name):
    s, d = golden_system(name)
    r = O.evaluate(s, d["X"])
    # spline radials: power-form quintics with large coefficients near the
    # nucleus amplify last-bit differences of the evaluation order
    tol2 = 5e-11 if s.spl is not None else 1e-11
    assert _rel(r["logpsi"], d["logpsi"]) < 1e-12
    assert _rel(r["e_ee"], d["e_ee"]) < 1e-13
    assert _rel(r["e_en"], d["e_en"]) < 1e-13
    assert _rel(r["e_ke"], d["e_ke"]) < tol2
    assert _rel(r["grad"], d["grad"]) < 1e-12
    assert _rel(r["lap"], d["lap"]) < tol2
    assert abs(s.e_nn - float(d["e_nn"])) < 1e-13


@pytest.mark.parametrize("name", CASES)
def test_reference_analytic_ke_matches_hessian(name):
    # the reference's own regression relation, on its own outputs
    _, _, _, d = load_golden(name)
    kh = d["e_ke_hessian"]
    assert np.max(np.abs(kh - d["e_ke"][:len(kh)]) / (np.abs(kh) + 1)) < 1e-9


def test_cusp_value_matches_reference_and_dot_form():
    g = np.load(f"{GOLDEN}/golden_cusp.npz")
    coeff = g["coeff"]
    for r, ref in zip(g["r"], g["val"]):
        ours = O.cusp_s(np.float64(r), 0.25, 8.0, 0.7, 1.3, coeff)
        s = r / 0.25
        b = (1 - 10 * s ** 3 + 15 * s ** 4 - 6 * s ** 5) if r < 0.25 else 0.0
        sl = 1.3 * np.exp(-8.0 * r)
        terms = np.concatenate([[(1 - b) * 0.7, b * sl], b * sl * s ** np.arange(2, 8)])
        np.testing.assert_allclose(ours, np.dot(coeff, terms), rtol=1e-13, atol=1e-15)
        np.testing.assert_allclose(ours, ref, rtol=1e-13, atol=1e-15)


def test_cusp_vgl_matches_reference():
    g = np.load(f"{GOLDEN}/golden_cusp.npz")
    for r, ref in zip(g["r_vgl"], g["vgl"]):
        f, fp, fl = O.cusp_s_vgl(np.float64(r), 0.2, 8.0, 0.7, -1.1, 3.3, 1.3, g["coeff"])
        np.testing.assert_allclose([f, fp, fl], ref, rtol=1e-12, atol=1e-12)


def test_closed_form_j1_without_cusp():
    mf, _, _, d = load_golden("h2o_nocusp")
    s = build_system(mf, {"J1_pade": {"O": np.array(0.9), "H": np.array(0.4)}})
    X = d["X"][:4]
    b = np.where(np.array(mf.mol.elements) == "O", 0.9, 0.4)
    r = np.linalg.norm(X[:, None, :, :] - s.nuc[None, :, None, :], axis=-1)
    ref = np.sum(-s.Z[None, :, None] * r / (1.0 + b[None, :, None] * r), axis=(1, 2))
    np.testing.assert_allclose(O.jastrow_value(s, X), ref, rtol=0, atol=1e-12)


def test_binning_analysis_matches_reference():
    g = np.load(f"{GOLDEN}/golden_binning.npz")
    ours = O.binning_analysis(g["series"])
    np.testing.assert_allclose(ours, g["result"], rtol=1e-12)


@pytest.mark.parametrize("am", [0, 1, 2, 3, 4])
def test_harmonic_gradients_vs_autograd(am):
    rng = np.random.default_rng(am * 17 + 3)
    for _ in range(8):
        dr = rng.normal(size=3)
        Y, G = O.harmonics(am, dr)
        t = torch.tensor(dr, requires_grad=True)

        def f(v):
            x, y, z = v[0], v[1], v[2]
            out = []
            for terms in O.HARMONICS[am]:
                acc = 0.0
                for c, i, j, k in terms:
                    acc = acc + c * x ** i * y ** j * z ** k
                out.append(acc * torch.ones((), dtype=torch.float64))
            return torch.stack(out)
        J = torch.autograd.functional.jacobian(f, t).numpy()
        np.testing.assert_allclose(G, J, atol=1e-13)
        np.testing.assert_allclose(Y, f(t).detach().numpy(), atol=1e-14)


def test_harmonics_are_harmonic():
    # solid harmonics have zero Laplacian, which the VGL assembly relies on
    rng = np.random.default_rng(7)
    for am in (2, 3, 4):
        dr = rng.normal(size=3)
        h = 1e-3
        lap = 0.0
        for k in range(3):
            e = np.zeros(3)
            e[k] = h
            lap = lap + (O.harmonics(am, dr + e)[0] - 2 * O.harmonics(am, dr)[0]
                         + O.harmonics(am, dr - e)[0]) / h ** 2
        assert np.max(np.abs(lap)) < 1e-5


@pytest.mark.parametrize("name", ["h2o_cusp", "fg_shells"])
def test_gradient_and_laplacian_vs_finite_differences(name):
    s, d = golden_system(name)
    X = d["X"][:2].copy()
    r = O.evaluate(s, X)
    h = 1e-5
    for w in range(2):
        for e in (0, 3):
            for k in range(3):
                Xp = X[w:w + 1].copy()
                Xm = X[w:w + 1].copy()
                Xp[0, e, k] += h
                Xm[0, e, k] -= h
                fd = (O.log_psi(s, Xp)[0] - O.log_psi(s, Xm)[0]) / (2 * h)
                assert abs(fd - r["grad"][w, e, k]) < 1e-6 * (1 + abs(fd))


def test_analytic_ke_vs_torch_hessian():
    """Analytic KE of the oracle against a float64 autograd Hessian of a
    torch restatement of log|psi| (the reference's _local_energy_ke_hessian
    relation, gto.py:2487-2504), on H2/STO-3G with Jastrow."""
    s, d = golden_system("h2_sto3g")
    X = d["X"][:3]
    r = O.evaluate(s, X)
    for w in range(3):
        x = torch.tensor(X[w].reshape(-1), requires_grad=True)

        def logpsi(v):
            v = v.reshape(2, 3)
            out = 0.0
            vals = []
            for e in range(2):
                ao = []
                for sh in s.shells:
                    dr = v[e] - torch.tensor(s.nuc[sh.iat])
                    r2 = (dr * dr).sum()
                    ao.append((torch.tensor(sh.norm) * torch.exp(-torch.tensor(sh.alpha) * r2)).sum())
                vals.append(torch.stack(ao) @ torch.tensor(s.C))
            out = torch.log(torch.abs(vals[0][0])) + torch.log(torch.abs(vals[1][0]))
            rij = torch.sqrt(((v[0] - v[1]) ** 2).sum())
            a, b = s.j2[1]
            return out + a * rij / (1 + b * rij)
        H = torch.autograd.functional.hessian(logpsi, x)
        g = torch.autograd.grad(logpsi(x), x)[0]
        ke = -0.5 * (torch.trace(H) + (g * g).sum())
        assert abs(float(ke) - r["e_ke"][w]) < 1e-9 * (1 + abs(float(ke)))


def test_read_shell_normalisation():
    # s and p shells are unit-normalised over the contraction
    entry = [0, [13.0, 0.02], [2.0, 0.14], [0.45, 0.48]]
    sh = read_shell(entry, 0, 0)[0]
    a = sh.alpha
    S = np.sum(sh.norm[:, None] * sh.norm[None, :] * (np.pi / (a[:, None] + a[None, :])) ** 1.5)
    assert abs(S - 1.0) < 1e-13
    entry = [1, [3.0, 0.3], [0.7, 0.7]]
    sh = read_shell(entry, 0, 0)[0]
    a = sh.alpha
    asum = a[:, None] + a[None, :]
    S = np.sum(sh.norm[:, None] * sh.norm[None, :] * 0.5 * np.pi ** 1.5 / asum ** 2.5)
    assert abs(S - 1.0) < 1e-13


def test_named_systems_shapes():
    expect = {"H2": (2, 1, 2), "LiH": (4, 2, 19), "H2O": (10, 5, 24),
              "N2": (14, 7, 28), "H2O_dimer": (20, 10, 48)}
    for name, (ne, nocc, nbf) in expect.items():
        mf = M.make_mf(name)
        s = build_system(mf, M.default_params_corr(mf.mol))
        assert (s.n_e, s.nocc, s.nbf) == (ne, nocc, nbf), name


def test_oracle_sampler_energy_h2_is_finite():
    mf = M.make_mf("H2")
    s = build_system(mf, M.default_params_corr(mf.mol))
    X = seeded_walkers(s, 64, 0.5, 0)
    e = O.local_energy(s, X)
    assert np.all(np.isfinite(e))
