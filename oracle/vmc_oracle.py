"""CPU oracle of the reference's VMC sampler (TEST INFRASTRUCTURE).

Restates the reference's sampling algorithm on top of ``gto_oracle``:
all-electron Gaussian proposals with the MIN_DIST_THRESHOLD rejection
(``OmegaQMC/vmc_gto.py:815-839``), Metropolis acceptance
``u < exp(2 (ln psi_new - ln psi_old))`` (``vmc_gto.py:893-902``), step
adaptation ``log s += 0.05 (acc - 0.4)`` during equilibration
(``vmc_gto.py:121-126, 1338-1357``) and one local energy per production
step (``vmc_gto.py:985-1034``).  numpy's PCG64 stands in for JAX's
threefry stream, so agreement with the GPU sampler is statistical.
"""
from __future__ import annotations

import numpy as np

from . import gto_oracle as O

TARGET_ACCEPTANCE_RATE = 0.4
STEP_SIZE_ADAPTATION_RATE = 0.05


def _invalid(system, X):
    n_e = X.shape[1]
    i, j = np.triu_indices(n_e, k=1)
    dee = np.linalg.norm(X[:, i] - X[:, j], axis=-1)
    den = np.linalg.norm(X[:, :, None, :] - system.nuc[None, None], axis=-1)
    m = np.min(den.reshape(X.shape[0], -1), axis=1)
    if dee.shape[1]:
        m = np.minimum(m, np.min(dee, axis=1))
    return m < O.MIN_DIST_THRESHOLD


def metropolis_all_electron(system, X, step, rng, logpsi=None):
    """One all-electron move of every walker; returns (X, logpsi, accepted)."""
    if logpsi is None:
        logpsi = O.log_psi(system, X)
    prop = X + step * rng.standard_normal(X.shape)
    ratio = np.where(_invalid(system, prop), 0.0, 1.0)
    lp_new = O.log_psi(system, prop)
    acc = rng.random(X.shape[0]) < np.exp(2.0 * (lp_new - logpsi)) * ratio
    X = np.where(acc[:, None, None], prop, X)
    logpsi = np.where(acc, lp_new, logpsi)
    return X, logpsi, acc


def run_vmc(system, X, n_equil, n_prod, mc_timestep=0.1, seed=0):
    """Equilibrate with step adaptation, then produce one E_L per step.

    Returns (E_L walker-mean series (n_prod,), acceptance, final step)."""
    rng = np.random.default_rng(seed)
    step = (3.0 * mc_timestep) ** 0.5
    lp = O.log_psi(system, X)
    for _ in range(n_equil):
        X, lp, acc = metropolis_all_electron(system, X, step, rng, lp)
        step = float(np.exp(np.log(step) + STEP_SIZE_ADAPTATION_RATE
                            * (acc.mean() - TARGET_ACCEPTANCE_RATE)))
    series = np.zeros(n_prod)
    accs = 0.0
    for t in range(n_prod):
        X, lp, acc = metropolis_all_electron(system, X, step, rng, lp)
        accs += acc.mean()
        series[t] = O.local_energy(system, X).mean()
    return series, accs / n_prod, step, X
