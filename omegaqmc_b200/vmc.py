"""``get_vmc_gto_func``: the reference's VMC driver surface on the B200 kernels.

Mirrors ``OmegaQMC.vmc_gto.get_vmc_gto_func`` (``OmegaQMC/vmc_gto.py:1620-1765``)
and the driver's ``__call__`` (``vmc_gto.py:1233-1617``): walker
initialisation (``vmc_gto.py:64-118``), basin thermalisation (``925-957,
1036-1053``), equilibration with step adaptation (``121-126, 1338-1357``),
production blocks with one local energy per step (``985-1034``), the
per-block log line (``1503-1551``), the final ``do_binning_analysis``
(``utils.py:86-150``) and the checkpoint with the reference's keys
(``1459-1478, 1606-1617``; HDF5 when h5py is importable, else ``.npz``).

The moves are single-electron sweeps (every electron proposed once per step,
Sherman-Morrison inverse updates, periodic FP64 refresh) instead of the
reference's all-electron move; ``proposal="scaled"`` selects the
nucleus-scaled Gaussian with its exact Metropolis-Hastings correction.
"""
from __future__ import annotations

import math
import os
import pathlib
import sys
import warnings
from datetime import datetime

import numpy as np
import torch

from .batch import BatchedSampler
from .context import GTOContext
from .cusp import cusp_params_for_mol
from . import replicas as RP
from .sampler import NSUM, WalkerEnsemble, init_walkers_ball
from .system import build_system

__all__ = ["get_vmc_gto_func", "VMCDriverGTO", "binning_analysis"]

TARGET_ACCEPTANCE_RATE = 0.4
STEP_SIZE_ADAPTATION_RATE = 0.05
BASIN_RELOC_SIGMA = 1.5
N_BASIN_THERMAL_STEPS = 800


def binning_analysis(a):
    """(mean, serr, sdev, kappa) with kappa = 1 + 2 sum ac_k up to the first
    negative autocorrelation (``OmegaQMC/utils.py:86-150``)."""
    a = np.asarray(a, dtype=np.float64)
    n = a.shape[0]
    xbar = a.mean()
    sdev = a.std()
    x = a - xbar
    nfft = 1 << int(math.ceil(math.log2(max(2 * n - 1, 1))))
    fx = np.fft.rfft(x, nfft)
    ac = np.fft.irfft(fx * np.conj(fx), nfft)[:n]
    if ac[0] == 0:
        return float(xbar), 0.0, float(sdev), 1.0
    ac = ac / ac[0]
    kappa = 1.0
    for k in range(1, n):
        if ac[k] < 0:
            break
        kappa += 2.0 * ac[k]
    return float(xbar), float(sdev * math.sqrt(kappa / n)), float(sdev), float(kappa)


def key_data_from_seed(seed):
    """The checkpoint's ``rng_key``: two uint32 words, the key data of
    ``jax.random.PRNGKey(seed)`` for the threefry generator (high word,
    low word), which the reference restores with ``jax.random.wrap_key_data``
    (``OmegaQMC/vmc_gto.py:1403-1410, 1606-1610``)."""
    seed = int(seed) & (2**64 - 1)
    return np.array([seed >> 32, seed & 0xFFFFFFFF], dtype=np.uint32)


def seed_from_key_data(key):
    """Inverse of :func:`key_data_from_seed`: the 64-bit seed of a
    checkpoint's ``rng_key`` (two uint32 words, as the reference writes
    them); a single integer is taken as the seed itself."""
    k = np.asarray(key).ravel()
    if k.size == 2:
        return (int(k[0]) & 0xFFFFFFFF) << 32 | (int(k[1]) & 0xFFFFFFFF)
    if k.size == 1:
        return int(k[0])
    raise ValueError(f"rng_key must hold one seed or two uint32 words, got {k.size} values")


def _validate_params_corr(params_corr):
    """Empty entries are dropped; J2 cusp coefficients are checked
    (``vmc_gto.py:542-626``)."""
    if params_corr is None:
        return {}
    out = {}
    for k, v in params_corr.items():
        if not isinstance(k, str):
            raise TypeError("params_corr keys must be strings")
        if isinstance(v, dict):
            if len(v) == 0:
                continue
            out[k] = v
        else:
            v = np.asarray(v)
            if k == "J2_pade" and v.shape[0] < 2:
                warnings.warn(f'Correlation parameter set "{k}" requires 2 elements, '
                              "but the user provided fewer.  Deleting...")
                continue
            out[k] = v
    eps = np.finfo(np.float64).eps
    j2 = out.get("J2_pade")
    if isinstance(j2, dict):
        if "like" in j2 and abs(float(np.ravel(j2["like"])[0]) - 0.25) > eps:
            warnings.warn(f"J2_pade['like'][0] = {float(np.ravel(j2['like'])[0]):.8f}, "
                          "expected 0.25 (same-spin cusp condition)")
        if "unlike" in j2 and abs(float(np.ravel(j2["unlike"])[0]) - 0.5) > eps:
            warnings.warn(f"J2_pade['unlike'][0] = {float(np.ravel(j2['unlike'])[0]):.8f}, "
                          "expected 0.5 (opposite-spin cusp condition)")
    return out


def get_vmc_gto_func(mf, params_corr, cusp_scheme="Quady2025", gr_scheme="scheme1",
                     force_estimator="simple", force_warp="swct", prefix="vmc",
                     symmop_list=None, cluster_idx=None, mo_relax=True, trial=None,
                     jastrow_config=None, *, params_cusp=None, precision="fp64",
                     proposal="plain", specialize=True, move="single", persistent=True):
    """Build a callable VMC driver (``vmc_gto.py:1620-1765``).

    Extra keywords (not in the reference): ``params_cusp`` supplies cusp
    constants instead of fitting them; ``precision`` is ``"fp64"`` or
    ``"mixed"``; ``proposal`` is ``"plain"`` (fixed-width Gaussian) or
    ``"scaled"`` (nucleus-scaled width); ``specialize`` compiles kernels for
    this molecule (NVRTC) when available; ``move`` is ``"single"``
    (single-electron sweeps) or ``"all"`` (the reference's all-electron
    step, one proposal moving every electron per sweep); ``persistent`` runs
    the production blocks as fused persistent launches (refresh, sweeps and
    local energies in one kernel, the same Markov chain) wherever the batched
    kernel accepts the configuration.  A multi-determinant ``trial`` samples in
    FP64 through the library's multi-determinant kernels."""
    if trial is not None and precision != "fp64":
        raise ValueError("multi-determinant trials are sampled in precision='fp64'")
    if symmop_list not in (None, "E", ["E"]):
        raise NotImplementedError("symmetry-adapted (correlated-sampling) operations are "
                                  "not supported on this path")
    for s in (".chk.h5", ".grd.h5", ".chk.npz"):
        if prefix.endswith(s):
            prefix = prefix[: -len(s)]
    params_corr = _validate_params_corr(params_corr)
    if cusp_scheme == "Quady2025":
        if params_cusp is None:
            params_cusp = cusp_params_for_mol(mf.mol)
    elif cusp_scheme is not None:
        raise ValueError(f"unknown cusp_scheme {cusp_scheme!r}")
    else:
        params_cusp = None
    timestamp_init = datetime.now()
    print("Begin time: {}".format(timestamp_init))
    return VMCDriverGTO(mf, params_corr, params_cusp, prefix, timestamp_init,
                        precision=precision, proposal=proposal, specialize=specialize,
                        jastrow_config=jastrow_config, trial=trial, move=move,
                        persistent=persistent)


class VMCDriverGTO:
    """Runs VMC sampling of one trial wavefunction (``vmc_gto.py:672-1617``)."""

    def __init__(self, mf, params_corr, params_cusp, prefix, timestamp_init,
                 precision="fp64", proposal="plain", specialize=True, jastrow_config=None,
                 trial=None, move="single", persistent=True):
        self.mf = mf
        self.params_corr = params_corr
        self.params_cusp = params_cusp
        self.system = build_system(mf, params_corr, params_cusp, jastrow_config, trial)
        self.ctx = GTOContext(self.system)
        if specialize and trial is None:
            try:
                self.ctx.specialize()
            except NotImplementedError as e:
                warnings.warn(f"kernel specialisation unavailable, using table-driven "
                              f"kernels: {e}")
        if proposal == "scaled":
            self.ctx.set_proposal(1, 1.0, 0.05)
        elif proposal != "plain":
            raise ValueError("proposal must be 'plain' or 'scaled'")
        # move="all": the reference's all-electron Gaussian step
        # (metropolis_move_alle, vmc_gto.py:815-838), one proposal per sweep
        if move == "all":
            if proposal != "plain":
                raise ValueError("all-electron steps use the plain Gaussian proposal")
            self.ctx.set_move_kind(1)
        elif move != "single":
            raise ValueError("move must be 'single' or 'all'")
        self.proposal = proposal
        self.move = move
        self.equilibration_seconds = None
        self.persistent = bool(persistent)
        self.precision = precision
        self.ofname_chkpt = prefix + ".chk"
        self.timestamp_init = timestamp_init
        self.enr_nn = self.system.e_nn
        self.results = None

    # ------------------------------------------------------------------
    def _device_equilibration(self, world):
        """Whether equilibration runs on the device (``oqmc_equilibrate``):
        one process, single-determinant trial, single-electron moves."""
        return world == 1 and self.system.md is None and self.move == "single"

    def _fused_sampler(self, ens, step, n_meas):
        """The fused persistent launch (FP64 refresh, sweeps and local energies
        in one kernel per <= 50 sweeps) for the production blocks.  Same
        proposals, acceptance and random numbers as the separate move and
        local-energy kernels (Philox counters (walker, sweep, electron)), so
        the chain is the same.  Its tile shape is autotuned on a copy of the
        walkers, whose positions are then restored, so tuning leaves the
        chain untouched.  None where the batched kernel refuses the
        configuration (radial splines, multi-determinant trials, all-electron
        steps) or NVRTC is absent; the production blocks then run on the
        separate kernels."""
        if not self.persistent:
            return None
        try:
            fused = BatchedSampler([self.ctx], [ens.X.clone()], [step], precision=self.precision,
                                   proposal=self.proposal, scale_r0=1.0, scale_fmin=0.05,
                                   cap=max(1, n_meas))
        except NotImplementedError:
            return None
        fused.tune(4, seed=(ens.seed ^ 0x7E57) & 0x7FFFFFFF)
        fused.walkers[0].copy_(ens.X)
        return fused

    def _fused_block(self, fused, ens, n_sw, every, n_meas):
        """One production block on the fused launch: launches of at most 50
        sweeps (the refresh cadence of the separate kernels), each a multiple
        of the measurement interval, continuing the ensemble's sweep counter
        and measurement slots.  Returns the block's (n_meas, 8) sums."""
        fused.reset(ens.step_count)
        done = 0
        while done < n_sw:
            chunk = min(n_sw - done, max(every, (ens.refresh_every // every) * every))
            fused.run(chunk, every, ens.seed)
            done += chunk
        ens.step_count += n_sw
        ens.X.copy_(fused.walkers[0])
        return fused.sums[0][:n_meas]

    def _save(self, path, data):
        try:
            import h5py
        except ImportError:
            np.savez(path + ".npz", **{k.replace("/", "_"): v for k, v in data.items()})
            return path + ".npz"
        p = pathlib.Path(path + ".h5")
        if p.exists():
            p.unlink()
        with h5py.File(str(p), "a") as f:
            for k, v in data.items():
                f.create_dataset(k, data=v)
        return str(p)

    def _load(self):
        p = self.ofname_chkpt
        if os.path.exists(p + ".h5"):
            import h5py
            with h5py.File(p + ".h5", "r") as f:
                return {k: f[k][()] for k in ("block_count", "mc_stepsize", "rng_key",
                                             "walkers", "E_blocks")}
        d = np.load(p + ".npz")
        return {k: d[k] for k in ("block_count", "mc_stepsize", "rng_key", "walkers",
                                  "E_blocks")}

    def __call__(self, rng_key, num_walkers=1000, num_steps_per_block=100, num_steps_decorr=1,
                 num_blocks=1000, num_blocks_equil=100, mc_timestep=0.1, fname_log=None,
                 mode_restart=False, num_steps_basin=N_BASIN_THERMAL_STEPS,
                 compute_gradients=False, gpu_memory_check="error"):
        """Execute a VMC run (``vmc_gto.py:1233-1617``); returns None and keeps the
        block energies in ``self.results``."""
        if gpu_memory_check not in ("error", "warn", "off"):
            raise ValueError("gpu_memory_check must be 'error', 'warn' "
                             f"or 'off', got {gpu_memory_check!r}")
        if compute_gradients:
            raise NotImplementedError("force estimators are not on this path")
        seed = rng_key if isinstance(rng_key, int) else seed_from_key_data(rng_key)
        s = self.system
        # replicas: with an initialised torch.distributed process group every
        # rank samples num_walkers walkers of its own and the block statistics
        # are summed over the ranks (the reference shards the walker axis,
        # OmegaQMC/utils.py:1148-1159)
        rank, world = RP.world_info()
        X = init_walkers_ball(s, num_walkers, RP.rank_seed(seed, rank))
        mc_stepsize = (3 * mc_timestep) ** 0.5
        E_b = []
        block_cnt_start = 1
        if mode_restart:
            d = self._load()
            block_cnt_start = int(d["block_count"]) + 1
            mc_stepsize = float(d["mc_stepsize"])
            seed = seed_from_key_data(d["rng_key"])
            X = np.asarray(d["walkers"])
            E_b = list(np.asarray(d["E_blocks"]))
            print("Restarting ...")
        ens = WalkerEnsemble(self.ctx, X, self.precision,
                             seed=RP.rank_seed(seed + 7919 * block_cnt_start, rank))
        if not mode_restart and num_steps_basin > 0:
            acc = ens.basin(num_steps_basin, BASIN_RELOC_SIGMA)
            print(f"ℹ️\tBasin thermalization: {num_steps_basin} "
                  f"relocation steps, acceptance {acc:.2f}")
        ratio = TARGET_ACCEPTANCE_RATE
        n_equil = num_blocks_equil * num_steps_per_block
        if not mode_restart and n_equil > 0:
            t_eq = datetime.now()
            if self._device_equilibration(world):
                # the whole scan on the device: sweep, adapt, sweep, ...
                mc_stepsize, accs, _ = ens.equilibrate(n_equil, mc_stepsize,
                                                       TARGET_ACCEPTANCE_RATE,
                                                       STEP_SIZE_ADAPTATION_RATE)
                ratio = float(accs[-1])
            else:
                # replicas adapt one width from the acceptance of all ranks;
                # other move kinds adapt on the host
                one = torch.zeros(1, NSUM, dtype=torch.float64, device=ens.X.device)
                for _ in range(n_equil):
                    one.zero_()
                    ens.run(1, mc_stepsize, sums=one)
                    RP.combine_sums(one)
                    ratio = float(one[0, 5]) / (ens.W * world * s.n_e)
                    mc_stepsize = float(np.exp(np.log(mc_stepsize) + STEP_SIZE_ADAPTATION_RATE
                                               * (ratio - TARGET_ACCEPTANCE_RATE)))
            self.equilibration_seconds = (datetime.now() - t_eq).total_seconds()
            print(f"ℹ️\tEquilibration acceptance rate: {ratio:.2f}")
            print(f"ℹ️\tEquilibration: {n_equil} steps in "
                  f"{self.equilibration_seconds:.2f} s")
        mc_timestep = mc_stepsize * mc_stepsize / 3
        print(f"ℹ️\tAdjusted step size: {mc_stepsize:.4f} bohr "
              f"~ {mc_timestep:.4f} Ha⁻¹ in Brownian time")
        if rank > 0:
            fout = open(os.devnull, "w")
        else:
            fout = sys.stdout if not fname_log else open(fname_log, "w", 1)
        print("# block_cnt        E_loc_mean      E_loc_std"
              "       eePotential     enPotential     Kinetic"
              "          weight_block        Δt_block"
              " acc_ratio", file=fout)
        t_prev = datetime.now()
        block_cnt = block_cnt_start - 1
        fused = self._fused_sampler(ens, mc_stepsize, num_steps_per_block)
        for block_cnt in range(block_cnt_start, block_cnt_start + num_blocks):
            n_sw = num_steps_per_block * num_steps_decorr
            if fused is not None:
                blk = self._fused_block(fused, ens, n_sw, num_steps_decorr, num_steps_per_block)
            else:
                blk = ens.run(n_sw, mc_stepsize, measure_every=num_steps_decorr)
            sums = RP.combine_sums(blk).cpu().numpy()
            nv = np.maximum(sums[:, 6], 1.0)
            ee_s, en_s, ke_s = sums[:, 0] / nv, sums[:, 1] / nv, sums[:, 2] / nv
            E_loc_s = ee_s + en_s + ke_s + self.enr_nn
            E_mean = float(E_loc_s.mean())
            std_E_s = float(E_loc_s.std())
            E_b.append(E_mean)
            t_cur = datetime.now()
            weight = float(sums[:, 6].sum())
            acc = float(sums[:, 5].sum()) / (n_sw * ens.W * world * s.n_e)
            print(f"{block_cnt:>8d}{E_mean:>24.8e}{std_E_s:>16.8e}"
                  f"{ee_s.mean():>16.8e}{en_s.mean():>16.8e}{ke_s.mean():>16.8e}"
                  f"{weight:>16.8e}{(t_cur - t_prev).total_seconds():>16.6f}"
                  f"{acc:>10.4f}", file=fout)
            t_prev = t_cur
        if fout is not sys.stdout:
            fout.close()
        if fused is not None:
            fused.close()
            ens.refresh()
        t_fin = datetime.now()
        print("End time: {}\t({:.6f} seconds total)".format(
            t_fin, (t_fin - self.timestamp_init).total_seconds()))
        e_mean, e_serr, _, e_kappa = binning_analysis(np.array(E_b))
        e_neff = len(E_b) / e_kappa
        print(f"ℹ️\tVMC energy: {e_mean:.8f} ± {e_serr:.8f} Ha"
              f" (N_eff = {e_neff:.1f})")
        mol = self.mf.mol
        asym = [mol.atom_symbol(i) for i in range(mol.natm)]
        torch.cuda.synchronize()
        data = {
            "version": "0.1.0",
            "timestamps/start": str(self.timestamp_init),
            "timestamps/end": str(t_fin),
            "system/atom_symbols": " ".join(asym),
            "system/atom_coords": mol.atom_coords(),
            "system/ao_basis": " ".join([str(mol.basis)] * mol.natm),
            "system/units": "BOHR",
            "E_blocks": np.array(E_b),
            "rng_key": key_data_from_seed(seed),
            "block_count": np.int32(block_cnt),
            "mc_stepsize": float(mc_stepsize),
            "walkers": ens.X.cpu().numpy(),
        }
        path = self._save(self.ofname_chkpt if world == 1 else
                          f"{self.ofname_chkpt}.rank{rank}", data)
        self.results = {"E_blocks": np.array(E_b), "energy": e_mean, "serr": e_serr,
                        "kappa": e_kappa, "mc_stepsize": mc_stepsize, "chk": path}
        return None
