"""The reference-facing driver and get_psi_fun on the GPU."""
import os

import numpy as np
import pytest
import torch

from helpers import golden_system, load_golden, seeded_walkers
from omegaqmc_b200 import generate_molecular_orbitals, get_psi_fun, get_vmc_gto_func
from omegaqmc_b200 import molecules as M

pytestmark = pytest.mark.gpu


def test_driver_runs_logs_and_restarts(tmp_path, capsys):
    mf = generate_molecular_orbitals("H 0 0 -0.7; H 0 0 0.7", basis="sto-3g")
    prefix = str(tmp_path / "h2")
    drv = get_vmc_gto_func(mf, {"J2_pade": {"like": np.array([0.25, 1.0]),
                                            "unlike": np.array([0.5, 1.0])}},
                           cusp_scheme=None, prefix=prefix)
    log = str(tmp_path / "h2.log")
    drv(888, num_walkers=512, num_steps_per_block=20, num_blocks=6, num_blocks_equil=2,
        num_steps_basin=20, fname_log=log)
    lines = open(log).read().splitlines()
    assert lines[0].startswith("# block_cnt")
    assert len(lines) == 7
    E = np.array([float(l.split()[1]) for l in lines[1:]])
    assert np.all(np.isfinite(E)) and np.all(E < -0.9) and np.all(E > -1.3)
    out = capsys.readouterr().out
    assert "VMC energy:" in out and "Basin thermalization" in out
    assert os.path.exists(drv.results["chk"])
    drv(888, num_walkers=512, num_steps_per_block=20, num_blocks=3, mode_restart=True,
        fname_log=log)
    assert len(drv.results["E_blocks"]) == 9
    with pytest.raises(ValueError):
        drv(1, num_walkers=8, gpu_memory_check="maybe")
    with pytest.raises(NotImplementedError):
        drv(1, num_walkers=8, compute_gradients=True)


def test_driver_all_electron_moves(tmp_path, capsys):
    """move="all": the reference's all-electron step through the driver."""
    mf = generate_molecular_orbitals("H 0 0 -0.7; H 0 0 0.7", basis="sto-3g")
    J2 = {"J2_pade": {"like": np.array([0.25, 1.0]), "unlike": np.array([0.5, 1.0])}}
    with pytest.raises(ValueError):
        get_vmc_gto_func(mf, J2, cusp_scheme=None, prefix=str(tmp_path / "x"), move="some")
    with pytest.raises(ValueError):
        get_vmc_gto_func(mf, J2, cusp_scheme=None, prefix=str(tmp_path / "x"), move="all",
                         proposal="scaled")
    drv = get_vmc_gto_func(mf, J2, cusp_scheme=None, prefix=str(tmp_path / "h2a"), move="all")
    log = str(tmp_path / "h2a.log")
    drv(5, num_walkers=512, num_steps_per_block=20, num_blocks=4, num_blocks_equil=2,
        num_steps_basin=20, fname_log=log)
    rows = [l.split() for l in open(log).read().splitlines()[1:]]
    assert len(rows) == 4
    E = np.array([float(r[1]) for r in rows])
    acc = np.array([float(r[-1]) for r in rows])
    assert np.all(E < -0.9) and np.all(E > -1.3)
    # step adaptation drives the all-electron acceptance towards 0.4
    assert np.all((acc > 0.2) & (acc < 0.7)), acc


def test_driver_fused_blocks_follow_the_split_chain(tmp_path):
    """Production blocks on the fused persistent launch continue the same
    Markov chain as the separate move and local-energy kernels."""
    mf = generate_molecular_orbitals("H 0 0 -0.7; H 0 0 0.7", basis="sto-3g")
    J2 = {"J2_pade": {"like": np.array([0.25, 1.0]), "unlike": np.array([0.5, 1.0])}}
    out = {}
    for fused in (True, False):
        drv = get_vmc_gto_func(mf, J2, cusp_scheme=None, prefix=str(tmp_path / f"h2{fused}"),
                               persistent=fused)
        drv(31, num_walkers=512, num_steps_per_block=30, num_blocks=3, num_blocks_equil=1,
            num_steps_basin=10, fname_log=str(tmp_path / f"h2{fused}.log"))
        d = np.load(drv.results["chk"])
        out[fused] = (d["walkers"], drv.results["E_blocks"])
    same = np.all(out[True][0] == out[False][0], axis=(1, 2)).mean()
    assert same > 0.95, same
    np.testing.assert_allclose(out[True][1], out[False][1], atol=5e-3)


def test_get_psi_fun_matches_golden_per_walker():
    mf, params, cusp, d = load_golden("h2o_cusp")
    log_psi, (e_ee, e_nn, e_en, e_ke), (get_mo, _), _ = get_psi_fun(mf, params_cusp=cusp)
    nuc = mf.mol.atom_coords()
    for w in range(3):
        x = d["X"][w]
        assert abs(log_psi(x, nuc, params) - d["logpsi"][w]) < 1e-10 * (1 + abs(d["logpsi"][w]))
        assert abs(e_ke(x, nuc, params) - d["e_ke"][w]) < 1e-9 * (1 + abs(d["e_ke"][w]))
        assert abs(e_ee(x) - d["e_ee"][w]) < 1e-12 * (1 + abs(d["e_ee"][w]))
        assert abs(e_en(x, nuc) - d["e_en"][w]) < 1e-12 * (1 + abs(d["e_en"][w]))
    assert abs(e_nn(nuc) - float(d["e_nn"])) < 1e-12
    # batched torch input gives CUDA tensors
    X = torch.tensor(d["X"], device="cuda")
    lp = log_psi(X, nuc, params)
    assert lp.is_cuda and lp.shape == (d["X"].shape[0],)
    mo, _ = get_mo(d["X"][0], nuc)
    assert mo.shape == (10, 5)


def test_get_psi_fun_error_conventions():
    mf = M.make_mf("H2O")
    log_psi, *_ = get_psi_fun(mf)
    x = seeded_walkers(__import__("omegaqmc_b200").build_system(mf, {}), 1, 0.8, 0)[0]
    with pytest.raises(ValueError, match="expected b or"):
        log_psi(x, mf.mol.atom_coords(), {"J1_pade": {"O": np.array([0.1, 0.2, 0.3]),
                                                     "H": np.array(0.4)}})
    with pytest.warns(UserWarning, match="a is fixed at -Z"):
        log_psi(x, mf.mol.atom_coords(), {"J1_pade": {"O": np.array([-0.05, 0.9]),
                                                     "H": np.array(0.4)}})
    # without jastrow_config every element gets the 10-bohr one-body spline,
    # and an element missing from J1_bspline raises KeyError as in the
    # reference's J1_bspline_fn (gto.py:1752-1756)
    with pytest.raises(KeyError):
        log_psi(x, mf.mol.atom_coords(), {"J1_bspline": {"O": np.zeros(4)}})
