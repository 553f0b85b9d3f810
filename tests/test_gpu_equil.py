"""Equilibration with the step width adapted on the device
(``oqmc_equilibrate``): the reference's rule log s <- log s + 0.05 (acc -
0.4) after every sweep (OmegaQMC/vmc_gto.py:121-126, 1338-1357) gives the
same width sequence, acceptances and walkers as the host loop that reads
each sweep's acceptance back (the driver's former equilibration), for a
fixed seed; the driver reports its equilibration time."""
import numpy as np
import pytest
import torch

from helpers import golden_system, seeded_walkers
from omegaqmc_b200 import generate_molecular_orbitals, get_vmc_gto_func
from omegaqmc_b200.context import GTOContext
from omegaqmc_b200.sampler import NSUM, WalkerEnsemble

pytestmark = pytest.mark.gpu


def _host_loop(ens, n, step, target=0.4, rate=0.05):
    one = torch.zeros(1, NSUM, dtype=torch.float64, device="cuda")
    steps, accs = [], []
    for _ in range(n):
        one.zero_()
        ens.run(1, step, sums=one)
        acc = float(one[0, 5]) / (ens.W * ens.ctx.n_e)
        step = float(np.exp(np.log(step) + rate * (acc - target)))
        steps.append(step)
        accs.append(acc)
    return step, np.array(accs), np.array(steps)


@pytest.mark.parametrize("name,prec,proposal,spec", [("bench_h2o", "fp64", 0, True),
                                                     ("bench_h2o", "mixed", 1, True),
                                                     ("bench_lih", "fp64", 1, True),
                                                     ("bench_lih", "mixed", 0, False)])
def test_device_adaptation_follows_host_loop(name, prec, proposal, spec):
    s, _ = golden_system(name)
    ctx = GTOContext(s)
    if spec:
        ctx.specialize()            # else the table-driven move kernel
    if proposal:
        ctx.set_proposal(1, 1.0, 0.05)
    X0 = seeded_walkers(s, 2048, 1.0, 3)
    n, step0 = 130, 0.9            # crosses two refreshes (every 50 sweeps)
    eh = WalkerEnsemble(ctx, X0, prec, seed=41)
    sh, acc_h, steps_h = _host_loop(eh, n, step0)
    ed = WalkerEnsemble(ctx, X0, prec, seed=41)
    sd, acc_d, steps_d = ed.equilibrate(n, step0)
    torch.cuda.synchronize()
    acc_d, steps_d = acc_d.cpu().numpy(), steps_d.cpu().numpy()
    np.testing.assert_allclose(steps_d, steps_h, rtol=1e-12, atol=0)
    np.testing.assert_allclose(acc_d, acc_h, rtol=0, atol=1e-12)
    assert sd == pytest.approx(sh, rel=1e-12)
    # the widths agree to rounding (device exp/log against numpy), so the
    # positions agree to rounding unless a decision flipped
    close = (ed.X - eh.X).abs().reshape(ed.W, -1).amax(dim=1) < 1e-10
    assert close.float().mean().item() > 0.999, close.float().mean().item()
    assert ed.step_count == eh.step_count and ed.since_refresh == eh.since_refresh
    # the width moved towards the 0.4 target
    assert abs(acc_d[-20:].mean() - 0.4) < abs(acc_d[0] - 0.4) + 0.05
    assert ctx.flags() == 0


def test_device_equilibration_refuses_all_electron_steps():
    s, _ = golden_system("bench_h2")
    ctx = GTOContext(s)
    ctx.set_move_kind(1)
    ens = WalkerEnsemble(ctx, seeded_walkers(s, 64, 0.5, 0), "fp64", seed=1)
    with pytest.raises(NotImplementedError):
        ens.equilibrate(3, 0.5)


def test_driver_equilibrates_on_device(tmp_path, capsys):
    mf = generate_molecular_orbitals("H 0 0 -0.7; H 0 0 0.7", basis="sto-3g")
    J2 = {"J2_pade": {"like": np.array([0.25, 1.0]), "unlike": np.array([0.5, 1.0])}}
    drv = get_vmc_gto_func(mf, J2, cusp_scheme=None, prefix=str(tmp_path / "h2"))
    drv(3, num_walkers=1024, num_steps_per_block=50, num_blocks=2, num_blocks_equil=20,
        num_steps_basin=10, fname_log=str(tmp_path / "h2.log"))
    out = capsys.readouterr().out
    assert "Equilibration: 1000 steps in" in out
    assert drv.equilibration_seconds is not None and drv.equilibration_seconds < 30
    rate = float(out.split("Equilibration acceptance rate:")[1].split()[0])
    assert 0.3 < rate < 0.5
