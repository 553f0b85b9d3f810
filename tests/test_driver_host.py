"""Host logic of the VMC driver's fused production blocks (no GPU): launch
sizes follow the refresh cadence and the measurement interval, and the
ensemble's sweep counter and walkers continue across blocks."""
import pytest
import torch

from omegaqmc_b200.vmc import VMCDriverGTO


class _FakeFused:
    def __init__(self, W, n_e, n_meas):
        self.walkers = [torch.zeros(W, n_e, 3, dtype=torch.float64)]
        self.sums = [torch.zeros(n_meas, 8, dtype=torch.float64)]
        self.calls = []

    def reset(self, step_base):
        self.calls.append(("reset", step_base))

    def run(self, n, every, seed):
        self.calls.append(("run", n, every, seed))
        self.walkers[0] += n


class _FakeEnsemble:
    def __init__(self, W, n_e):
        self.X = torch.zeros(W, n_e, 3, dtype=torch.float64)
        self.step_count = 120
        self.refresh_every = 50
        self.seed = 77


@pytest.mark.parametrize("per_block,every", [(100, 1), (30, 1), (40, 3), (5, 60)])
def test_fused_block_launches(per_block, every):
    ens = _FakeEnsemble(4, 2)
    fused = _FakeFused(4, 2, per_block)
    n_sw = per_block * every
    out = VMCDriverGTO._fused_block(None, fused, ens, n_sw, every, per_block)
    assert fused.calls[0] == ("reset", 120)
    runs = [c for c in fused.calls if c[0] == "run"]
    assert sum(r[1] for r in runs) == n_sw
    for _, n, e, seed in runs:
        assert e == every and n % every == 0 and seed == 77
        assert n <= max(every, 50)
    assert ens.step_count == 120 + n_sw
    assert torch.all(ens.X == n_sw)          # walkers copied back from the launch
    assert out.shape == (per_block, 8)
