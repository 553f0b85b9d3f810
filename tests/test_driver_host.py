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


def test_rng_key_is_threefry_key_data():
    """rng_key in the checkpoint is what jax.random.key_data(PRNGKey(seed))
    holds for the threefry generator, two uint32 words (high, low), which
    the reference's restart wraps back into a key
    (OmegaQMC/vmc_gto.py:1403-1410, 1606-1610)."""
    import numpy as np
    from omegaqmc_b200.vmc import key_data_from_seed, seed_from_key_data
    for seed in (0, 1, 888, 2**32 - 1, 2**32 + 5, 2**64 - 1):
        k = key_data_from_seed(seed)
        assert k.dtype == np.uint32 and k.shape == (2,)
        assert seed_from_key_data(k) == seed
    assert list(key_data_from_seed(42)) == [0, 42]          # PRNGKey(42) key data
    assert seed_from_key_data(np.array([7], dtype=np.int64)) == 7
    with pytest.raises(ValueError):
        seed_from_key_data(np.zeros(3, dtype=np.uint32))


def _ckpt(W=3, n_e=2):
    import numpy as np
    from omegaqmc_b200.vmc import key_data_from_seed
    return {"version": "0.1.0", "timestamps/start": "t0", "timestamps/end": "t1",
            "system/atom_symbols": "H H", "system/atom_coords": np.zeros((2, 3)),
            "system/ao_basis": "sto-3g sto-3g", "system/units": "BOHR",
            "E_blocks": np.array([-1.1, -1.2]), "rng_key": key_data_from_seed(2**33 + 9),
            "block_count": np.int32(2), "mc_stepsize": 0.45,
            "walkers": np.arange(W * n_e * 3, dtype=np.float64).reshape(W, n_e, 3)}


@pytest.mark.parametrize("use_h5", [False, True])
def test_checkpoint_round_trip(tmp_path, use_h5, monkeypatch):
    """The checkpoint keeps the reference's dataset names and types; HDF5
    where h5py imports (the reference's format), else .npz with the same
    keys."""
    import sys
    import types
    import numpy as np
    from omegaqmc_b200.vmc import seed_from_key_data
    if use_h5:
        pytest.importorskip("h5py")
    else:
        monkeypatch.setitem(sys.modules, "h5py", None)
    base = str(tmp_path / "run.chk")
    data = _ckpt()
    path = VMCDriverGTO._save(None, base, data)
    assert path.endswith(".h5" if use_h5 else ".npz")
    d = VMCDriverGTO._load(types.SimpleNamespace(ofname_chkpt=base))
    assert int(d["block_count"]) == 2 and float(d["mc_stepsize"]) == 0.45
    assert seed_from_key_data(d["rng_key"]) == 2**33 + 9
    assert np.array_equal(d["walkers"], data["walkers"])
    assert np.array_equal(d["E_blocks"], data["E_blocks"])
