"""The VMC driver with two replica ranks (gloo process group, both ranks on
cuda:0; their kernels never wait on each other): every block's log line is
the walker-weighted mean over the union of both ranks' walkers, the ranks
sample different walkers, and each rank writes its own checkpoint
(the reference shards its walker axis and reduces block means,
OmegaQMC/utils.py:1148-1159, vmc_gto.py:1331-1333)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, tmp, out):
    import datetime
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        torch.cuda.set_device(0)
        from omegaqmc_b200 import generate_molecular_orbitals, get_vmc_gto_func
        from omegaqmc_b200 import replicas as RP
        from omegaqmc_b200 import vmc as V
        local, combined = [], []
        orig = RP.combine_sums

        def spy(s):
            if hasattr(s, "shape") and len(s.shape) == 2 and s.shape[0] == 20:
                local.append(np.array(s.cpu() if hasattr(s, "cpu") else s))
                r = orig(s)
                combined.append(np.array(r.cpu() if hasattr(r, "cpu") else r))
                return r
            return orig(s)

        V.RP.combine_sums = spy
        mf = generate_molecular_orbitals("H 0 0 -0.7; H 0 0 0.7", basis="sto-3g")
        J2 = {"J2_pade": {"like": np.array([0.25, 1.0]), "unlike": np.array([0.5, 1.0])}}
        drv = get_vmc_gto_func(mf, J2, cusp_scheme=None, prefix=os.path.join(tmp, "h2"))
        drv(321, num_walkers=512, num_steps_per_block=20, num_blocks=2, num_blocks_equil=1,
            num_steps_basin=10, fname_log=os.path.join(tmp, "h2.log"))
        out[rank] = {"local": local, "combined": combined, "chk": drv.results["chk"],
                     "e_nn": drv.enr_nn}
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(600)
def test_two_replica_driver(tmp_path):
    ctx = mp.get_context("spawn")
    man = ctx.Manager()
    out = man.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, str(tmp_path), out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(500)
    for p in procs:
        if p.is_alive():
            p.kill()
        assert p.exitcode == 0
    r0, r1 = out[0], out[1]
    assert len(r0["local"]) == len(r1["local"]) == 2          # one combine per block
    rows = [l.split() for l in open(tmp_path / "h2.log").read().splitlines()[1:]]
    assert len(rows) == 2
    for b in range(2):
        s0, s1 = r0["local"][b], r1["local"][b]
        assert not np.array_equal(s0, s1)                      # different walkers
        np.testing.assert_allclose(r0["combined"][b], s0 + s1, rtol=1e-15)
        np.testing.assert_allclose(r1["combined"][b], s0 + s1, rtol=1e-15)
        tot = s0 + s1
        e_series = (tot[:, 0] + tot[:, 1] + tot[:, 2]) / tot[:, 6] + r0["e_nn"]
        assert float(rows[b][1]) == pytest.approx(e_series.mean(), rel=1e-7)
        assert float(rows[b][6]) == pytest.approx(tot[:, 6].sum(), rel=1e-7)   # weight
        assert tot[0, 6] == 2 * 512
    # each rank's own checkpoint, with its own walkers
    assert r0["chk"] != r1["chk"]
    w0 = np.load(r0["chk"])["walkers"]
    w1 = np.load(r1["chk"])["walkers"]
    assert w0.shape == w1.shape == (512, 2, 3) and not np.array_equal(w0, w1)
