"""Batched persistent launch over uneven molecules (oqmc_batch_*).

The batch kernel draws the same Philox numbers as the per-system kernels, so
per molecule a batched launch must leave the walkers of the per-system path
(FP64 refresh, then sweeps) and the same measurement sums up to summation
order."""
import numpy as np
import pytest
import torch

from helpers import seeded_walkers
from omegaqmc_b200 import molecules as M
from omegaqmc_b200.batch import BatchedSampler
from omegaqmc_b200.context import GTOContext
from omegaqmc_b200.sampler import NSUM, PREC
from omegaqmc_b200.system import build_system

pytestmark = pytest.mark.gpu

NAMES = ["H2", "LiH", "H2O"]
WALKERS = [300, 200, 500]          # not multiples of the tile sizes: ragged tails
STEPS = [0.5, 0.6, 0.8]
PROPS = ["plain", "scaled", "scaled"]


def _system(name):
    mf = M.make_mf(name)
    return build_system(mf, M.benchmark_params_corr(mf.mol))


@pytest.fixture(scope="module")
def contexts():
    ctxs = []
    for n in NAMES:
        c = GTOContext(_system(n))
        c.specialize()
        ctxs.append(c)
    return ctxs


def _walkers(ctxs, seed=1):
    return [torch.as_tensor(seeded_walkers(c.system, W, 1.0, seed + k), device="cuda")
            for k, (c, W) in enumerate(zip(ctxs, WALKERS))]


def _per_system(ctx, X0, precision, prop, step, n_sweeps, me, seed, step_base):
    ctx.set_proposal(1 if prop == "scaled" else 0, 1.0, 0.05)
    X = X0.clone()
    st = ctx.new_state(X.shape[0], PREC[precision])
    sums = torch.zeros(n_sweeps // me, NSUM, dtype=torch.float64, device="cuda")
    ctx.refresh(X, st, PREC[precision])
    ctx.sweeps(X, st, PREC[precision], n_sweeps, step, seed, step_base, sums, measure_every=me)
    torch.cuda.synchronize()
    ctx.set_proposal(0)
    return X, sums


# (threads per CTA, walkers per tile): lanes per walker threads / walkers,
# (1, 2, 4) and (8, 4, 1) for H2, LiH, H2O
SHAPES = [(128, [128, 64, 32]), (256, [32, 64, 256])]


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_batch_reproduces_per_system_path(contexts, precision, shape):
    X0 = _walkers(contexts)
    b = BatchedSampler(contexts, [x.clone() for x in X0], STEPS, precision=precision,
                       proposal=PROPS, cap=16)
    b.configure(shape[0], shape[1], variant=0)
    n, me, seed, base = 20, 5, 1234, 100
    b.reset(base)
    b.run(n, me, seed)
    torch.cuda.synchronize()
    assert b.flags() == 0
    for k, ctx in enumerate(contexts):
        X, sums = _per_system(ctx, X0[k], precision, PROPS[k], STEPS[k], n, me, seed, base)
        same = torch.all((b.walkers[k] == X).reshape(X.shape[0], -1), dim=1)
        frac = float(same.float().mean())
        assert frac > 0.99, (NAMES[k], frac)
        moved = torch.any((X != X0[k]).reshape(X.shape[0], -1), dim=1)
        assert float(moved.float().mean()) > 0.5
        bs = b.sums[k][: n // me].cpu().numpy()
        rs = sums.cpu().numpy()
        np.testing.assert_array_equal(bs[:, 6], rs[:, 6])          # finite walkers
        if frac == 1.0:
            np.testing.assert_array_equal(bs[:, 5], rs[:, 5])      # accepted moves
            np.testing.assert_allclose(bs[:, :5], rs[:, :5], rtol=1e-9, atol=1e-9)
        else:
            np.testing.assert_allclose(bs[:, 5], rs[:, 5], rtol=2e-2)


def test_graph_replay_equals_launches(contexts):
    X0 = _walkers(contexts, seed=7)
    b = BatchedSampler(contexts, [x.clone() for x in X0], STEPS, proposal=PROPS, cap=32)
    b.configure(128, [64, 64, 64], variant=2)
    b.reset(0)
    for _ in range(3):
        b.run(10, 5, 99)
    torch.cuda.synchronize()
    ref_X = [x.clone() for x in b.walkers]
    ref_S = [s.clone() for s in b.sums]
    for k in range(len(contexts)):
        b.walkers[k].copy_(X0[k])
    b.reset(0)
    b.capture(3, 10, 5, 99)
    b.replay()
    torch.cuda.synchronize()
    for k in range(len(contexts)):
        assert torch.equal(b.walkers[k], ref_X[k])
        np.testing.assert_allclose(b.sums[k][:6].cpu().numpy(), ref_S[k][:6].cpu().numpy(),
                                   rtol=1e-12, atol=1e-12)
    # the device counters advanced: a second replay fills the next six slots
    b.replay()
    torch.cuda.synchronize()
    assert float(b.sums[0][6:12, 6].sum()) == 6 * WALKERS[0]
    assert b.flags() == 0


def test_autotuner_picks_a_valid_shape(contexts):
    X0 = _walkers(contexts, seed=3)
    b = BatchedSampler(contexts, X0, STEPS, proposal=PROPS, cap=4)
    cfg, ms = b.tune(n_sweeps=4)
    assert ms > 0.0
    t = cfg["threads"]
    assert t in (64, 128, 256) and cfg["grid"] >= 1 and cfg["smem"] > 0
    for w in cfg["walkers_per_tile"]:
        assert w % 32 == 0 and t % w == 0
    b.reset(0)
    b.run(10, 5, 5)
    torch.cuda.synchronize()
    for k in range(len(contexts)):
        e, acc, nw = b.energies(k, 2)
        assert np.all(nw == WALKERS[k]) and np.all(np.isfinite(e))
    assert b.flags() == 0


def test_bad_tile_shapes_are_rejected(contexts):
    b = BatchedSampler(contexts, _walkers(contexts), STEPS, cap=1)
    with pytest.raises(ValueError):
        b.configure(128, [96, 64, 32])       # 96 does not divide 128
    with pytest.raises(ValueError):
        b.configure(256, [64, 64, 64], variant=1)   # variant 1 allows 128 threads
    with pytest.raises(ValueError):
        b.configure(128, [256, 64, 64])
    b.configure(64, [32, 32, 64])
    assert b.config()["threads"] == 64


def test_step_adaptation_reaches_the_target_acceptance(contexts):
    b = BatchedSampler(contexts, _walkers(contexts, seed=5), STEPS, proposal=PROPS, cap=8)
    b.configure(128, [64, 64, 64], variant=2)
    steps = b.adapt_steps(0.5, rounds=30)
    assert all(s > 0 for s in steps)
    b.reset(0)
    b.run(40, 20, 3)
    torch.cuda.synchronize()
    for k, c in enumerate(contexts):
        acc = float(b.sums[k][:2, 5].sum()) / (40 * WALKERS[k] * c.n_e)
        assert abs(acc - 0.5) < 0.1, (NAMES[k], acc)
    # switch molecule 0 to the nucleus-scaled proposal in place
    b.set_proposal(0, proposal="scaled", scale_r0=1.0, scale_fmin=0.02)
    assert b.config()["walkers_per_tile"] == [64, 64, 64]
    b.reset(0)
    b.run(10, 5, 4)
    torch.cuda.synchronize()
    assert b.flags() == 0


def test_full_size_headline_launch_is_consistent():
    """At the headline size (H2O, 65,536 walkers, mixed, nucleus-scaled): after
    50 sweeps in one persistent launch every walker is finite and measured,
    and the last sweep's walker-mean local energy (mixed, Sherman-Morrison
    state) equals the FP64 evaluation of the final positions to the mixed
    tolerance."""
    ctx = GTOContext(_system("H2O"))
    ctx.specialize()
    W = 65536
    X0 = torch.as_tensor(seeded_walkers(ctx.system, W, 1.0, 3), device="cuda")
    b = BatchedSampler([ctx], [X0], [0.6], precision="mixed", proposal="scaled",
                       scale_r0=1.0, scale_fmin=0.02, cap=64)
    b.tune(4, seed=5)
    b.reset(0)
    b.run(50, 1, 77)
    torch.cuda.synchronize()
    assert b.flags() == 0
    s = b.sums[0][:50].cpu().numpy()
    assert np.all(s[:, 6] == W)
    acc = s[:, 5].sum() / (50 * W * ctx.n_e)
    assert 0.2 < acc < 0.9
    X = b.walkers[0]
    assert torch.isfinite(X).all()
    ref = ctx.evaluate(X, want_grad=False, want_lap=False)["e_loc"]
    e_last = s[-1, 3] / s[-1, 6]
    assert abs(e_last - float(ref.mean())) < 1e-4 * max(1.0, float(ref.abs().mean()) / 10)


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_batch_lanes_with_bspline_and_three_body_jastrows(precision):
    """The lanes path splits the Jastrow change over the lanes (B-spline
    pairs and nuclei, the three-body term on lane 0): with B-spline and J3
    trials (golden cases the reference evaluated) at 2 and 4 lanes per
    walker a batched launch still leaves the per-system path's walkers."""
    from helpers import golden_system
    ctxs = []
    for name in ("h2o_bspline", "h2o_j3"):
        c = GTOContext(golden_system(name)[0])
        c.specialize()
        ctxs.append(c)
    X0 = [torch.as_tensor(seeded_walkers(c.system, 200, 0.8, 9 + k), device="cuda")
          for k, c in enumerate(ctxs)]
    steps, props = [0.5, 0.5], ["plain", "scaled"]
    b = BatchedSampler(ctxs, [x.clone() for x in X0], steps, precision=precision,
                       proposal=props, cap=8)
    b.configure(128, [64, 32], variant=0)            # 2 and 4 lanes per walker
    n, me, seed, base = 12, 4, 321, 40
    b.reset(base)
    b.run(n, me, seed)
    torch.cuda.synchronize()
    assert b.flags() == 0
    for k, ctx in enumerate(ctxs):
        X, sums = _per_system(ctx, X0[k], precision, props[k], steps[k], n, me, seed, base)
        same = torch.all((b.walkers[k] == X).reshape(X.shape[0], -1), dim=1)
        assert float(same.float().mean()) > 0.98, k
        bs = b.sums[k][: n // me].cpu().numpy()
        np.testing.assert_array_equal(bs[:, 6], sums.cpu().numpy()[:, 6])
