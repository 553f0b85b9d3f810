"""Learned proposal: the tensor-core network kernels against the CPU oracle
(oracle/mlp_oracle.py), training, and the sampler that uses it."""
import numpy as np
import pytest
import torch

from helpers import seeded_walkers
from oracle import gto_oracle as O
from oracle import mlp_oracle as P
from omegaqmc_b200 import molecules as M
from omegaqmc_b200.context import GTOContext
from omegaqmc_b200.learned import MLPProposal, collect_training_set, features, train_proposal
from omegaqmc_b200.sampler import WalkerEnsemble, NSUM
from omegaqmc_b200.system import build_system

pytestmark = pytest.mark.gpu


def _bf16_bits(x):
    """float array -> int16 tensor of BF16 bit patterns (round to nearest even)."""
    b = P.bf16(np.asarray(x, dtype=np.float32)).view(np.uint32) >> 16
    return torch.as_tensor(b.astype(np.uint16).view(np.int16), device="cuda")


def _bits_to_float(t):
    u = t.cpu().numpy().view(np.uint16).astype(np.uint32) << 16
    return u.view(np.float32)


@pytest.fixture(scope="module")
def n2():
    mf = M.make_mf("N2")
    s = build_system(mf, M.benchmark_params_corr(mf.mol))
    return s, GTOContext(s)


def _trained_like_params(seed):
    """Oracle-initialised parameters with a larger output layer, so that the
    outputs (and gradients) are not all near zero."""
    th = P.init_params(seed)
    o, _ = P.OFFSETS["W4"]
    th[o:o + P.NOUT * P.H] *= 10.0
    th[P.OFFSETS["b1"][0]:P.OFFSETS["b1"][0] + P.H] = 0.05
    return th.astype(np.float32)


def test_features_match_oracle(n2):
    s, ctx = n2
    X0 = seeded_walkers(s, 64, 1.0, 1)
    X1 = X0 + 0.1 * np.random.default_rng(2).normal(size=X0.shape)
    f, t = features(ctx, X0, X1)
    got = _bits_to_float(f).reshape(64, s.n_e, P.K0)
    for e in range(s.n_e):
        ref = P.bf16(P.features(X0, e, s.nuc).astype(np.float32))
        np.testing.assert_array_equal(got[:, e], ref)
    np.testing.assert_array_equal(t.cpu().numpy().reshape(64, s.n_e, 3),
                                  (X1 - X0).astype(np.float32))


@pytest.mark.parametrize("R", [128, 300])
def test_forward_matches_oracle(R):
    mlp = MLPProposal(seed=5)
    th = _trained_like_params(7)
    mlp.set_params(th)
    rng = np.random.default_rng(R)
    F = rng.normal(size=(R, P.K0)).astype(np.float32)
    F[:, 31] = 1.0
    out = mlp.forward(_bf16_bits(F)).cpu().numpy()
    ref, _ = P.forward(th.astype(np.float64), P.bf16(F).astype(np.float64), emulate_bf16=True)
    scale = np.abs(ref).max()
    assert np.max(np.abs(out - ref)) < 5e-3 * scale, np.max(np.abs(out - ref)) / scale
    assert mlp.flags() == 0


@pytest.mark.parametrize("R", [128, 300])
def test_gradients_match_oracle(R):
    mlp = MLPProposal(seed=5)
    th = _trained_like_params(11)
    mlp.set_params(th)
    rng = np.random.default_rng(100 + R)
    F = rng.normal(size=(R, P.K0)).astype(np.float32)
    F[:, 31] = 1.0
    d = (0.4 * rng.normal(size=(R, 3))).astype(np.float32)
    g, loss = mlp.backward(_bf16_bits(F), torch.as_tensor(d, device="cuda"))
    g = g.cpu().numpy()
    Fb = P.bf16(F).astype(np.float64)
    ref = P.backward(th.astype(np.float64), Fb, d.astype(np.float64), emulate_bf16=True)
    assert abs(loss - P.nll(th.astype(np.float64), Fb, d.astype(np.float64), True)) < 1e-3 * (1 + abs(loss))
    for name, (o, s) in P.OFFSETS.items():
        n = int(np.prod(s))
        a, b = g[o:o + n], ref[o:o + n]
        rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)
        assert rel < 2e-2, (name, rel)
    # and the emulated gradient is the exact gradient up to BF16 rounding
    exact = P.backward(th.astype(np.float64), Fb, d.astype(np.float64))
    assert np.linalg.norm(ref - exact) / np.linalg.norm(exact) < 5e-2
    assert mlp.flags() == 0


def test_training_reduces_the_loss(n2):
    s, ctx = n2
    ens = WalkerEnsemble(ctx, seeded_walkers(s, 2048, 1.0, 3), "mixed", seed=4)
    ens.run(300, 0.3)
    feat, tgt = collect_training_set(ens, 20000, 8, 0.3)
    mlp = MLPProposal(seed=1)
    hist = train_proposal(mlp, feat, tgt, steps=300, batch=4096, lr=2e-3, log_every=50)
    assert hist[-1][1] < hist[0][1] - 0.5, hist
    assert np.all(np.isfinite([h[1] for h in hist]))
    assert mlp.flags() == 0


def _tau_energy(sums):
    s = sums.cpu().numpy()
    ser = s[:, 3] / s[:, 6]
    m, se, _, kappa = O.binning_analysis(ser)
    return m, se, kappa, float(s[:, 5].sum())


def test_learned_proposal_is_exact_and_decorrelates_faster(n2):
    """N2, 16384 walkers: the plain fixed-width sampler and the learned
    proposal sample the same |psi|^2 (energies agree), and the learned one
    has a much shorter autocorrelation time of E_L per sweep and more
    decorrelated samples per second of GPU time."""
    s, ctx = n2
    ctx.specialize()
    W = 16384
    ens = WalkerEnsemble(ctx, seeded_walkers(s, W, 1.0, 9), "mixed", seed=21)
    step = 0.5
    ens.run(3000, step)
    # plain sampler: the comparison (and the source of the training data)
    n_plain = 6000
    sp = torch.zeros(n_plain, NSUM, dtype=torch.float64, device="cuda")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    ens.run(n_plain, step, sums=sp)
    e1.record()
    torch.cuda.synchronize()
    t_plain = e0.elapsed_time(e1) / n_plain
    mp, sep, kp, _ = _tau_energy(sp)
    feat, tgt = collect_training_set(ens, 10**6, 8, step)
    mlp = MLPProposal(seed=3)
    train_proposal(mlp, feat, tgt, steps=2000, batch=8192, lr=2e-3)
    del feat, tgt
    # learned proposal on a copy of the equilibrated walkers
    lens = WalkerEnsemble(ctx, ens.X, "mixed", seed=77)
    ctx.set_mlp_proposal(mlp)
    try:
        lens.run(100, step)
        n_l = 800
        sl = torch.zeros(n_l, NSUM, dtype=torch.float64, device="cuda")
        e0.record()
        lens.run(n_l, step, sums=sl)
        e1.record()
        torch.cuda.synchronize()
        t_l = e0.elapsed_time(e1) / n_l
    finally:
        ctx.set_mlp_proposal(None)
    ml, sel, kl, accl = _tau_energy(sl)
    acc = accl / (n_l * W * s.n_e)
    assert ctx.flags() == 0 and mlp.flags() == 0
    assert acc > 0.2
    assert abs(ml - mp) < 4.0 * np.hypot(sel, sep), (ml, sel, mp, sep)
    assert kl < kp / 5.0, (kl, kp)
    # decorrelated samples per second: W / (tau * seconds per sweep)
    assert (1.0 / (kl * t_l)) > 1.5 * (1.0 / (kp * t_plain)), (kl, t_l, kp, t_plain)
