"""The learned-proposal oracle: analytic gradients against finite
differences, the mixture density against sampling, and the features."""
import numpy as np

from oracle import mlp_oracle as P


def _data(R=64, seed=0):
    rng = np.random.default_rng(seed)
    F = rng.normal(size=(R, P.K0))
    F[:, 31] = 1.0
    d = rng.normal(scale=0.5, size=(R, 3))
    return F, d


def test_backward_matches_finite_differences():
    theta = P.init_params(3)
    theta[P.OFFSETS["W4"][0]:P.OFFSETS["W4"][0] + P.NOUT * P.H] *= 10.0   # larger outputs
    F, d = _data()
    g = P.backward(theta, F, d)
    rng = np.random.default_rng(1)
    idx = rng.choice(P.N_PARAMS, 60, replace=False)
    for n in ("b1", "b4", "W1", "W4"):              # make sure every block is probed
        o, s = P.OFFSETS[n]
        idx = np.append(idx, o + int(np.prod(s)) // 2)
    eps = 1e-6
    for i in idx:
        tp, tm = theta.copy(), theta.copy()
        tp[i] += eps
        tm[i] -= eps
        fd = (P.nll(tp, F, d) - P.nll(tm, F, d)) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])


def test_output_gradient_of_unused_outputs_is_zero():
    theta = P.init_params(4)
    F, d = _data(16)
    out, _ = P.forward(theta, F)
    g = P.output_grad(out, d)
    assert np.all(g[:, 40:] == 0.0)


def test_mixture_density_integrates_to_one_and_matches_sampling():
    theta = P.init_params(5)
    theta[P.OFFSETS["W4"][0]:P.OFFSETS["W4"][0] + P.NOUT * P.H] *= 8.0
    F, _ = _data(1, seed=2)
    out, _ = P.forward(theta, F)
    rng = np.random.default_rng(0)
    N = 200000
    outs = np.repeat(out, N, axis=0)
    d = P.sample(outs, rng.uniform(size=N), rng.normal(size=(N, 3)))
    # importance check: E_q[1/q] over a box equals its volume only if q is
    # normalised; use a Gaussian-smoothed histogram check on the x marginal
    lq = P.log_q(outs[:2000], d[:2000])
    assert np.all(np.isfinite(lq))
    # grid integration of the density over a box that holds the mass
    lo, hi = d.min(axis=0) - 1.0, d.max(axis=0) + 1.0
    g = [np.linspace(lo[k], hi[k], 61) for k in range(3)]
    G = np.stack(np.meshgrid(*g, indexing="ij"), axis=-1).reshape(-1, 3)
    q = np.exp(P.log_q(np.repeat(out, G.shape[0], axis=0), G))
    vol = np.prod([(g[k][1] - g[k][0]) for k in range(3)])
    assert abs(q.sum() * vol - 1.0) < 0.02
    # sample mean equals the mixture mean
    logw, mu, sig = P.mixture(out)
    mean = np.sum(np.exp(logw)[0][:, None] * mu[0], axis=0)
    assert np.allclose(d.mean(axis=0), mean, atol=5e-3 + 3 * d.std(axis=0).max() / np.sqrt(N))


def test_features_layout():
    nuc = np.array([[0.0, 0.0, -1.0], [0.0, 0.0, 1.0]])
    X = np.zeros((1, 10, 3))
    X[0, :, 2] = np.linspace(-2.0, 2.0, 10)
    X[0, 3, 0] = 0.1
    f = P.features(X, 3, nuc)
    xe = X[0, 3]
    assert np.allclose(f[0, 0:3], xe - nuc[0])          # nucleus at z=-1 is nearer
    assert np.allclose(f[0, 3:6], xe - nuc[1])
    r = [np.linalg.norm(X[0, j] - xe) for j in range(10) if j != 3]
    near = np.sort(r)[:8]
    got = np.linalg.norm(f[0, 6:30].reshape(8, 3), axis=1)
    assert np.allclose(got, near)
    assert f[0, 30] == -1.0 and f[0, 31] == 1.0
    # fewer than 8 other electrons: zero padding
    f2 = P.features(X[:, :4], 0, nuc)
    assert np.all(f2[0, 6 + 9:30] == 0.0)


def test_bf16_rounding_is_round_to_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 1e-3], dtype=np.float32)
    y = P.bf16(x)
    assert y[0] == 1.0 and y[1] == 1.0            # tie to even
    assert y[2] == np.float32(1.0 + 2 ** -7)      # above the tie rounds up
    assert y[3] == -2.5
    assert abs(y[4] - 1e-3) / 1e-3 < 2 ** -8
