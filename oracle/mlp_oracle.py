"""CPU oracle of the learned Metropolis proposal (test infrastructure only).

The reference has no learned proposal: its sampler moves electrons with a
plain Gaussian random walk (``metropolis_move_alle``,
OmegaQMC/vmc_gto.py:815-839) and accepts with the Metropolis ratio
(``metropolis_move_1w``, vmc_gto.py:841-905).  The learned proposal replaces
the random-walk displacement of one electron by a draw from a Gaussian
mixture whose parameters a small MLP computes from the electron's
surroundings, and keeps the chain exact by multiplying the acceptance ratio
by q(x | x') / q(x' | x) (the Metropolis-Hastings correction, as the
reference's basin move does with its proposal densities, vmc_gto.py:925-957).

This module restates, in numpy, everything the CUDA kernels compute so the
tests can check them:
  * ``features``: the 32 inputs of electron e;
  * ``forward``: 32 -> 128 -> 128 -> 128 (ReLU) -> 48 outputs, optionally
    with the kernels' BF16 rounding of operands (FP32 accumulation);
  * ``mixture``: the 8-component isotropic Gaussian mixture the outputs
    define, its log-density, sampling and the negative log-likelihood;
  * ``backward``: the analytic gradient of the mean NLL with respect to all
    parameters (checked against finite differences in the CPU tests).
"""
from __future__ import annotations

import numpy as np

K0, H, NOUT, NMIX = 32, 128, 48, 8
SIG_MIN = 0.02
LOG2PI = float(np.log(2.0 * np.pi))

# flat FP32 parameter vector: W1 b1 W2 b2 W3 b3 W4 b4 (weights row-major [out][in])
SHAPES = [("W1", (H, K0)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)),
          ("W3", (H, H)), ("b3", (H,)), ("W4", (NOUT, H)), ("b4", (NOUT,))]
OFFSETS = {}
_o = 0
for _n, _s in SHAPES:
    OFFSETS[_n] = (_o, _s)
    _o += int(np.prod(_s))
N_PARAMS = _o


def unpack(theta):
    return {n: np.asarray(theta[o:o + int(np.prod(s))]).reshape(s) for n, (o, s) in OFFSETS.items()}


def pack(p):
    out = np.zeros(N_PARAMS, dtype=np.float64)
    for n, (o, s) in OFFSETS.items():
        out[o:o + int(np.prod(s))] = np.asarray(p[n]).reshape(-1)
    return out


def init_params(seed):
    """He-uniform hidden layers, a small output layer (initial mixture close
    to N(0, 0.71^2) per component)."""
    rng = np.random.default_rng(seed)
    p = {}
    for n, (o, s) in OFFSETS.items():
        if n.startswith("b"):
            p[n] = np.zeros(s)
        else:
            fan_in = s[1]
            lim = np.sqrt(6.0 / fan_in) * (0.1 if n == "W4" else 1.0)
            p[n] = rng.uniform(-lim, lim, size=s)
    return pack(p)


def bf16(x):
    """Round to bfloat16 (round to nearest, ties to even), returned as float32."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return (u.astype(np.uint32) << 16).view(np.float32).reshape(a.shape)


# ---------------------------------------------------------------------------
# features
# ---------------------------------------------------------------------------
def features(X, e, nuc):
    """Inputs of electron e for walkers X (W, n_e, 3): position relative to
    the nearest and second-nearest nucleus, displacements to the 8 nearest
    other electrons (nearest first; zeros when there are fewer), spin (+1 up
    for even e, -1 down) and a constant 1.  Ties go to the lower index."""
    X = np.asarray(X, dtype=np.float64)
    W, ne, _ = X.shape
    nuc = np.asarray(nuc, dtype=np.float64)
    xe = X[:, e, :]
    out = np.zeros((W, K0), dtype=np.float64)
    dn = np.linalg.norm(xe[:, None, :] - nuc[None], axis=2)          # (W, natm)
    order = np.argsort(dn, axis=1, kind="stable")
    i0 = order[:, 0]
    i1 = order[:, 1] if nuc.shape[0] > 1 else order[:, 0]
    out[:, 0:3] = xe - nuc[i0]
    out[:, 3:6] = xe - nuc[i1]
    others = [j for j in range(ne) if j != e]
    if others:
        D = X[:, others, :] - xe[:, None, :]                          # (W, ne-1, 3)
        r = np.linalg.norm(D, axis=2)
        o = np.argsort(r, axis=1, kind="stable")[:, :8]
        for k in range(o.shape[1]):
            out[:, 6 + 3 * k:9 + 3 * k] = D[np.arange(W), o[:, k]]
    out[:, 30] = 1.0 if e % 2 == 0 else -1.0
    out[:, 31] = 1.0
    return out


# ---------------------------------------------------------------------------
# network
# ---------------------------------------------------------------------------
def forward(theta, F, emulate_bf16=False):
    """Outputs (R, 48) and the hidden activations; with ``emulate_bf16`` the
    inputs, weights and hidden activations are rounded to BF16 as the tensor
    cores consume them (accumulation in FP64 here, FP32 on the GPU)."""
    p = unpack(theta)
    rnd = bf16 if emulate_bf16 else (lambda v: np.asarray(v, dtype=np.float64))
    h0 = rnd(F).astype(np.float64)
    acts = [h0]
    h = h0
    for l in (1, 2, 3):
        z = h @ rnd(p[f"W{l}"]).astype(np.float64).T + p[f"b{l}"]
        h = rnd(np.maximum(z, 0.0)).astype(np.float64)
        acts.append(h)
    out = h @ rnd(p["W4"]).astype(np.float64).T + p["b4"]
    return out, acts


def softplus(x):
    return np.logaddexp(0.0, x)


def sigmoid(x):
    return 0.5 * (1.0 + np.tanh(0.5 * x))


def mixture(out):
    """(log weights (R, 8), means (R, 8, 3), sigmas (R, 8)) of the outputs:
    logits 0..7, means 8..31, sigma = SIG_MIN + softplus(raw 32..39)."""
    a = out[:, 0:NMIX]
    logw = a - np.logaddexp.reduce(a, axis=1, keepdims=True)
    mu = out[:, NMIX:4 * NMIX].reshape(-1, NMIX, 3)
    sig = SIG_MIN + softplus(out[:, 4 * NMIX:5 * NMIX])
    return logw, mu, sig


def log_q(out, d):
    """log density of displacements d (R, 3) under the mixtures of ``out``."""
    logw, mu, sig = mixture(out)
    r2 = np.sum((d[:, None, :] - mu) ** 2, axis=2)
    L = logw - 3.0 * np.log(sig) - 1.5 * LOG2PI - 0.5 * r2 / sig ** 2
    return np.logaddexp.reduce(L, axis=1)


def sample(out, u_comp, n3):
    """Displacement from component c = first index with CDF > u_comp, then
    mu_c + sigma_c n3 (the device's rule)."""
    logw, mu, sig = mixture(out)
    cdf = np.cumsum(np.exp(logw), axis=1)
    c = np.minimum(np.sum(cdf <= u_comp[:, None], axis=1), NMIX - 1)
    R = np.arange(out.shape[0])
    return mu[R, c] + sig[R, c][:, None] * n3


def nll(theta, F, d, emulate_bf16=False):
    out, _ = forward(theta, F, emulate_bf16)
    return float(-np.mean(log_q(out, d)))


def output_grad(out, d):
    """d(-log q)/d(out) per row (R, 48)."""
    logw, mu, sig = mixture(out)
    diff = d[:, None, :] - mu
    r2 = np.sum(diff ** 2, axis=2)
    L = logw - 3.0 * np.log(sig) - 1.5 * LOG2PI - 0.5 * r2 / sig ** 2
    gam = np.exp(L - np.logaddexp.reduce(L, axis=1, keepdims=True))
    g = np.zeros_like(out)
    g[:, 0:NMIX] = np.exp(logw) - gam
    g[:, NMIX:4 * NMIX] = (-gam[:, :, None] * diff / sig[:, :, None] ** 2).reshape(-1, 3 * NMIX)
    dsig = -gam * (r2 / sig ** 3 - 3.0 / sig)
    g[:, 4 * NMIX:5 * NMIX] = dsig * sigmoid(out[:, 4 * NMIX:5 * NMIX])
    return g


def backward(theta, F, d, emulate_bf16=False):
    """Gradient of the mean NLL over the R rows with respect to theta.  With
    ``emulate_bf16`` the output gradients and the ReLU-masked hidden
    gradients are rounded to BF16 before each GEMM, as in the kernel."""
    p = unpack(theta)
    rnd = bf16 if emulate_bf16 else (lambda v: np.asarray(v, dtype=np.float64))
    out, acts = forward(theta, F, emulate_bf16)
    R = F.shape[0]
    dz = output_grad(out, d) / R
    g = {}
    for l in (4, 3, 2, 1):
        dzr = rnd(dz).astype(np.float64)
        g[f"W{l}"] = dzr.T @ acts[l - 1]
        g[f"b{l}"] = dzr.sum(axis=0)
        if l > 1:
            dh = dzr @ rnd(p[f"W{l}"]).astype(np.float64)
            dz = dh * (acts[l - 1] > 0)
    return pack(g)
