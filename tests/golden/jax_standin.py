"""A small torch-backed stand-in for the parts of JAX the reference's
wavefunction code uses, so that code can be run unmodified on the CPU to
produce golden vectors (JAX and PySCF are not installed here).

Only fixture generation uses this module (``make_golden.py``); nothing in
the package or the GPU tests imports it.

Coverage: ``jax.jit`` (identity), ``jax.vmap`` (a loop over the mapped
axis), ``jax.grad`` / ``jax.jacobian`` (torch autograd, float64),
``jax.numpy`` (the functions the GTO path calls, mapped to torch),
``x.at[idx].set/add`` (functional updates; ``add`` accumulates repeated
indices like JAX), ``jax.lax.while_loop``, ``jax.scipy.signal.fftconvolve``.
"""
from __future__ import annotations

import math
import sys
import types

import numpy as np
import torch

torch.set_default_dtype(torch.float64)


def _t(x):
    """Convert to a float64/int64/bool tensor (recursively for lists)."""
    if isinstance(x, torch.Tensor):
        return x
    if isinstance(x, (list, tuple)):
        if len(x) and any(isinstance(e, (torch.Tensor, list, tuple)) for e in x):
            parts = [_t(e) for e in x]
            dt = torch.promote_types(parts[0].dtype, torch.float64) \
                if any(p.is_floating_point() for p in parts) else parts[0].dtype
            return torch.stack([p.to(dt) for p in parts])
        return _t(np.asarray(x))
    if isinstance(x, np.ndarray):
        if x.dtype == np.float32:
            x = x.astype(np.float64)
        return torch.from_numpy(np.ascontiguousarray(x).copy())
    if isinstance(x, (bool, np.bool_)):
        return torch.tensor(bool(x))
    if isinstance(x, (int, np.integer)):
        return torch.tensor(int(x), dtype=torch.int64)
    if isinstance(x, (float, np.floating)):
        return torch.tensor(float(x), dtype=torch.float64)
    return torch.as_tensor(x)


def _f(x):
    t = _t(x)
    return t if t.is_floating_point() else t.to(torch.float64)


# ---------------------------------------------------------------------------
# .at[...] functional updates
# ---------------------------------------------------------------------------
def _norm_index(idx):
    if not isinstance(idx, tuple):
        idx = (idx,)
    return tuple(_t(i) if isinstance(i, (np.ndarray, list)) else i for i in idx)


class _AtRef:
    def __init__(self, arr, idx):
        self.arr = arr
        self.idx = _norm_index(idx)

    def set(self, val):
        out = self.arr.clone()
        out[self.idx] = _t(val).to(out.dtype)
        return out

    def add(self, val):
        out = self.arr.clone()
        adv = [i for i in self.idx if isinstance(i, torch.Tensor)]
        if adv and all(isinstance(i, torch.Tensor) for i in self.idx):
            v = _t(val).to(out.dtype)
            tgt_shape = out[self.idx].shape
            out.index_put_(self.idx, v.expand(tgt_shape), accumulate=True)
            return out
        out[self.idx] = out[self.idx] + _t(val).to(out.dtype)
        return out


class _At:
    def __init__(self, arr):
        self.arr = arr

    def __getitem__(self, idx):
        return _AtRef(self.arr, idx)


_orig_getitem = torch.Tensor.__getitem__


def _getitem(self, idx):
    # JAX/numpy reverse slices (x[::-1]); torch slicing needs step > 0
    if isinstance(idx, slice) and idx.step is not None and idx.step < 0:
        if idx.step == -1 and idx.start is None and idx.stop is None:
            return torch.flip(self, [0])
        raise NotImplementedError("only x[::-1] reverse slices are supported")
    return _orig_getitem(self, idx)


torch.Tensor.__getitem__ = _getitem
# JAX arrays are immutable: augmented assignment rebinds the name
torch.Tensor.__iadd__ = lambda self, o: self + o
torch.Tensor.__isub__ = lambda self, o: self - o
torch.Tensor.__imul__ = lambda self, o: self * o
torch.Tensor.__itruediv__ = lambda self, o: self / o
torch.Tensor.at = property(lambda self: _At(self))
torch.Tensor.astype = lambda self, dt: self.to(dt)
torch.Tensor.copy = lambda self: self.clone()


# ---------------------------------------------------------------------------
# jax.numpy
# ---------------------------------------------------------------------------
jnp = types.ModuleType("jax.numpy")
jnp.pi = math.pi
jnp.float64 = torch.float64
jnp.float32 = torch.float32
jnp.int32 = torch.int32
jnp.int64 = torch.int64
jnp.bool_ = torch.bool
jnp.newaxis = None
jnp.ndarray = torch.Tensor


def _axis_kw(kw):
    if "axis" in kw:
        kw["dim"] = kw.pop("axis")
    if "keepdims" in kw:
        kw["keepdim"] = kw.pop("keepdims")
    return kw


def _array(x, dtype=None):
    t = _t(x)
    if dtype is not None:
        t = t.to(dtype if isinstance(dtype, torch.dtype) else torch.float64)
    return t


jnp.array = _array
jnp.asarray = _array
jnp.zeros = lambda shape, dtype=None: torch.zeros(shape, dtype=dtype or torch.float64)
jnp.ones = lambda shape, dtype=None: torch.ones(shape, dtype=dtype or torch.float64)
jnp.zeros_like = lambda x, dtype=None: torch.zeros_like(_f(x), dtype=dtype)
jnp.ones_like = lambda x, dtype=None: torch.ones_like(_f(x), dtype=dtype)
jnp.eye = lambda n, dtype=None: torch.eye(n, dtype=dtype or torch.float64)
jnp.arange = lambda *a, **k: torch.arange(*a, **k)


def _sum(x, axis=None, keepdims=False, **kw):
    x = _t(x)
    if axis is None:
        return x.sum()
    return x.sum(dim=axis, keepdim=keepdims)


jnp.sum = _sum
jnp.mean = lambda x, axis=None, keepdims=False: (
    _f(x).mean() if axis is None else _f(x).mean(dim=axis, keepdim=keepdims))
jnp.std = lambda x, axis=None: (
    _f(x).std(unbiased=False) if axis is None else _f(x).std(dim=axis, unbiased=False))
jnp.max = lambda x, axis=None: _t(x).max() if axis is None else _t(x).amax(dim=axis)
jnp.min = lambda x, axis=None: _t(x).min() if axis is None else _t(x).amin(dim=axis)
for _name in ("exp", "log", "sqrt", "abs", "sin", "cos", "tanh", "isfinite",
              "isnan", "floor", "sign", "log1p", "expm1"):
    setattr(jnp, _name, (lambda fn: (lambda x: fn(_f(x))))(getattr(torch, _name)))
jnp.square = lambda x: _f(x) * _f(x)
jnp.power = lambda x, y: torch.pow(_f(x), _t(y))
jnp.maximum = lambda a, b: torch.maximum(_f(a), _f(b))
jnp.minimum = lambda a, b: torch.minimum(_f(a), _f(b))


def _where(c, a=None, b=None):
    if a is None:
        return torch.where(_t(c))
    a, b = _t(a), _t(b)
    if a.is_floating_point() or b.is_floating_point():
        a, b = a.to(torch.float64), b.to(torch.float64)
    return torch.where(_t(c), a, b)


jnp.where = _where
jnp.all = lambda x: torch.all(_t(x))
jnp.logical_and = lambda a, b: torch.logical_and(_t(a), _t(b))
jnp.logical_or = lambda a, b: torch.logical_or(_t(a), _t(b))
jnp.any = lambda x: torch.any(_t(x))
jnp.concatenate = lambda xs, axis=0: torch.cat([_t(x) for x in xs], dim=axis)
jnp.stack = lambda xs, axis=0: torch.stack([_t(x) for x in xs], dim=axis)
jnp.ravel = lambda x: _t(x).reshape(-1)
jnp.broadcast_to = lambda x, shape: _t(x).expand(*shape)


def _searchsorted(a, v, side="left"):
    a, v = _t(a), _t(v)
    out = torch.searchsorted(a, v.reshape(-1), right=(side == "right"))
    return out.reshape(v.shape)


jnp.searchsorted = _searchsorted
jnp.count_nonzero = lambda x: torch.count_nonzero(_t(x))
jnp.finfo = lambda dt: torch.finfo(dt if isinstance(dt, torch.dtype) else torch.float64)
jnp.einsum = lambda eq, *ops: torch.einsum(eq, *[_f(o) for o in ops])
jnp.dot = lambda a, b: _f(a) @ _f(b)
jnp.outer = lambda a, b: torch.outer(_f(a), _f(b))
jnp.take = lambda x, idx, axis=None: torch.index_select(_t(x), axis, _t(idx))
jnp.clip = lambda x, a=None, b=None: torch.clamp(_t(x), a, b)


def _triu(n, k=0, m=None):
    ij = torch.triu_indices(n, m if m is not None else n, offset=k)
    return ij[0], ij[1]


jnp.triu_indices = _triu
jnp.trace = lambda x: torch.trace(_f(x))

linalg = types.ModuleType("jax.numpy.linalg")
linalg.slogdet = lambda x: tuple(torch.linalg.slogdet(_f(x)))
linalg.inv = lambda x: torch.linalg.inv(_f(x))
linalg.det = lambda x: torch.linalg.det(_f(x))
linalg.norm = lambda x, axis=None, keepdims=False: (
    torch.linalg.vector_norm(_f(x)) if axis is None
    else torch.linalg.vector_norm(_f(x), dim=axis, keepdim=keepdims))
jnp.linalg = linalg


# ---------------------------------------------------------------------------
# transformations
# ---------------------------------------------------------------------------
def jit(fun=None, **kw):
    if fun is None:
        return lambda f: f
    return fun


def _stack_tree(outs):
    first = outs[0]
    if isinstance(first, tuple):
        return tuple(_stack_tree([o[k] for o in outs]) for k in range(len(first)))
    if isinstance(first, list):
        return [_stack_tree([o[k] for o in outs]) for k in range(len(first))]
    return torch.stack([_t(o) for o in outs])


def vmap(fun, in_axes=0, out_axes=0):
    def wrapped(*args):
        axes = in_axes if isinstance(in_axes, (tuple, list)) else (in_axes,) * len(args)
        n = None
        for a, ax in zip(args, axes):
            if ax is not None:
                n = _t(a).shape[ax]
                break
        outs = []
        for k in range(n):
            call = [(_t(a).select(ax, k) if ax is not None else a)
                    for a, ax in zip(args, axes)]
            outs.append(fun(*call))
        return _stack_tree(outs)
    return wrapped


def grad(fun, argnums=0):
    def g(*args):
        args = list(args)
        x = _f(args[argnums])
        if not x.requires_grad:
            x = x.detach().clone().requires_grad_(True)
        args[argnums] = x
        y = fun(*args)
        if not (isinstance(y, torch.Tensor) and y.requires_grad):
            return torch.zeros_like(x)
        (gx,) = torch.autograd.grad(y, x, create_graph=True, allow_unused=True)
        return torch.zeros_like(x) if gx is None else gx
    return g


def jacobian(fun):
    def j(x):
        x = _f(x)
        return torch.autograd.functional.jacobian(lambda z: _t(fun(z)), x,
                                                  create_graph=True)
    return j


def hessian(fun):
    def h(x):
        x = _f(x)
        return torch.autograd.functional.hessian(lambda z: fun(z), x,
                                                 create_graph=False)
    return h


lax = types.ModuleType("jax.lax")


def _while_loop(cond, body, init):
    v = init
    while bool(cond(v)):
        v = body(v)
    return v


lax.while_loop = _while_loop
lax.cond = lambda p, t, f, *a: t(*a) if bool(p) else f(*a)

scipy = types.ModuleType("jax.scipy")
signal = types.ModuleType("jax.scipy.signal")


def _fftconvolve(a, b, mode="full"):
    import scipy.signal as ss
    return _t(ss.fftconvolve(_t(a).detach().numpy(), _t(b).detach().numpy(), mode=mode))


signal.fftconvolve = _fftconvolve
special = types.ModuleType("jax.scipy.special")
special.logsumexp = lambda x, axis=None: torch.logsumexp(
    _f(x), dim=axis if axis is not None else tuple(range(_t(x).ndim)))
scipy.signal = signal
scipy.special = special

sharding = types.ModuleType("jax.sharding")
sharding.Mesh = type("Mesh", (), {})
sharding.NamedSharding = type("NamedSharding", (), {})
sharding.PartitionSpec = type("PartitionSpec", (), {})


class _Config:
    def update(self, *a, **k):
        pass


jax = types.ModuleType("jax")
jax.jit = jit
jax.vmap = vmap
jax.grad = grad
jax.jacobian = jacobian
jax.hessian = hessian
jax.numpy = jnp
jax.lax = lax
jax.scipy = scipy
jax.sharding = sharding
jax.config = _Config()
jax.Array = torch.Tensor


def install():
    """Register the stand-in as ``jax`` in ``sys.modules``."""
    sys.modules["jax"] = jax
    sys.modules["jax.numpy"] = jnp
    sys.modules["jax.numpy.linalg"] = linalg
    sys.modules["jax.lax"] = lax
    sys.modules["jax.scipy"] = scipy
    sys.modules["jax.scipy.signal"] = signal
    sys.modules["jax.scipy.special"] = special
    sys.modules["jax.sharding"] = sharding
