"""ctypes binding of the oracle's C restatement (TEST INFRASTRUCTURE).

``liboracle_vmc.so`` is built from ``oracle/vmc_ref.c`` by
``oracle/build_oracle.py``.  Only the tests and the benchmark's CPU-baseline
leg load it.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import build_oracle

_lib = None


def load():
    global _lib
    if _lib is None:
        path = build_oracle.build()
        if path is None:
            raise ImportError("oracle/vmc_ref.c is missing")
        lib = ctypes.CDLL(path)
        lib.vmc_ref_eval.restype = ctypes.c_int
        lib.vmc_ref_eval.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                     ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        lib.vmc_ref_run.restype = ctypes.c_int
        lib.vmc_ref_run.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                    ctypes.c_int, ctypes.c_double, ctypes.c_uint64,
                                    ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        _lib = lib
    return _lib


def _desc(system):
    from omegaqmc_b200.context import pack_system
    return pack_system(system)


def supports(system):
    """True when the C restatement covers the system's trial (Padé J1/J2,
    cusp-corrected s shells, one determinant)."""
    return (system.md is None and system.bs1 is None and system.bs2 is None
            and system.j3 is None and system.spl is None)


def _check(system):
    if not supports(system):
        raise ValueError("the C restatement covers Padé Jastrows, cusp-corrected s shells "
                         "and single determinants only")


def evaluate(system, X, nthreads=0):
    """(logpsi (W,), eparts (W, 4): e_ee, e_en, e_ke, E_L) from the C
    restatement."""
    _check(system)
    d, keep = _desc(system)
    X = np.ascontiguousarray(X, dtype=np.float64)
    W = X.shape[0]
    lp = np.empty(W)
    ep = np.empty((W, 4))
    rc = load().vmc_ref_eval(ctypes.byref(d), X.ctypes.data, W, lp.ctypes.data,
                             ep.ctypes.data, int(nthreads))
    if rc != 0:
        raise ValueError("descriptor outside the C restatement")
    return lp, ep


def run(system, X, n_steps, step, seed=0, nthreads=0):
    """Reference-algorithm steps in place on X; returns (series (n,4), acc)."""
    _check(system)
    d, keep = _desc(system)
    assert X.dtype == np.float64 and X.flags.c_contiguous
    series = np.empty((n_steps, 4))
    acc = ctypes.c_double(0.0)
    load().vmc_ref_run(ctypes.byref(d), X.ctypes.data, X.shape[0], int(n_steps),
                       float(step), ctypes.c_uint64(seed), series.ctypes.data,
                       ctypes.byref(acc), int(nthreads))
    return series, acc.value
