"""ctypes binding of liboqmc_b200.so (declared in include/oqmc_b200.h).

The library is built in-tree by ``omegaqmc_b200.build``.  Loading fails
loudly when it is missing: there is no CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboqmc_b200.so")

OQ_OK = 0
OQ_ERR_ARG = -1
OQ_ERR_CUDA = -2
OQ_ERR_NAN = -3
OQ_ERR_SINGULAR = -4
OQ_ERR_TIMEOUT = -5
OQ_ERR_UNSUPPORTED = -6
OQ_ERR_NOMEM = -7
OQ_FLAG_NAN = 1
OQ_FLAG_SINGULAR = 2
PREC_FP64 = 0
PREC_MIXED = 1

c_int, c_double, c_void_p, c_size_t, c_uint64 = (
    ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint64)
P_int = ctypes.POINTER(ctypes.c_int)
P_double = ctypes.POINTER(ctypes.c_double)


class SystemDesc(ctypes.Structure):
    """Mirror of ``oqmc_system_desc``."""
    _fields_ = [
        ("natm", c_int), ("nbf", c_int), ("nocc", c_int), ("n_e", c_int),
        ("nuc", P_double), ("Z", P_double),
        ("ngroup", c_int),
        ("group_atom", P_int), ("group_am", P_int), ("group_nprim", P_int),
        ("group_ncol", P_int),
        ("alpha", P_double), ("norm", P_double), ("shell_cusp", P_int),
        ("C", P_double),
        ("has_j1", c_int), ("j1", P_double),
        ("has_j2", c_int), ("j2", P_double),
        ("cusp", c_int), ("cusp_rc", P_double), ("cusp_q0", P_double),
        ("cusp_coeff", P_double),
        ("e_nn", c_double),
        ("has_bs2", c_int), ("bs2_ncoef_like", c_int), ("bs2_ncoef_unlike", c_int),
        ("bs2_rcut", c_double), ("bs2_coef_like", P_double), ("bs2_coef_unlike", P_double),
        ("has_bs1", c_int), ("bs1_ntype", c_int), ("bs1_type", P_int), ("bs1_ncoef", P_int),
        ("bs1_rcut", P_double), ("bs1_coef", P_double),
        ("has_j3", c_int), ("j3_n_ei", c_int), ("j3_n_ee", c_int), ("j3_ntype", c_int),
        ("j3_rcut", c_double), ("j3_type", P_int), ("j3_on", P_int), ("j3_gamma", P_double),
        ("has_spl", c_int), ("spl_npts", c_int), ("spl_ntab", c_int), ("spl_smin", c_double),
        ("spl_shell", P_int), ("spl_knots", P_double), ("spl_coef", P_double),
    ]


class BatchSystem(ctypes.Structure):
    """Mirror of ``oqmc_batch_system``."""
    _fields_ = [
        ("walkers", c_void_p), ("W", c_int), ("proposal", c_int),
        ("step", c_double), ("scale_r0", c_double), ("scale_fmin", c_double),
        ("sums", c_void_p), ("cap", c_int),
    ]


class OqmcError(RuntimeError):
    """A liboqmc_b200 call failed; ``code`` is the OQ_ERR_* status."""

    def __init__(self, code, msg):
        super().__init__(f"liboqmc_b200 error {code}: {msg}")
        self.code = code


_lib = None

# (name, restype, argtypes)
_SIGS = [
    ("oqmc_version", ctypes.c_char_p, []),
    ("oqmc_set_move_kind", c_int, [c_void_p, c_int]),
    ("oqmc_set_multidet", c_int, [c_void_p, c_int, c_int, P_double, P_double, P_int, P_int]),
    ("oqmc_multidet_info", c_int, [c_void_p, ctypes.POINTER(c_int), ctypes.POINTER(c_int),
                                   ctypes.POINTER(c_int), ctypes.POINTER(c_int)]),
    ("oqmc_create", c_int, [ctypes.POINTER(c_void_p), ctypes.POINTER(SystemDesc)]),
    ("oqmc_destroy", c_int, [c_void_p]),
    ("oqmc_last_error", ctypes.c_char_p, [c_void_p]),
    ("oqmc_eval", c_int, [c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_void_p,
                          c_void_p, c_void_p]),
    ("oqmc_log_psi", c_int, [c_void_p, c_void_p, c_int, c_void_p, c_void_p]),
    ("oqmc_mo_values", c_int, [c_void_p, c_void_p, c_int, c_void_p, c_void_p]),
    ("oqmc_state_bytes", c_size_t, [c_void_p, c_int, c_int]),
    ("oqmc_refresh", c_int, [c_void_p, c_void_p, c_int, c_void_p, c_int, c_void_p]),
    ("oqmc_state_eval", c_int, [c_void_p, c_void_p, c_int, c_int, c_void_p, c_void_p,
                                c_void_p, c_void_p, c_void_p]),
    ("oqmc_equilibrate", c_int, [c_void_p, c_void_p, c_int, c_void_p, c_int, c_int, c_void_p,
                                 c_double, c_double, c_uint64, c_uint64, c_int, c_int,
                                 c_void_p, c_void_p, c_void_p]),
    ("oqmc_sweeps", c_int, [c_void_p, c_void_p, c_int, c_void_p, c_int, c_int, c_int,
                            c_double, c_uint64, c_uint64, c_void_p, c_void_p, c_void_p,
                            c_int, c_void_p]),
    ("oqmc_basin", c_int, [c_void_p, c_void_p, c_int, c_void_p, c_int, c_int, c_double,
                           c_uint64, c_uint64, c_void_p, c_void_p]),
    ("oqmc_sweeps_noalloc", c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_int,
                                    c_double, c_uint64, c_uint64, c_void_p, c_void_p,
                                    c_void_p, c_void_p]),
    ("oqmc_set_proposal", c_int, [c_void_p, c_int, c_double, c_double]),
    ("oqmc_specialize", c_int, [c_void_p, c_int]),
    ("oqmc_use_tensor_cores", c_int, [c_void_p, c_int]),
    ("oqmc_spec_source", c_int, [c_void_p, ctypes.c_char_p, c_size_t]),
    ("oqmc_spec_source_desc", c_int, [ctypes.POINTER(SystemDesc), ctypes.c_char_p, c_size_t]),
    ("oqmc_set_split", c_int, [c_void_p, c_double]),
    ("oqmc_get_flags", c_int, [c_void_p, ctypes.POINTER(ctypes.c_uint), c_int, c_void_p]),
    ("oqmc_measure_peak", c_int, [c_int, P_double, c_void_p]),
    ("oqmc_batch_create", c_int, [ctypes.POINTER(c_void_p), ctypes.POINTER(c_void_p), c_int,
                                  c_int]),
    ("oqmc_batch_destroy", c_int, [c_void_p]),
    ("oqmc_batch_last_error", ctypes.c_char_p, [c_void_p]),
    ("oqmc_batch_bind", c_int, [c_void_p, ctypes.POINTER(BatchSystem)]),
    ("oqmc_batch_configure", c_int, [c_void_p, c_int, P_int, c_int]),
    ("oqmc_batch_get_config", c_int, [c_void_p, P_int, P_int, P_int, P_int,
                                      ctypes.POINTER(c_size_t), P_int, P_int]),
    ("oqmc_batch_tune", c_int, [c_void_p, c_int, c_uint64, c_void_p,
                                ctypes.POINTER(ctypes.c_float)]),
    ("oqmc_batch_reset", c_int, [c_void_p, c_uint64, c_void_p]),
    ("oqmc_batch_run", c_int, [c_void_p, c_int, c_int, c_uint64, c_void_p]),
    ("oqmc_batch_capture", c_int, [c_void_p, c_int, c_int, c_int, c_uint64]),
    ("oqmc_batch_replay", c_int, [c_void_p, c_void_p]),
    ("oqmc_batch_busy", c_int, [c_void_p, ctypes.POINTER(ctypes.c_ulonglong), c_void_p]),
    ("oqmc_batch_get_flags", c_int, [c_void_p, ctypes.POINTER(ctypes.c_uint), c_int, c_void_p]),
    ("oqmc_batch_source_desc", c_int, [ctypes.POINTER(SystemDesc), c_int, ctypes.c_char_p,
                                       c_size_t, ctypes.POINTER(c_size_t)]),
    ("oqmc_mlp_num_params", c_int, []),
    ("oqmc_mlp_create", c_int, [ctypes.POINTER(c_void_p), c_uint64]),
    ("oqmc_mlp_destroy", c_int, [c_void_p]),
    ("oqmc_mlp_last_error", ctypes.c_char_p, [c_void_p]),
    ("oqmc_mlp_get_params", c_int, [c_void_p, ctypes.POINTER(ctypes.c_float)]),
    ("oqmc_mlp_set_params", c_int, [c_void_p, ctypes.POINTER(ctypes.c_float)]),
    ("oqmc_mlp_features", c_int, [c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_void_p,
                                  c_void_p]),
    ("oqmc_mlp_forward", c_int, [c_void_p, c_void_p, c_int, c_void_p, c_void_p]),
    ("oqmc_mlp_backward", c_int, [c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_void_p,
                                  c_void_p]),
    ("oqmc_mlp_step", c_int, [c_void_p, c_void_p, c_void_p, c_int, ctypes.c_float, c_void_p,
                              c_void_p]),
    ("oqmc_mlp_get_flags", c_int, [c_void_p, ctypes.POINTER(ctypes.c_uint), c_int, c_void_p]),
    ("oqmc_set_mlp_proposal", c_int, [c_void_p, c_void_p]),
    ("oqmc_set_mlp_groups", c_int, [c_void_p, c_int]),
    ("oqmc_param_count", c_int, [c_void_p]),
    ("oqmc_param_derivs", c_int, [c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_void_p,
                                  c_void_p]),
]

EXPORTED = [s[0] for s in _SIGS]


def load(path=None):
    """Load (once) and return the library handle with typed entry points."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or LIB_PATH
    if not os.path.exists(path):
        raise ImportError(
            f"{path} is missing: build it with `python -m omegaqmc_b200.build` "
            "(there is no CPU fallback)")
    lib = ctypes.CDLL(path)
    for name, res, args in _SIGS:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(code, ctx=None, batch=False, mlp=False):
    """Raise for a negative status, with the library's message (of a context,
    of a batch handle when ``batch`` is true, of a network when ``mlp``)."""
    if code == OQ_OK:
        return
    lib = load()
    msg = (lib.oqmc_batch_last_error(ctx) if batch else
           lib.oqmc_mlp_last_error(ctx) if mlp else lib.oqmc_last_error(ctx))
    msg = msg.decode(errors="replace")
    if code == OQ_ERR_ARG:
        raise ValueError(msg)
    if code == OQ_ERR_UNSUPPORTED:
        raise NotImplementedError(msg)
    raise OqmcError(code, msg)
