"""Compile the run-time specialised kernels of a system with NVRTC on the
host (no GPU needed): the same source and options the library uses in
``oqmc_specialize``, for checking and inspection."""
from __future__ import annotations

import ctypes
import os

from omegaqmc_b200 import _lib as L
from omegaqmc_b200.context import pack_system

CSRC = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "omegaqmc_b200", "csrc")
HEADERS = ("oqmc_common.cuh", "oqmc_ao.cuh", "oqmc_eval.cuh", "oqmc_sweep.cuh", "oqmc_batch.cuh",
           "oqmc_tc.cuh", "oqmc_mlp.cuh", "oqmc_mlp_sweep.cuh")


def spec_source(system):
    """The generated specialisation source of ``system``."""
    lib = L.load()
    d, keep = pack_system(system)
    n = lib.oqmc_spec_source_desc(ctypes.byref(d), None, 0)
    L.check(min(n, 0), None)
    buf = ctypes.create_string_buffer(n + 1)
    lib.oqmc_spec_source_desc(ctypes.byref(d), buf, n + 1)
    return buf.value.decode()


def _nvrtc():
    for n in ("libnvrtc.so.12", "libnvrtc.so", "/usr/local/cuda/lib64/libnvrtc.so.12"):
        try:
            return ctypes.CDLL(n)
        except OSError:
            continue
    raise OSError("libnvrtc not found")


def batch_source(systems):
    """The generated source of the batched kernel for a list of systems."""
    lib = L.load()
    packed = [pack_system(s) for s in systems]
    arr = (L.SystemDesc * len(systems))(*[p[0] for p in packed])
    n = ctypes.c_size_t()
    L.check(lib.oqmc_batch_source_desc(arr, len(systems), None, 0, ctypes.byref(n)), None, True)
    buf = ctypes.create_string_buffer(n.value + 1)
    L.check(lib.oqmc_batch_source_desc(arr, len(systems), buf, n.value + 1, None), None, True)
    return buf.value.decode()


BATCH_KERNELS = [f"k_batch<{t}, {mt}, {mb}>" for t in ("float, float", "double, double")
                 for mt, mb in ((256, 1), (128, 3), (256, 2))]


def compile_source(src, names):
    """NVRTC-compile ``src`` with the library's headers and options for
    sm_100a; returns (ok, log, cubin bytes)."""
    nv = _nvrtc()
    hs = [open(os.path.join(CSRC, h), "rb").read() for h in HEADERS]
    prog = ctypes.c_void_p()
    arr_s = (ctypes.c_char_p * len(hs))(*hs)
    arr_n = (ctypes.c_char_p * len(hs))(*[h.encode() for h in HEADERS])
    rc = nv.nvrtcCreateProgram(ctypes.byref(prog), src.encode(), b"oqmc_rtc.cu", len(hs),
                               arr_s, arr_n)
    if rc:
        return False, f"nvrtcCreateProgram {rc}", b""
    for n in names:
        nv.nvrtcAddNameExpression(prog, n.encode())
    opts = [b"--gpu-architecture=sm_100a", b"--std=c++17", b"-lineinfo",
            b"--device-as-default-execution-space"]
    rc = nv.nvrtcCompileProgram(prog, len(opts), (ctypes.c_char_p * len(opts))(*opts))
    n = ctypes.c_size_t()
    nv.nvrtcGetProgramLogSize(prog, ctypes.byref(n))
    log = ctypes.create_string_buffer(n.value + 1)
    nv.nvrtcGetProgramLog(prog, log)
    cubin = b""
    if rc == 0:
        nv.nvrtcGetCUBINSize(prog, ctypes.byref(n))
        cb = ctypes.create_string_buffer(n.value)
        nv.nvrtcGetCUBIN(prog, cb)
        cubin = cb.raw
    nv.nvrtcDestroyProgram(ctypes.byref(prog))
    return rc == 0, log.value.decode(errors="replace"), cubin


def compile_mlp_sweep(system):
    """NVRTC-compile the learned-proposal sweep kernel of ``system`` (the
    source oqmc_set_mlp_proposal builds); returns (ok, log, cubin bytes)."""
    src = spec_source(system).replace('#include "oqmc_sweep.cuh"', '#include "oqmc_mlp_sweep.cuh"')
    return compile_source(src, [f"k_moves_mlp<{system.nocc}, OqSpecBasis, {g}>" for g in (2, 4)])


def compile_spec(system):
    """NVRTC-compile the specialised kernels; returns (ok, log, cubin bytes)."""
    nocc = system.nocc
    names = []
    for t in ("double, double", "float, float"):
        names.append(f"k_eloc<{nocc}, {t}, OqSpecBasis>")
        for prop in (0, 1):
            names.append(f"k_moves<{nocc}, {t}, {prop}, OqSpecBasis>")
    return compile_source(spec_source(system), names)
