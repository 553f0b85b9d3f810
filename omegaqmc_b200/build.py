"""Build liboqmc_b200.so in-tree for sm_100a.

The determinant-size instantiations (``csrc/oqmc_inst.cu`` with
``-DOQ_N=<nocc>``) compile as separate objects in parallel; the C-ABI host
code is ``csrc/oqmc.cu``.  Objects are cached in ``_build/`` keyed by a hash
of the sources and flags, so an unchanged tree relinks in seconds.

Usage: ``python -m omegaqmc_b200.build [--force] [-j N]``
"""
from __future__ import annotations

import argparse
import glob
import hashlib
import os
import shutil
import subprocess
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "liboqmc_b200.so")
NOCC_LIST = (1, 2, 3, 4, 5, 6, 7, 8, 10, 12, 14, 16)
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
         "--expt-relaxed-constexpr"]


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found; the CUDA toolkit is required to build")


def _src_hash(extra):
    h = hashlib.sha256()
    files = sorted(glob.glob(os.path.join(CSRC, "*")) +
                   [os.path.join(HERE, "..", "include", "oqmc_b200.h")])
    for f in files:
        with open(f, "rb") as fh:
            h.update(os.path.basename(f).encode())
            h.update(fh.read())
    h.update(" ".join(ARCH + FLAGS + extra).encode())
    return h.hexdigest()[:16]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return r


RTC_HEADERS = ("oqmc_common.cuh", "oqmc_ao.cuh", "oqmc_eval.cuh", "oqmc_sweep.cuh",
               "oqmc_batch.cuh", "oqmc_tc.cuh", "oqmc_mlp.cuh", "oqmc_mlp_sweep.cuh")


def _embed_headers():
    """Write _build/oqmc_rtc_src.inc: the kernel headers as string literals for
    the run-time (NVRTC) specialisation."""
    out = ["// generated by omegaqmc_b200/build.py from csrc/*.cuh", "#pragma once",
           f"static const int kOqRtcCount = {len(RTC_HEADERS)};",
           "static const char* const kOqRtcNames[] = {" +
           ", ".join(f'"{h}"' for h in RTC_HEADERS) + "};",
           "static const char* const kOqRtcSrcs[] = {"]
    for h in RTC_HEADERS:
        txt = open(os.path.join(CSRC, h)).read()
        assert ")OQRTC\"" not in txt
        out.append('R"OQRTC(' + txt + ')OQRTC",')
    out.append("};")
    path = os.path.join(BUILD, "oqmc_rtc_src.inc")
    new = "\n".join(out) + "\n"
    if not os.path.exists(path) or open(path).read() != new:
        with open(path, "w") as f:
            f.write(new)


def build(force=False, jobs=None, verbose=False):
    """Compile and link the library; returns its path."""
    nvcc = _nvcc()
    os.makedirs(BUILD, exist_ok=True)
    key = _src_hash([])
    stamp = os.path.join(BUILD, "stamp")
    if (not force and os.path.exists(LIB) and os.path.exists(stamp)
            and open(stamp).read().strip() == key):
        return LIB
    jobs = jobs or max(1, min(len(NOCC_LIST) + 1, os.cpu_count() or 4))
    _embed_headers()
    units = [(os.path.join(CSRC, "oqmc.cu"), os.path.join(BUILD, "oqmc.o"), []),
             (os.path.join(CSRC, "oqmc_peak.cu"), os.path.join(BUILD, "oqmc_peak.o"), []),
             (os.path.join(CSRC, "oqmc_noalloc.cu"), os.path.join(BUILD, "oqmc_noalloc.o"), []),
             (os.path.join(CSRC, "oqmc_rtc.cu"), os.path.join(BUILD, "oqmc_rtc.o"),
              ["-I" + BUILD]),
             (os.path.join(CSRC, "oqmc_batch.cu"), os.path.join(BUILD, "oqmc_batch.o"), []),
             (os.path.join(CSRC, "oqmc_mlp.cu"), os.path.join(BUILD, "oqmc_mlp.o"), [])]
    for n in NOCC_LIST:
        units.append((os.path.join(CSRC, "oqmc_inst.cu"),
                      os.path.join(BUILD, f"oqmc_inst_{n}.o"), [f"-DOQ_N={n}"]))

    def compile_one(u):
        src, obj, defs = u
        cmd = [nvcc] + ARCH + FLAGS + defs + ["-c", src, "-o", obj]
        if verbose:
            cmd.append("-Xptxas=-v")
        return _run(cmd)

    with ThreadPoolExecutor(jobs) as ex:
        results = list(ex.map(compile_one, units))
    if verbose:
        for r in results:
            print(r.stderr)
    tmp = LIB + ".tmp"
    _run([nvcc] + ARCH + ["-shared", "-o", tmp] + [u[1] for u in units] + ["-lcudart", "-ldl"])
    os.replace(tmp, LIB)
    with open(stamp, "w") as f:
        f.write(key)
    from . import rhf
    rhf._load()          # host integral library of the RHF front end
    return LIB


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=None)
    ap.add_argument("-v", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, jobs=a.j, verbose=a.v))


if __name__ == "__main__":
    main()
