"""Build the oracle's C restatement (test infrastructure) in place.

Produces ``oracle/liboracle_vmc.so`` from ``oracle/vmc_ref.c`` when that
source exists; the tests and the CPU baseline leg of the benchmark load it.
"""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "vmc_ref.c")
LIB = os.path.join(HERE, "liboracle_vmc.so")


def build(force=False):
    if not os.path.exists(SRC):
        return None
    if (not force and os.path.exists(LIB)
            and os.path.getmtime(LIB) >= os.path.getmtime(SRC)):
        return LIB
    cmd = ["gcc", "-O3", "-march=x86-64-v3", "-fopenmp", "-fPIC", "-shared",
           "-o", LIB + ".tmp", SRC, "-lm"]
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force=True))
