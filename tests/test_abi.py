"""The C-ABI library loads and exports every symbol the header declares
(no compute calls: this runs without a GPU)."""
import ctypes
import os
import re

import numpy as np
import pytest

from omegaqmc_b200 import _lib as L
from omegaqmc_b200 import molecules as M
from omegaqmc_b200.context import pack_system
from omegaqmc_b200.system import build_system

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    out = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", fn)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            out |= set(re.findall(r"\b(oqmc_[a-z0-9_]+)\s*\(", txt))
    return out


def test_library_exports_every_declared_symbol():
    lib = L.load()
    syms = header_symbols()
    assert syms, "no declarations found"
    for s in sorted(syms):
        assert hasattr(lib, s), s
    assert syms <= set(L.EXPORTED) | {"oqmc_version"}, syms - set(L.EXPORTED)


def test_version_string():
    assert b"sm_100a" in L.load().oqmc_version()


def test_descriptor_layout_matches_system():
    for name in M.NAMED_SYSTEMS:
        mf = M.make_mf(name)
        s = build_system(mf, M.default_params_corr(mf.mol))
        d, arr = pack_system(s)
        assert d.nbf == s.nbf and d.nocc == s.nocc and d.n_e == s.n_e
        nao = sum((2 * am + 1) * nc for am, nc in zip(arr["group_am"], arr["group_ncol"]))
        assert nao == s.nbf
        assert len(arr["norm"]) == int(np.sum(arr["group_nprim"] * arr["group_ncol"]))
        assert len(arr["alpha"]) == s.n_exp()


def test_error_path_without_device_work():
    # an invalid descriptor is rejected on the host before any CUDA call
    lib = L.load()
    h = ctypes.c_void_p()
    d = L.SystemDesc()
    d.natm = 0
    code = lib.oqmc_create(ctypes.byref(h), ctypes.byref(d))
    assert code == L.OQ_ERR_UNSUPPORTED
    assert b"natm" in lib.oqmc_last_error(None)
    with pytest.raises(NotImplementedError):
        L.check(code, None)
