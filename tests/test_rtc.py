"""The run-time specialisation source compiles for sm_100a (NVRTC on the
host, no GPU) and carries the system's data."""
import pytest

from omegaqmc_b200 import molecules as M
from omegaqmc_b200 import rtc_check as R
from omegaqmc_b200.system import build_system


def test_spec_source_has_system_constants():
    mf = M.make_mf("H2")
    s = build_system(mf, M.benchmark_params_corr(mf.mol))
    src = R.spec_source(s)
    assert "struct OqSpecBasis" in src and "mo_vgl" in src
    assert "3.4252509" in src          # an H STO-3G exponent, compiled in


@pytest.mark.parametrize("name", ["H2O"])
def test_spec_compiles_for_sm100a(name):
    try:
        R._nvrtc()
    except OSError:
        pytest.skip("NVRTC not installed")
    mf = M.make_mf(name)
    s = build_system(mf, M.benchmark_params_corr(mf.mol))
    ok, log, cubin = R.compile_spec(s)
    assert ok, log
    assert len(cubin) > 10000
