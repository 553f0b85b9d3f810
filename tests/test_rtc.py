"""The run-time specialisation source compiles for sm_100a (NVRTC on the
host, no GPU) and carries the system's data."""
import pytest

from omegaqmc_b200 import molecules as M
import rtc_check as R
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


def test_batch_source_dispatches_every_system():
    systems = [build_system(M.make_mf(n), M.benchmark_params_corr(M.make_mf(n).mol))
               for n in ("H2", "LiH")]
    src = R.batch_source(systems)
    assert "struct OqSpecBasis_0" in src and "struct OqSpecBasis_1" in src
    assert "oq_batch_tile<1, T, Real, OqSpecBasis_0, 0>(a, d, oq_jas_0" in src
    assert "oq_batch_tile<2, T, Real, OqSpecBasis_1, 0>(a, d, oq_jas_1" in src
    assert "__constant__ OqJas oq_jas_1 = {2, " in src


def test_batch_kernel_compiles_for_sm100a():
    try:
        R._nvrtc()
    except OSError:
        pytest.skip("NVRTC not installed")
    systems = [build_system(M.make_mf(n), M.benchmark_params_corr(M.make_mf(n).mol))
               for n in ("H2", "LiH")]
    ok, log, cubin = R.compile_source(R.batch_source(systems), R.BATCH_KERNELS[:1])
    assert ok, log
    assert len(cubin) > 10000


def test_tuned_batch_module_compiles_for_sm100a():
    """The module compiled after tuning fixes each molecule's move code (one
    lane per walker: mode 1, several: mode 2); it must compile too."""
    try:
        R._nvrtc()
    except OSError:
        pytest.skip("NVRTC not installed")
    systems = [build_system(M.make_mf(n), M.benchmark_params_corr(M.make_mf(n).mol))
               for n in ("H2", "LiH")]
    src = R.batch_source(systems)
    fixed = (src.replace("OqSpecBasis_0, 0>(a, d,", "OqSpecBasis_0, 1>(a, d,")
                .replace("OqSpecBasis_1, 0>(a, d,", "OqSpecBasis_1, 2>(a, d,"))
    assert fixed != src
    ok, log, cubin = R.compile_source(fixed, R.BATCH_KERNELS[:1])
    assert ok, log
    ok0, _, cubin0 = R.compile_source(src, R.BATCH_KERNELS[:1])
    assert ok0 and len(cubin) < len(cubin0)


@pytest.mark.parametrize("name", ["H2O", "LiH", "N2"])
def test_generated_code_leaves_out_round_off_coefficients(name):
    """H2O (C2v) orbitals have exact zeros on the AOs of other irreducible
    representations, which the eigensolver returns at ~1e-15: the generated
    MO-value code evaluates only the coefficients above 1e-12 of their
    orbital's largest one, and the benchmark's flop model counts the same."""
    import re
    import numpy as np
    import bench
    mf = M.make_mf(name)
    s = build_system(mf, M.benchmark_params_corr(mf.mol))
    src = R.spec_source(s)
    mo_val = src.split("mo_vgl(")[0]
    kept = re.findall(r"mv\[\d+\] \+= \(T\)\(([-0-9.eE+]+)\)", mo_val)
    C = np.abs(np.asarray(s.C))
    assert len(kept) == bench.mo_terms(s) < C.size
    assert min(abs(float(c)) for c in kept) > 1e-6
    # the dropped ones are round-off: below 1e-12 of their orbital's scale
    small = C[(C > 0) & (C <= 1e-12 * C.max(axis=0, keepdims=True))]
    assert small.size == C.size - len(kept) - np.count_nonzero(C == 0)


def test_spec_compiles_with_f_and_g_shells():
    """The generated orbital code of a basis with f and g shells (the
    reference-made golden case) compiles for sm_100a, contracted form
    included."""
    try:
        R._nvrtc()
    except OSError:
        pytest.skip("NVRTC not installed")
    from helpers import golden_system
    s, _ = golden_system("fg_shells")
    src = R.spec_source(s)
    assert "oq_harm_table" in src
    ok, log, cubin = R.compile_spec(s)
    assert ok, log
