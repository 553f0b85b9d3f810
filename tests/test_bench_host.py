"""Host-side logic of bench.py that decides whether a bench line is valid:
the clock summary keeps only the nvidia-smi rows taken inside the timed
region and reports every throttle reason seen there (no GPU needed)."""
import os
import sys

import pytest

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


def _row(mhz, active="Not Active", hw="Not Active", cap="Not Active"):
    # index, clocks.sm, clocks.max.sm, power, reasons.active, hw_slowdown,
    # hw_thermal_slowdown, sw_thermal_slowdown, sw_power_cap
    return ["0", str(mhz), "1965", "800.0", active, hw, "Not Active", "Not Active", cap]


def test_clock_summary_keeps_rows_of_the_timed_region():
    c = bench.ClockSampler(0)
    c.rows = [_row(345), _row(1965), _row(1965), _row(1950, cap="Active")]
    c.first = 1          # the row read before the timed region started
    s = c.summary()
    assert s["samples"] == 3
    assert s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"]


def test_clock_summary_flags_slowdowns_and_empty_records():
    c = bench.ClockSampler(0)
    c.rows = [_row(1965), _row(1500, hw="Active")]
    c.first = 0
    assert c.summary()["reasons"] == ["hw_slowdown"]
    c.first = 2          # nothing after the first row: all rows are used
    assert c.summary()["samples"] == 2
    empty = bench.ClockSampler(0)
    assert empty.summary()["reasons"] == ["unsampled"]


class _Ens:
    def __init__(self, since=0, every=50):
        self.since_refresh = since
        self.refresh_every = every


def test_sweep_launch_count_follows_the_ensemble_chunking():
    # 100 sweeps from a fresh refresh phase: two 50-sweep calls, each with two
    # layout conversions and 50 move + 50 local-energy kernels, then a refresh
    # (conversion + refresh kernel) after each
    assert bench.sweep_launches(_Ens(0), 100) == 2 * (2 + 100 + 2)
    # 30 sweeps left in the phase: a 30-sweep call, refresh, then 20 more
    assert bench.sweep_launches(_Ens(20), 50) == (2 + 60 + 2) + (2 + 40)
    # measurements every 4 sweeps: a 48-sweep call (12 measurements), then 2
    # sweeps with no measurement still take a move kernel, then the refresh
    assert bench.sweep_launches(_Ens(0), 50, measure_every=4) == (2 + 24) + (2 + 0 + 1) + 2


def test_kappa_spread_of_segments():
    """tau_int's stated uncertainty: kappa of each consecutive segment, their
    mean and standard error."""
    import numpy as np
    rng = np.random.default_rng(3)
    x = np.zeros(40000)
    for i in range(1, x.size):
        x[i] = 0.6 * x[i - 1] + rng.standard_normal()
    k = bench.kappa_spread(x, 4)
    assert k["segments"] == 4 and k["segment_sweeps"] == 10000 and len(k["kappas"]) == 4
    # AR(1) with phi = 0.6: tau_int = (1 + phi) / (1 - phi) = 4
    assert abs(k["mean"] - 4.0) < 0.5 and 0 < k["serr"] < 0.5
    assert bench.binning_analysis(x)[3] == pytest.approx(k["mean"], rel=0.2)


def test_headline_config_constants():
    # the timed region is long enough for the clock record and fits the sums buffer
    assert bench.MIN_TIMED_S >= 2.0
    assert bench.MAX_TIMED_SWEEPS % bench.REFRESH_EVERY == 0
    assert bench.PLAIN_SEGS * bench.PLAIN_SEG >= 50000
    assert set(bench.CONFIGS) == {"h2", "lih"}
