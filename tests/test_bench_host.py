"""Host-side logic of bench.py that decides whether a bench line is valid:
the clock summary keeps only the nvidia-smi rows taken inside the timed
region and reports every throttle reason seen there (no GPU needed)."""
import os
import sys

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
