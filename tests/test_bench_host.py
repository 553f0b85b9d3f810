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
