"""Host-side pieces of the benchmark's contract that need no GPU: the clock
record taken during the timed region (median SM clock, maximum, and which
throttle reasons were active in any sample)."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path[:0] = [ROOT]

import bench  # noqa: E402


def _clocks(text):
    c = bench.Clocks(0)
    c.out = text
    return c.summary()


def _row(sm, mx, hw="Not Active", hwt="Not Active", swt="Not Active", cap="Not Active"):
    return f"0, {sm}, {mx}, 700.00, 0x0000000000000000, {hw}, {hwt}, {swt}, {cap}"


def test_clock_summary_median_max_and_reasons():
    rows = [_row(1965, 1965), _row(1950, 1965), _row(1800, 1965, cap="Active"), _row(1965, 1965)]
    s = _clocks("\n".join(rows) + "\n")
    assert s["sm_mhz"] == 1957.5 and s["sm_max_mhz"] == 1965 and s["samples"] == 4
    assert s["reasons"] == ["sw_power_cap"]


def test_clock_summary_reports_rejecting_reasons():
    s = _clocks("\n".join([_row(1965, 1965), _row(1400, 1965, hwt="Active"), _row(1300, 1965, hw="Active")]))
    assert s["reasons"] == ["hw_slowdown", "hw_thermal_slowdown"]


def test_clock_summary_skips_unreadable_values_and_lines():
    s = _clocks("garbage\n" + _row("[N/A]", 1965) + "\n" + _row(1965, "[N/A]") + "\n")
    assert s["sm_mhz"] == 1965 and s["sm_max_mhz"] == 1965 and s["samples"] == 2


def test_clock_summary_without_samples():
    assert _clocks("")["reasons"] == ["unsampled"]
    assert _clocks(None)["sm_mhz"] is None
