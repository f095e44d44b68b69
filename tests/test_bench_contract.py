"""Host-side pieces of the benchmark's contract that need no GPU: the clock
record taken during the timed region (median SM clock, maximum, and which
throttle reasons were active in any sample)."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path[:0] = [ROOT, os.path.join(ROOT, "sep-graph_b200")]

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


def test_algorithmic_bytes_and_roofline_arithmetic():
    # SSSP: offsets + (index + weight) per reached edge + distances; BFS: index only
    assert bench.sssp_bytes(10, 100) == 4 * 11 + 8 * 100 + 4 * 10
    assert bench.bfs_bytes(10, 100) == 4 * 11 + 4 * 100 + 4 * 10
    r = bench._roof(2e9, 1.0, 4000.0)  # 2 GB in 1 ms = 2000 GB/s
    assert abs(r["GBs"] - 2000.0) < 1e-9 and abs(r["frac_hbm"] - 0.5) < 1e-12
    assert abs(r["frac_hbm_nominal_8TBs"] - 0.25) < 1e-12


def test_reached_edges_counts_out_degrees_of_reached_vertices():
    import numpy as np
    import types

    h = types.SimpleNamespace(offsets=np.array([0, 2, 3, 3, 6], np.uint32))
    vals = np.array([0, 1, bench.INF, 2], np.uint32)
    assert bench.reached_edges(h, vals) == 2 + 1 + 3


def test_traffic_comes_from_the_committed_summaries():
    # the headline's delta-stepping launch has a committed full-size capture; plain push has none
    t = bench.read_traffic("delta8")
    assert t is not None and t > 1e8
    assert bench.read_traffic("push") is None
    peak, kind = bench.peak_hbm()
    assert peak > 0 and kind in ("measured", "fallback")


def test_cpu_baseline_record():
    import sepgraph as sg

    h = sg.HostGraph.rmat(10, 8, seed=1).gen_weights(1, 64, 2)
    srcs = [int(s) for s in h.pick_sources(3, 3)]
    b = bench.cpu_baseline(h, srcs, budget_s=5.0)
    assert b["value"] > 0 and b["cores"] == 1 and b["kind"] in ("reference", "port") and b["unit"] == bench.METRIC
