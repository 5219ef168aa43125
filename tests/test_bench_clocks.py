"""bench.py's clock record: nvidia-smi samples are kept only from inside the
timed region (the first sample after its start when the region is shorter
than the 200 ms sampling period), with the throttle reasons active there."""
from __future__ import annotations

import bench


def _line(sm, smax=1965, reasons=()):
    act = ["Active" if nm in reasons else "Not Active" for nm in bench.CLOCK_REASONS]
    return f"0, {sm}, {smax}, 700.0, 0x0, " + ", ".join(act)


def test_samples_inside_the_region_only():
    lines = [(0.0, _line(345)), (0.2, _line(1965)), (0.4, _line(1950, reasons=("sw_power_cap",))),
             (0.6, _line(1965)), (0.8, _line(400, reasons=("hw_slowdown",)))]
    c = bench.summarize_clocks(lines, 0.1, 0.7)
    assert c["samples"] == 3 and c["samples_total"] == 5
    assert c["sm_mhz"] == 1965 and c["sm_max_mhz"] == 1965
    assert c["reasons"] == ["sw_power_cap"]
    assert c["timed_region_s"] == 0.6


def test_short_region_takes_the_next_sample():
    lines = [(0.0, _line(345)), (0.2, _line(1965, reasons=("hw_thermal_slowdown",))), (0.4, _line(500))]
    c = bench.summarize_clocks(lines, 0.05, 0.15)
    assert c["samples"] == 1 and c["sm_mhz"] == 1965
    assert c["reasons"] == ["hw_thermal_slowdown"]


def test_no_region_keeps_every_sample_and_skips_bad_lines():
    lines = [(0.0, "garbage"), (0.1, _line(1900)), (0.2, "0, [N/A], 1965, 1, 2, 3, 4, 5, 6"),
             (0.3, _line(1960))]
    c = bench.summarize_clocks(lines)
    assert c["samples"] == 2 and c["sm_mhz"] == 1930.0 and c["reasons"] == []
    assert bench.summarize_clocks([])["reasons"] == ["no samples"]
