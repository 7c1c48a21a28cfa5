"""bench.py host logic on the CPU: the clock-sample summary that decides
whether a measurement is kept (hw/thermal slowdowns reject it, a power cap is
noted) and its handling of missing fields."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import pytest  # noqa: E402
import bench  # noqa: E402


def row(sm, mx=1965, hw="Not Active", hwt="Not Active", swt="Not Active", cap="Not Active"):
    return f"0, {sm}, {mx}, 950.0, 0x0, {hw}, {hwt}, {swt}, {cap}\n"


def test_clock_summary_under_load():
    lines = [row(210)] + [row(1800)] * 5 + [row(1900, cap="Active")] * 4
    s = bench.ClockSampler.parse(lines)
    assert s["sm_max_mhz"] == 1965 and s["samples"] == 10
    assert s["sm_mhz"] == 1800.0                      # idle sample (210 MHz) left out of the median
    assert s["reasons"] == ["sw_power_cap"]


def test_clock_summary_reasons_and_missing_fields():
    lines = [row(1500, hwt="Active"), row("[N/A]", mx="[N/A]"), "garbage\n", row(1600, hw="Active")]
    s = bench.ClockSampler.parse(lines)
    assert s["reasons"] == ["hw_slowdown", "hw_thermal_slowdown"]
    assert s["sm_max_mhz"] == 1965 and s["sm_mhz"] == 1550.0
    assert bench.ClockSampler.parse([])["reasons"] == ["no samples"]
    only_na = bench.ClockSampler.parse([row("[N/A]", mx="[N/A]")])
    assert only_na["sm_mhz"] is None and only_na["sm_max_mhz"] is None


def test_class_rates():
    """Per-class achieved rates of the bench line: algorithmic flops and bytes
    over the class's event time, as fractions of the FP64 and HBM peaks;
    classes with no recorded time are left out."""
    prof = {"rcholqr": {"launches": 515, "seconds": 0.5, "flops": 2.0e12, "bytes": 5.0e11},
            "copy": {"launches": 784, "seconds": 0.1, "flops": 0.0, "bytes": 1.5e11},
            "cov": {"launches": 0, "seconds": 0.0, "flops": 0.0, "bytes": 0.0}}
    r = bench.class_rates(prof, 40.0, 6000.0)
    assert set(r) == {"rcholqr", "copy"}
    assert r["rcholqr"]["tflops"] == pytest.approx(4.0) and r["rcholqr"]["fp64_frac"] == pytest.approx(0.1)
    assert r["copy"]["gbs"] == pytest.approx(1500.0) and r["copy"]["hbm_frac"] == pytest.approx(0.25)
    assert r["copy"]["tflops"] == 0.0
