"""Host-side pieces of bench.py, on the CPU: the clock record that decides
whether a timed run is kept (throttle reasons seen Active during the timed
region), and the measured-peak lookup."""
import importlib.util
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
_spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
bench = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(bench)


def test_clock_summary_reads_clocks_and_reasons():
    lines = [
        "0, 1965, 1965, 812.3, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active\n",
        "0, 1950, 1965, 990.1, 0x0000000000000004, Not Active, Not Active, Not Active, Active\n",
        "0, 1965, 1965, 640.0, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active\n",
        "garbage line\n",
        "0, [N/A], 1965, 1.0, 0x0, Not Active, Not Active, Not Active, Not Active\n",
    ]
    out = bench.Clocks.summary(lines)
    assert out["samples"] == 3 and out["sm_mhz"] == 1965.0 and out["sm_max_mhz"] == 1965.0
    assert out["reasons"] == ["sw_power_cap"]
    hot = bench.Clocks.summary(["0, 1500, 1965, 900, 0x8, Active, Not Active, Active, Not Active\n"])
    assert hot["reasons"] == ["hw_slowdown", "sw_thermal_slowdown"]
    assert bench.Clocks.summary([])["sm_mhz"] is None


def test_measured_peak_lookup_names_its_source():
    gbs, kind = bench.measured_peaks()
    assert kind in ("measured", "fallback") and gbs > 1000.0
