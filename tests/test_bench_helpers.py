"""Pure helpers of bench.py (CPU): the filter-stage rates and the workload
override, so that a change to them cannot break the benchmark line."""
import argparse
import os
import sys

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_filter_stage():
    cnt = [0, 0, 2_000_000_000, 1_000_000_000, 0, 0, 0, 0]
    f = bench.filter_stage(cnt, 2000.0, 0.5, 30.0)  # phase A: 1 s
    assert abs(f["seconds"] - 1.0) < 1e-12
    assert abs(f["candidates_per_s"] - 2e9) < 1e-3 and abs(f["window_tests_per_s"] - 1e9) < 1e-3
    assert abs(f["fp64_tflops"] - (27 * 2e9 + 3 * 1e9) / 1e12) < 1e-12
    assert abs(f["frac_of_fp64_peak"] - f["fp64_tflops"] / 30.0) < 1e-15
    assert bench.filter_stage(cnt, 2000.0, None, 30.0) is None
    assert bench.filter_stage(cnt, 0.0, 0.5, 30.0) is None
    assert bench.filter_stage(cnt, 2000.0, 0.5, None)["frac_of_fp64_peak"] is None


def test_config_override():
    a = argparse.Namespace(config=1, grid=8)
    c = bench.config_of(a)
    assert c["grid"] == 8 and "overridden" in c["workload"]
    assert bench.CONFIGS[1]["grid"] == 16  # the table itself is left as it was
    assert bench.config_of(argparse.Namespace(config=3, grid=None))["grid"] == 24
