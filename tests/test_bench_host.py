"""Host-side pieces of bench.py that need no GPU: the clock-sample summary
(window selection, reasons, fallback without a sampler), the config both arms
print, and the host-memory bound of the CPU baseline."""
import importlib.util
import os

import pytest

from conftest import ROOT


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_clock_summary_takes_the_timed_window(bench):
    c = bench.ClockSampler(0)
    # samples at t = 0..9: idle-ish clocks before t = 5, loaded clocks with a power cap inside [5, 8]
    c.samples = [(float(t), 1000.0 if t < 5 else 1800.0, {"sw_power_cap"} if 5 <= t <= 8 else set())
                 for t in range(10)]
    c.smax = 1965.0
    c.nvml = ("stub", None, {})
    c.t = type("T", (), {"join": lambda self, timeout=None: None})()
    s = c.stop(window=(5.0, 8.0))
    assert s["sm_mhz"] == 1800.0 and s["samples"] == 4 and s["window"] == "timed region"
    assert s["reasons"] == ["sw_power_cap"] and s["sm_max_mhz"] == 1965.0


def test_clock_summary_falls_back_to_all_samples(bench):
    c = bench.ClockSampler(0)
    c.samples = [(0.0, 1900.0, set()), (1.0, 1950.0, {"hw_slowdown"}), (2.0, 1965.0, set())]
    c.smax = 1965.0
    c.nvml = ("stub", None, {})
    c.t = type("T", (), {"join": lambda self, timeout=None: None})()
    s = c.stop(window=(1.5, 1.6))  # fewer than three samples inside: all of them
    assert s["samples"] == 3 and s["sm_mhz"] == 1950.0 and s["sm_mhz_min"] == 1900.0
    assert s["reasons"] == ["hw_slowdown"] and s["window"].startswith("all samples")


def test_clock_summary_without_any_sampler(bench):
    c = bench.ClockSampler(0)
    s = c.stop()
    assert s["sm_mhz"] is None and s["reasons"] == ["clock sampling unavailable"]


def test_both_arms_print_the_same_config(bench):
    a, b = bench.bench_config(1), bench.bench_config(1)
    assert a == b and a["dims"] == [32, 32, 32, 64] and a["beta"] == 6.2
    assert bench.bench_config(4)["parallelism"] == "replicas x4"


def test_host_memory_bound_is_positive(bench):
    m = bench.host_memory_available()
    assert m is None or m > 0
