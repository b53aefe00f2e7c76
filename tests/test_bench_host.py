"""Host-side arithmetic of bench.py, with no GPU: the roofline of each form
against the measured peaks, the headline count fixture, the serving target
check, and the parsing of the clock samples taken during the timed region."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import bench  # noqa: E402

PEAKS = {"hbm_gbs": 6540.0, "bf16_tflops": 1662.0, "bf16_tflops_sustained": 1383.7}


def test_roofline_per_form():
    pairs = 1e6 * (1e6 - 1) / 2
    flops = 2.0 * bench.DIM * pairs
    r = bench.roofline("fp16", 83.6, pairs, PEAKS, "measured")
    assert r["bound"] == "tensor" and r["kernel"] == "k_join_tc"
    assert r["algorithmic_flops_per_launch"] == flops
    assert r["achieved"] == pytest.approx(flops / 0.0836 / 1e12)
    assert r["peak"] == PEAKS["bf16_tflops_sustained"]
    assert r["frac"] == pytest.approx(r["achieved"] / r["peak"]) and 0.5 < r["frac"] < 0.6
    assert bench.roofline("tf32", 100.0, pairs, PEAKS, "measured")["peak"] == pytest.approx(1383.7 / 2)
    assert bench.roofline("bf16x3", 100.0, pairs, PEAKS, "measured")["peak"] == pytest.approx(1383.7 / 3)
    p = bench.roofline("plain", 5329.0, pairs, PEAKS, "measured")
    assert p["kernel"] == "k_join_fp64" and p["algorithmic_flops_per_launch"] == 3.0 * bench.DIM * pairs


def test_peaks_measured_or_fallback(tmp_path, monkeypatch):
    peaks, src = bench.load_peaks()
    if os.path.exists(os.path.join(ROOT, "MEASURED_PEAKS.json")):
        assert src == "measured" and peaks["bf16_tflops_sustained"] > 0
    monkeypatch.setattr(bench, "ROOT", str(tmp_path))
    peaks, src = bench.load_peaks()
    assert src == "fallback" and peaks["hbm_gbs"] == 6650.0 and peaks["bf16_tflops"] == 1590.0


def test_headline_count_fixture():
    assert bench.golden_count(bench.N_POINTS) == 16_377_640
    assert bench.golden_count(600_000) is None


def _serving(ratio, p99_server, p99_plain):
    leg = {"requests": 100, "requests_per_s": 10.0, "p50_ms": 1.0, "p99_ms": 2.0, "ok": True}
    return {"workload": "w", "form": "auto", "throughput_ratio_vs_plain": ratio, "saturated": dict(leg),
            "open_loop_same_rate": dict(leg, p99_ms=p99_server, offered_rate=5.0),
            "baseline_open_loop": dict(leg, p99_ms=p99_plain, offered_rate=5.0)}


def test_serving_target_check():
    assert bench.serving_summary(None) is None
    s = bench.serving_summary(_serving(10.4, 120.0, 1700.0))
    assert s["target_3x_at_le_p99"] is True
    assert s["p99_at_plain_rate_ms"] == {"server": 120.0, "plain_one_at_a_time": 1700.0}
    assert bench.serving_summary(_serving(2.9, 120.0, 1700.0))["target_3x_at_le_p99"] is False
    assert bench.serving_summary(_serving(10.4, 1800.0, 1700.0))["target_3x_at_le_p99"] is False


def test_clock_samples_parsed():
    cs = bench.ClockSampler(0)
    rows = [
        "0, 1965, 1965, 300.1, 0x0, Not Active, Not Active, Not Active, Not Active",  # before the timed region
        "0, 1860, 1965, 990.0, 0x4, Not Active, Not Active, Not Active, Active",
        "0, 1845, 1965, 995.0, 0x4, Not Active, Not Active, Not Active, Active",
        "0, 1875, 1965, 985.0, 0x0, Not Active, Not Active, Not Active, Not Active",
    ]
    cs.out.write(rows[0] + "\n")
    cs.mark()
    cs.out.write("\n".join(rows[1:]) + "\n")
    s = cs.summary()
    assert s == {"sm_mhz": 1860.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"], "samples": 3}
    assert not os.path.exists(cs.out.name)


def test_clock_samples_flag_thermal_slowdown():
    cs = bench.ClockSampler(0)
    cs.mark()
    cs.out.write("0, 1400, 1965, 700.0, 0x40, Not Active, Active, Not Active, Not Active\n")
    assert cs.summary()["reasons"] == ["hw_thermal_slowdown"]
    empty = bench.ClockSampler(0)
    assert empty.summary() == {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
