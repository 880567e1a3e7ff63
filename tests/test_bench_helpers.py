"""Host helpers of bench.py: the nvidia-smi clock sampler's parser and the
roofline peak source (no GPU)."""
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


class _DoneProc:
    def terminate(self):
        pass

    def wait(self, timeout=None):
        return 0

    def kill(self):
        pass


def _sampler_with(tmp_path, lines):
    path = tmp_path / "clocks.csv"
    path.write_text("".join(line + "\n" for line in lines))
    s = bench.ClockSampler(0)
    s.proc = _DoneProc()
    s.path = str(path)
    return s


def test_clock_parser_median_max_and_reasons(tmp_path):
    # index, clocks.sm, clocks.max.sm, power.draw, active mask, hw_slowdown,
    # hw_thermal_slowdown, sw_thermal_slowdown, sw_power_cap
    s = _sampler_with(tmp_path, [
        "0, 1965, 1965, 700.1, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
        "0, 1950, 1965, 980.5, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
        "0, 1965, 1965, 950.0, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
        "garbage line",
        "0, [N/A], 1965, 1.0, 0x0, Not Active, Not Active, Not Active, Not Active",
    ])
    out = s.stop()
    assert out == {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"], "samples": 3}
    assert not os.path.exists(s.path)


def test_clock_parser_reports_throttle_reasons(tmp_path):
    s = _sampler_with(tmp_path, [
        "0, 1200, 1965, 500.0, 0x8, Active, Not Active, Active, Not Active",
    ])
    out = s.stop()
    assert out["reasons"] == ["hw_slowdown", "sw_thermal_slowdown"]
    assert out["sm_mhz"] == 1200.0


def test_clock_parser_without_samples_is_none(tmp_path):
    assert _sampler_with(tmp_path, []).stop() is None
    assert bench.ClockSampler(0).stop() is None  # never started


def test_peaks_source():
    peak, kind = bench._peaks()
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            assert peak == float(json.load(f)["hbm_gbs"]) and kind == "measured"
    else:
        assert (peak, kind) == (6650.0, "fallback")
