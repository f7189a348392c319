"""Host logic of bench.py's clock record on CPU: the nvidia-smi samples taken
during the timed region are reduced to the median SM clock, the maximum SM
clock and the throttle reasons seen active in any sample."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def _sampler(lines):
    s = bench.ClockSampler(0)
    s.lines = lines
    return s


def _line(sm, reasons=("Not Active",) * 4, max_sm=1965, power=900.0):
    return ", ".join(["0", str(sm), str(max_sm), str(power), "0x0000000000000000", *reasons])


def test_median_clock_and_no_reason():
    s = _sampler([_line(1965), _line(1950), _line(1965)])
    assert s.summary() == {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": [], "samples": 3}


def test_reasons_seen_in_any_sample_are_reported():
    power_cap = ("Not Active", "Not Active", "Not Active", "Active")
    thermal = ("Not Active", "Active", "Not Active", "Not Active")
    s = _sampler([_line(1305, power_cap), _line(1965), _line(1290, thermal)])
    out = s.summary()
    assert out["reasons"] == ["hw_thermal_slowdown", "sw_power_cap"]
    assert out["sm_mhz"] == 1305.0
    assert out["samples"] == 3


def test_malformed_and_missing_samples():
    assert _sampler([]).summary() is None
    assert _sampler(["garbage", "0, [N/A], 1965, 1.0, 0x0, a, b, c, d"]).summary() is None
    assert bench.ClockSampler(0).summary() is None  # never entered
    out = _sampler(["short, line", _line(1800)]).summary()
    assert out["samples"] == 1 and out["sm_mhz"] == 1800.0


def test_l2_note_states_whether_the_working_set_exceeds_l2():
    assert "more than the 126 MB L2" in bench.l2_note(1.506e9)
    assert "fits in the 126 MB L2" in bench.l2_note(1.0e6)
