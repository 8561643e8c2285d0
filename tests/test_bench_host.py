"""The bench's clock record on the host: nvidia-smi's CSV lines (index,
clocks.sm, clocks.max.sm, power.draw, the active-reasons mask, then
hw_slowdown, hw_thermal_slowdown, sw_thermal_slowdown, sw_power_cap) are
reduced to the median SM clock, the maximum clock and the set of throttle
reasons seen active; malformed lines are skipped."""
import bench


class _Proc:
    def terminate(self):
        pass

    def wait(self, timeout=None):
        pass

    def kill(self):
        pass


class _Thread:
    def join(self, timeout=None):
        pass


def _stopped(lines):
    cs = bench.ClockSampler(0)
    cs.proc, cs.t, cs.lines = _Proc(), _Thread(), list(lines)
    return cs.stop()


def test_clock_record():
    rec = _stopped([
        "0, 1965, 1965, 910.2, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
        "0, 1800, 1965, 998.0, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
        "0, 1905, 1965, 950.0, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
        "garbage",
        "0, [N/A], 1965, 950.0, 0x0, Not Active, Not Active, Not Active, Not Active",
    ])
    assert rec == {"sm_mhz": 1905.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"], "samples": 3}


def test_clock_record_slowdowns_and_empty():
    rec = _stopped([
        "0, 1500, 1965, 700.0, 0x8, Active, Not Active, Not Active, Not Active",
        "0, 1400, 1965, 700.0, 0x60, Not Active, Active, Active, Not Active",
    ])
    assert rec["reasons"] == ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown"]
    assert rec["sm_mhz"] == 1450.0 and rec["samples"] == 2
    assert _stopped(["no samples"]) is None
    assert bench.ClockSampler(0).stop() is None  # never started
