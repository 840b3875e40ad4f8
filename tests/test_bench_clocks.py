"""The bench's clock sampler (bench.Clocks) on the CPU: a fake NVML module
stands in for the driver library, and a fake nvidia-smi process for the
fallback.  The sampler only reads; these tests check what it reports (median
SM clock, the maximum, the clock-event reasons seen in any sample) and that it
falls back when an NVML read fails."""
from __future__ import annotations

import os
import sys
import time
import types

import pytest

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


def fake_nvml(clocks, reasons, fail_reasons=False):
    """A stand-in for pynvml: nvmlDeviceGetClockInfo walks `clocks`,
    nvmlDeviceGetCurrentClocksEventReasons `reasons` (the last value
    repeats)."""
    state = {"k": 0}
    m = types.ModuleType("pynvml")
    m.NVML_CLOCK_SM = 1
    m.nvmlInit = lambda: None
    m.nvmlDeviceGetHandleByPciBusId = lambda bus: "h"
    m.nvmlDeviceGetHandleByIndex = lambda i: "h"
    m.nvmlDeviceGetMaxClockInfo = lambda h, kind: 1965

    def clock(h, kind):
        v = clocks[min(state["k"], len(clocks) - 1)]
        return v

    def reason(h):
        if fail_reasons:
            raise RuntimeError("not supported")
        v = reasons[min(state["k"], len(reasons) - 1)]
        state["k"] += 1
        return v

    m.nvmlDeviceGetClockInfo = clock
    m.nvmlDeviceGetCurrentClocksEventReasons = reason
    return m


def test_nvml_samples_give_median_clock_and_reasons(monkeypatch):
    # power cap (0x4) in one sample, hw slowdown (0x8) in another
    m = fake_nvml([1965, 1965, 1800, 1965, 1965], [0, 0x4, 0, 0x8, 0])
    monkeypatch.setitem(sys.modules, "pynvml", m)
    c = bench.Clocks(0)
    assert c.thread is not None
    time.sleep(0.05)
    out = c.stop()
    assert out["source"] == "NVML, 5 ms"
    assert out["sm_max_mhz"] == 1965.0
    assert out["sm_mhz"] == 1965.0
    assert out["samples"] >= 3
    assert out["reasons"] == ["hw_slowdown", "sw_power_cap"]


def test_failing_nvml_read_falls_back_to_nvidia_smi(monkeypatch):
    monkeypatch.setitem(sys.modules, "pynvml", fake_nvml([1965], [0], fail_reasons=True))
    started = {}

    class FakeSmi:
        def __init__(self, cmd, **kw):
            started["cmd"] = cmd

        def terminate(self):
            pass

        def communicate(self, timeout=None):
            lines = ["0, 1965, 1965, 700.0, 0x0, Not Active, Not Active, Not Active, Not Active",
                     "0, 1950, 1965, 990.0, 0x4, Not Active, Not Active, Not Active, Active",
                     "0, 1965, 1965, 720.0, 0x0, Not Active, Not Active, Not Active, Not Active"]
            return "\n".join(lines) + "\n", ""

    monkeypatch.setattr(bench.subprocess, "Popen", FakeSmi)
    monkeypatch.setattr(bench.time, "sleep", lambda s: None)
    c = bench.Clocks(0)
    assert c.thread is None and "nvidia-smi" in started["cmd"][0]
    out = c.stop()
    assert out["source"] == "nvidia-smi, 200 ms"
    assert out["samples"] == 3 and out["sm_mhz"] == 1965.0 and out["sm_max_mhz"] == 1965.0
    assert out["reasons"] == ["sw_power_cap"]


def test_no_sampler_at_all_reports_none(monkeypatch):
    m = types.ModuleType("pynvml")

    def broken():
        raise OSError("no library")

    m.nvmlInit = broken
    monkeypatch.setitem(sys.modules, "pynvml", m)

    def no_smi(*a, **k):
        raise OSError("nvidia-smi not found")

    monkeypatch.setattr(bench.subprocess, "Popen", no_smi)
    assert bench.Clocks(0).stop() is None


if __name__ == "__main__":
    sys.exit(pytest.main([__file__, "-q"]))
