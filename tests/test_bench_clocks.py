"""The bench's clock sampler on a fake NVML (no GPU): samples are taken while
the timed region runs, and the throttle-reason bits map to the names the bench
line reports."""
import sys
import time
import types

import bench


def _fake_nvml(reasons: int):
    n = types.ModuleType("pynvml")
    n.NVML_CLOCK_SM = 1
    n.nvmlClocksEventReasonSwPowerCap = 0x4
    n.nvmlClocksEventReasonHwSlowdown = 0x8
    n.nvmlClocksEventReasonSwThermalSlowdown = 0x20
    n.nvmlClocksEventReasonHwThermalSlowdown = 0x40
    n.nvmlInit = lambda: None
    n.nvmlShutdown = lambda: None
    n.nvmlDeviceGetHandleByPciBusId_v2 = lambda bus: "handle"
    n.nvmlDeviceGetHandleByIndex = lambda idx: "handle"
    n.nvmlDeviceGetClockInfo = lambda h, kind: 1965
    n.nvmlDeviceGetMaxClockInfo = lambda h, kind: 1965
    n.nvmlDeviceGetPowerUsage = lambda h: 812_000
    n.nvmlDeviceGetCurrentClocksEventReasons = lambda h: reasons
    return n


def _sample(monkeypatch, reasons: int) -> dict:
    monkeypatch.setitem(sys.modules, "pynvml", _fake_nvml(reasons))
    with bench.ClockSampler(0) as clocks:
        time.sleep(0.1)
    return clocks.summary()


def test_nvml_samples_during_region(monkeypatch):
    s = _sample(monkeypatch, 0)
    assert s["source"] == "nvml"
    assert s["samples"] >= 3
    assert s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == []


def test_nvml_reason_names(monkeypatch):
    s = _sample(monkeypatch, 0x4 | 0x40)
    assert s["reasons"] == ["hw_thermal_slowdown", "sw_power_cap"]
