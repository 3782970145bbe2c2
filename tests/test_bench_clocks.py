"""bench.py's clock sampler on CPU, against a fake NVML module: the samples
taken while the timed region runs give the median SM clock, the maximum, the
throttle reasons seen and the peak power; without NVML or nvidia-smi the
summary says "unsampled" instead of failing."""
import os
import sys
import time
import types

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def fake_nvml(clocks, reasons, calls):
    nv = types.ModuleType("pynvml")
    nv.NVML_CLOCK_SM = 1
    nv.nvmlClocksEventReasonSwPowerCap = 0x4
    nv.nvmlClocksEventReasonHwSlowdown = 0x8
    nv.nvmlClocksEventReasonSwThermalSlowdown = 0x20
    nv.nvmlClocksEventReasonHwThermalSlowdown = 0x40
    state = {"i": 0}

    def clock(h, kind):
        calls.append(("clock", h))
        v = clocks[min(state["i"], len(clocks) - 1)]
        return v

    def why(h):
        v = reasons[min(state["i"], len(reasons) - 1)]
        state["i"] += 1
        return v

    nv.nvmlInit = lambda: calls.append("init")
    nv.nvmlShutdown = lambda: calls.append("shutdown")
    nv.nvmlDeviceGetHandleByIndex = lambda i: ("idx", i)
    nv.nvmlDeviceGetHandleByUUID = lambda u: ("uuid", u)
    nv.nvmlDeviceGetMaxClockInfo = lambda h, k: 1965
    nv.nvmlDeviceGetClockInfo = clock
    nv.nvmlDeviceGetPowerUsage = lambda h: 800500
    nv.nvmlDeviceGetCurrentClocksEventReasons = why
    return nv


@pytest.mark.parametrize("gpu,handle", [("3", ("idx", 3)), ("GPU-1234-abcd", ("uuid", "GPU-1234-abcd"))])
def test_nvml_sampler_summary(monkeypatch, gpu, handle):
    calls = []
    nv = fake_nvml([1965, 1965, 1950, 1965, 1965], [0, 0x4, 0, 0, 0], calls)
    monkeypatch.setitem(sys.modules, "pynvml", nv)
    with bench.ClockSampler(gpu, period_s=0.002) as clk:
        time.sleep(0.1)
    s = clk.summary()
    assert s["sampler"].startswith("nvml")
    assert s["samples"] >= 5
    assert s["sm_mhz"] == 1965 and s["sm_max_mhz"] == 1965
    assert s["reasons"] == ["sw_power_cap"]
    assert s["power_w_max"] == pytest.approx(800.5)
    assert ("clock", handle) in calls and calls[0] == "init" and calls[-1] == "shutdown"


def test_throttle_reasons_are_reported():
    rows_bits = 0x8 | 0x40
    calls = []
    nv = fake_nvml([1200], [rows_bits], calls)
    sys.modules["pynvml"] = nv
    try:
        with bench.ClockSampler("0", period_s=0.002) as clk:
            time.sleep(0.03)
        s = clk.summary()
    finally:
        del sys.modules["pynvml"]
    assert s["reasons"] == ["hw_slowdown", "hw_thermal_slowdown"] and s["sm_mhz"] == 1200


def test_without_nvml_or_nvidia_smi_the_summary_says_unsampled(monkeypatch):
    broken = types.ModuleType("pynvml")

    def fail():
        raise RuntimeError("no driver")

    broken.nvmlInit = fail
    monkeypatch.setitem(sys.modules, "pynvml", broken)
    monkeypatch.setenv("PATH", "/nonexistent")
    with bench.ClockSampler("0") as clk:
        pass
    assert clk.summary()["reasons"] == ["unsampled"]
