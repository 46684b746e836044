"""bench.py's clock sampler on a fake NVML: samples taken while the timed
region runs, the median SM clock, and the clock-event reasons decoded from
the NVML bit mask (read-only queries; nothing is set)."""

from __future__ import annotations

import time
import types

import bench


def _fake_nvml(reasons: int):
    nv = types.SimpleNamespace()
    nv.NVML_CLOCK_SM = 1
    nv.nvmlClocksEventReasonHwSlowdown = 0x8
    nv.nvmlClocksEventReasonHwThermalSlowdown = 0x40
    nv.nvmlClocksEventReasonSwThermalSlowdown = 0x20
    nv.nvmlClocksEventReasonSwPowerCap = 0x4
    nv.nvmlDeviceGetMaxClockInfo = lambda h, kind: 1965
    clocks = iter([1965, 1950, 1965] * 10000)
    nv.nvmlDeviceGetClockInfo = lambda h, kind: next(clocks)
    nv.nvmlDeviceGetCurrentClocksEventReasons = lambda h: reasons
    return nv


def _run(monkeypatch, reasons: int) -> dict:
    nv = _fake_nvml(reasons)
    monkeypatch.setattr(bench.ClockSampler, "_nvml_handle", lambda self: (nv, object()))
    clk = bench.ClockSampler(0)
    clk.start()
    time.sleep(0.05)
    return clk.stop()


def test_samples_during_the_region(monkeypatch):
    out = _run(monkeypatch, 0)
    assert out["samples"] >= 5
    assert out["sm_mhz"] in (1950.0, 1965.0) and out["sm_max_mhz"] == 1965.0
    assert out["reasons"] == []


def test_reasons_decoded(monkeypatch):
    out = _run(monkeypatch, 0x4 | 0x40 | 0x1)
    assert out["reasons"] == ["hw_thermal_slowdown", "sw_power_cap"]
