"""bench.py's clock sampler against a fake NVML: samples are taken from a
thread during the timed region, the median SM clock and the active clock-event
reasons are reported, and nothing is written to the device."""
import time

import bench


class FakeNVML:
    NVML_CLOCK_SM = 1

    def __init__(self, clocks, reasons):
        self.clocks = list(clocks)
        self.reasons = list(reasons)
        self.i = 0
        self.calls = []

    def nvmlDeviceGetMaxClockInfo(self, h, kind):
        self.calls.append("max")
        return 1965

    def nvmlDeviceGetClockInfo(self, h, kind):
        self.calls.append("clock")
        v = self.clocks[min(self.i, len(self.clocks) - 1)]
        return v

    def nvmlDeviceGetCurrentClocksEventReasons(self, h):
        self.calls.append("reasons")
        v = self.reasons[min(self.i, len(self.reasons) - 1)]
        self.i += 1
        return v


def _sampler(monkeypatch, fake):
    s = bench.ClockSampler(0)
    monkeypatch.setattr(s, "_nvml_handle", lambda: (fake, object()))
    return s


def test_nvml_sampling_reports_median_and_reasons(monkeypatch):
    fake = FakeNVML([1965, 1950, 1965, 1965], [0, 0x4, 0, 0])  # sw_power_cap once
    s = _sampler(monkeypatch, fake)
    s.start()
    time.sleep(0.05)
    out = s.stop()
    assert out["source"].startswith("nvml")
    assert out["samples"] >= 3
    assert out["sm_max_mhz"] == 1965.0
    assert out["sm_mhz"] == 1965.0
    assert out["reasons"] == ["sw_power_cap"]
    assert set(fake.calls) <= {"max", "clock", "reasons"}  # reads only


def test_nvml_sampling_flags_thermal_slowdown(monkeypatch):
    fake = FakeNVML([1200], [0x40 | 0x8])
    s = _sampler(monkeypatch, fake)
    s.start()
    time.sleep(0.02)
    out = s.stop()
    assert out["reasons"] == ["hw_slowdown", "hw_thermal_slowdown"]
    assert out["sm_mhz"] == 1200.0


def test_unsampled_without_nvml_or_nvidia_smi(monkeypatch):
    s = bench.ClockSampler(0)

    def no_nvml():
        raise RuntimeError("no NVML")

    monkeypatch.setattr(s, "_nvml_handle", no_nvml)
    monkeypatch.setattr(bench.subprocess, "Popen", lambda *a, **k: (_ for _ in ()).throw(FileNotFoundError()))
    s.start()
    assert s.stop() == {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
