"""The bench's clock sampler against a fake NVML (no GPU): reason bits decode
to the contract's names, summary() keeps the samples of the timed window,
only read queries are made, and a missing NVML falls back without hanging."""
import sys
import time
import types

import bench


class FakeNvml(types.ModuleType):
    """Getters only, so any call that would change a GPU setting fails."""

    NVML_CLOCK_SM = 1
    nvmlClocksEventReasonSwPowerCap = 0x4
    nvmlClocksEventReasonHwSlowdown = 0x8
    nvmlClocksEventReasonSwThermalSlowdown = 0x20
    nvmlClocksEventReasonHwThermalSlowdown = 0x40

    def __init__(self, reasons=0x4, clocks=(1965, 1950, 1940), fail_init=False):
        super().__init__("pynvml")
        self.reasons, self.clocks, self.fail_init = reasons, list(clocks), fail_init
        self.calls = []
        self.i = 0

    def nvmlInit(self):
        self.calls.append("nvmlInit")
        if self.fail_init:
            raise RuntimeError("NVML Shared Library Not Found")

    def nvmlDeviceGetHandleByPciBusId(self, bus):
        self.calls.append(("byPci", bus))
        return "h"

    def nvmlDeviceGetHandleByIndex(self, i):
        self.calls.append(("byIndex", i))
        return "h"

    def nvmlDeviceGetMaxClockInfo(self, h, kind):
        self.calls.append("max")
        return 1965

    def nvmlDeviceGetClockInfo(self, h, kind):
        v = self.clocks[min(self.i, len(self.clocks) - 1)]
        self.i += 1
        return v

    def nvmlDeviceGetCurrentClocksEventReasons(self, h):
        return self.reasons


def _sample(monkeypatch, fake, secs=0.08):
    monkeypatch.setitem(sys.modules, "pynvml", fake)
    clk = bench.ClockSampler(0, "00000000:1B:00.0", period_s=0.002).__enter__()
    t0 = clk.mark()
    time.sleep(secs)
    t1 = clk.mark()
    time.sleep(0.02)
    clk.__exit__()
    return clk, t0, t1


def test_nvml_samples_inside_window(monkeypatch):
    fake = FakeNvml(reasons=0x4)
    clk, t0, t1 = _sample(monkeypatch, fake)
    s = clk.summary(t0, t1)
    assert s["source"].startswith("nvml")
    assert s["samples"] >= 5, s
    assert s["reasons"] == ["sw_power_cap"]
    assert s["sm_max_mhz"] == 1965.0
    assert all(t0 <= r[0] <= t1 for r in clk.rows if r[0] >= t0 and r[0] <= t1)
    assert ("byPci", "00000000:1B:00.0") in fake.calls
    # only getters were called
    names = {c if isinstance(c, str) else c[0] for c in fake.calls}
    assert names <= {"nvmlInit", "byPci", "byIndex", "max"}


def test_reason_bits_decode(monkeypatch):
    fake = FakeNvml(reasons=0x4 | 0x8 | 0x20 | 0x40)
    clk, t0, t1 = _sample(monkeypatch, fake, 0.03)
    assert clk.summary(t0, t1)["reasons"] == ["hw_slowdown", "hw_thermal_slowdown", "sw_power_cap",
                                               "sw_thermal_slowdown"]
    fake = FakeNvml(reasons=0)
    clk, t0, t1 = _sample(monkeypatch, fake, 0.03)
    assert clk.summary(t0, t1)["reasons"] == []


def test_window_median_and_short_window():
    clk = bench.ClockSampler(0)
    clk.rows = [(1.0, 1965.0, 1965.0, set()), (2.0, 1500.0, 1965.0, {"sw_power_cap"}),
                (3.0, 1800.0, 1965.0, set()), (4.0, 1900.0, 1965.0, {"hw_slowdown"})]
    s = clk.summary(1.5, 3.5)
    assert s["samples"] == 2 and s["sm_mhz"] == 1650.0 and s["reasons"] == ["sw_power_cap"]
    # a window shorter than the period takes the first sample after its start
    s = clk.summary(2.1, 2.2)
    assert s["samples"] == 1 and s["sm_mhz"] == 1800.0


def test_missing_nvml_falls_back(monkeypatch):
    monkeypatch.setitem(sys.modules, "pynvml", FakeNvml(fail_init=True))
    monkeypatch.setenv("PATH", "/nonexistent")   # no nvidia-smi either
    t = time.monotonic()
    clk = bench.ClockSampler(0).__enter__()
    clk.__exit__()
    assert time.monotonic() - t < 2.0
    s = clk.summary()
    assert s["reasons"] == ["unsampled"] and s["samples"] == 0
