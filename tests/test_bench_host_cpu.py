"""bench.py's host-side helpers on CPU: the clock samplers that run during the
timed region (they only read the GPU's clocks and clock-event reasons, never
set anything: checked against a fake NVML that fails on any other call), the
parsing of nvidia-smi's samples, the algorithmic byte and flop counts behind
the roofline, and the peak the roofline divides by."""
import json
import sys
import time
import types

import numpy as np
import pytest

import bench

READS = {"nvmlInit", "nvmlShutdown", "nvmlDeviceGetHandleByPciBusId", "nvmlDeviceGetHandleByIndex",
         "nvmlDeviceGetMaxClockInfo", "nvmlDeviceGetClockInfo", "nvmlDeviceGetCurrentClocksEventReasons"}


class FakeNvml(types.ModuleType):
    """pynvml with the read calls the sampler may make; any other NVML call
    (a setter, a reset, a lock) fails the test."""

    NVML_CLOCK_SM = 1

    def __init__(self, clocks=(1965, 1965, 1800), reasons=(0x0, 0x4, 0x4 | 0x8), init_error=False):
        super().__init__("pynvml")
        self.calls, self.clocks, self.reasons, self.init_error, self.i = [], clocks, reasons, init_error, 0

    def _call(self, name):
        assert name in READS, f"NVML call {name} is not a read"
        self.calls.append(name)

    def __getattr__(self, name):
        if name.startswith("nvml"):
            raise AssertionError(f"NVML call {name} is not a read")
        raise AttributeError(name)

    def nvmlInit(self):
        self._call("nvmlInit")
        if self.init_error:
            raise RuntimeError("NVML not found")

    def nvmlShutdown(self):
        self._call("nvmlShutdown")

    def nvmlDeviceGetHandleByPciBusId(self, bus):
        self._call("nvmlDeviceGetHandleByPciBusId")
        return "handle"

    def nvmlDeviceGetHandleByIndex(self, index):
        self._call("nvmlDeviceGetHandleByIndex")
        return "handle"

    def nvmlDeviceGetMaxClockInfo(self, h, kind):
        self._call("nvmlDeviceGetMaxClockInfo")
        return 1965

    def nvmlDeviceGetClockInfo(self, h, kind):
        self._call("nvmlDeviceGetClockInfo")
        return self.clocks[self.i % len(self.clocks)]

    def nvmlDeviceGetCurrentClocksEventReasons(self, h):
        self._call("nvmlDeviceGetCurrentClocksEventReasons")
        r = self.reasons[self.i % len(self.reasons)]
        self.i += 1
        return r


def test_nvml_sampler_reads_only_and_names_the_reasons(monkeypatch):
    fake = FakeNvml()
    monkeypatch.setitem(sys.modules, "pynvml", fake)
    with bench.NvmlClockSampler("cpu", 0) as c:
        t0 = time.time()
        while len(c.samples) < 6 and time.time() - t0 < 10:
            time.sleep(0.01)
    s = c.summary()
    assert s["samples"] >= 6 and s["sm_max_mhz"] == 1965.0
    assert s["sm_mhz"] in (1800.0, 1965.0)
    assert s["reasons"] == ["hw_slowdown", "sw_power_cap"]
    assert set(fake.calls) <= READS and "nvmlShutdown" in fake.calls


def test_nvml_reason_bits():
    """NVML's clock-event reason bits: SwPowerCap 0x4, HwSlowdown 0x8,
    SwThermalSlowdown 0x20, HwThermalSlowdown 0x40."""
    assert dict(bench.NvmlClockSampler.REASONS) == {"sw_power_cap": 0x4, "hw_slowdown": 0x8,
                                                    "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40}


def test_without_nvml_the_sampler_falls_back_to_nvidia_smi(monkeypatch):
    monkeypatch.setitem(sys.modules, "pynvml", FakeNvml(init_error=True))
    started = []

    def no_smi(cmd, **kw):
        started.append(cmd)
        raise FileNotFoundError("nvidia-smi")

    monkeypatch.setattr(bench.subprocess, "Popen", no_smi)
    with bench.NvmlClockSampler("cpu", 3) as c:
        pass
    assert started and started[0][0] == "nvidia-smi" and "--id=3" in started[0]
    assert not any(a.startswith(("-lgc", "-ac", "-pm", "-r", "--lock", "--reset")) for a in started[0])
    assert c.summary() == {"sm_mhz": None, "sm_max_mhz": None, "samples": 0, "reasons": []}


def test_nvidia_smi_lines():
    c = bench.ClockSampler(0)
    c.lines = ["0, 1965, 1965, 650.31, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
               "0, 1800, 1965, 999.02, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
               "0, [N/A], 1965, 700.0, 0x0, Not Active, Not Active, Not Active, Not Active",
               "garbage",
               "0, 1700, 1965, 990.0, 0x0000000000000024, Not Active, Not Active, Active, Active"]
    assert c.summary() == {"sm_mhz": 1800.0, "sm_max_mhz": 1965.0, "samples": 3,
                           "reasons": ["sw_power_cap", "sw_thermal_slowdown"]}


def test_algorithmic_bytes_and_flop():
    m, n = np.array([2, 3, 64]), np.array([2, 1, 32])
    nbytes, flop = bench.algorithmic(m, n)
    # per matrix 4 (mn + mk + k + kn) + 56: 56 + 56, 32 + 56, 4 (2048 + 2048 + 32 + 1024) + 56
    assert nbytes == 112 + 88 + 20664
    # nt (nt - 1) / 2 pairs x (12 mt + 6 nt) per sweep on the tall view
    assert flop.tolist() == [36, 0, 496 * (12 * 64 + 6 * 32)]
    _, flop_wide = bench.algorithmic(n, m)
    assert flop_wide.tolist() == flop.tolist()


def test_peaks(monkeypatch, tmp_path):
    (tmp_path / "MEASURED_PEAKS.json").write_text(json.dumps({"hbm_gbs": 6551.0, "bf16_tflops": 1500.0}))
    monkeypatch.setattr(bench, "ROOT", tmp_path)
    assert bench.peaks() == (6551.0, "measured")
    (tmp_path / "MEASURED_PEAKS.json").unlink()
    assert bench.peaks() == (6650.0, "fallback")


@pytest.mark.parametrize("scaling", ("weak", "strong"))
def test_workload_config(scaling):
    c = bench.workload_config(4, scaling)
    assert c["workload"] == bench.WORKLOAD and c["scaling_mode"] == scaling
    assert c["parallelism"].startswith("dp4") and "no collective" in c["parallelism"]
