"""bench.py's NVML clock sampler, on a fake NVML (no GPU): it reads the SM
clock, its maximum and the clock-event reasons from a thread, summarises
them as the bench line's `clocks` object, and falls back to the
nvidia-smi sampler when NVML cannot be used."""
import sys
import time
import types

import bench


class _Props:
    uuid = "0000-test"
    pci_domain_id, pci_bus_id, pci_device_id = 0, 0x1B, 0


def _fake_nvml(reasons):
    nv = types.ModuleType("pynvml")
    nv.NVML_CLOCK_SM = 1
    nv.nvmlClocksEventReasonHwSlowdown = 0x8
    nv.nvmlClocksEventReasonHwThermalSlowdown = 0x40
    nv.nvmlClocksEventReasonSwThermalSlowdown = 0x20
    nv.nvmlClocksEventReasonSwPowerCap = 0x4
    nv.nvmlInit = lambda: None
    nv.nvmlDeviceGetHandleByUUID = lambda u: ("h", u)
    calls = {"n": 0}

    def clock(h, kind):
        calls["n"] += 1
        return 1965 if calls["n"] % 7 else 300  # an idle reading now and then
    nv.nvmlDeviceGetClockInfo = clock
    nv.nvmlDeviceGetMaxClockInfo = lambda h, kind: 1965
    nv.nvmlDeviceGetCurrentClocksEventReasons = lambda h: reasons
    return nv


def test_nvml_sampler_summary(monkeypatch):
    import torch

    monkeypatch.setitem(sys.modules, "pynvml", _fake_nvml(0x4))
    monkeypatch.setattr(torch.cuda, "get_device_properties", lambda d: _Props())
    s = bench.clock_sampler(torch.device("cpu"))
    assert isinstance(s, bench.NvmlClockSampler)
    s.start()
    time.sleep(0.08)
    c = s.stop()
    assert c["samples"] >= 3 and c["sm_mhz"] == 1965.0 and c["sm_max_mhz"] == 1965.0
    assert c["reasons"] == ["sw_power_cap"]


def test_sampler_falls_back_without_nvml(monkeypatch):
    import torch

    broken = types.ModuleType("pynvml")

    def fail():
        raise RuntimeError("no driver")
    broken.nvmlInit = fail
    monkeypatch.setitem(sys.modules, "pynvml", broken)
    assert isinstance(bench.clock_sampler(torch.device("cpu")), bench.ClockSampler)
