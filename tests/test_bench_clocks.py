"""bench.py's in-process clock sampler (NvmlClockSampler) against a fake NVML:
the summary a bench line carries decides whether a timing is kept (throttle
reasons hw_slowdown / hw_thermal_slowdown / sw_thermal_slowdown reject it,
sw_power_cap is noted), so its reading of the reason bits, the loaded-sample
median and the sample count are checked here without a GPU."""
import itertools
import os
import sys
import time
import types

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def fake_nvml(samples):
    """samples: list of (sm_mhz, power_w, reason_bits), cycled."""
    it = itertools.cycle(samples)
    cur = {"s": next(it)}
    nv = types.SimpleNamespace()
    nv.NVML_CLOCK_SM = 1
    nv.nvmlClocksThrottleReasonSwPowerCap = 0x4
    nv.nvmlClocksThrottleReasonHwSlowdown = 0x8
    nv.nvmlClocksThrottleReasonSwThermalSlowdown = 0x20
    nv.nvmlClocksThrottleReasonHwThermalSlowdown = 0x40
    nv.calls = {"init": 0, "shutdown": 0}

    def init():
        nv.calls["init"] += 1

    def shutdown():
        nv.calls["shutdown"] += 1

    def clock(h, which):
        cur["s"] = next(it)  # each sample starts with the SM clock query
        return cur["s"][0]

    def by_pci(bus):
        raise RuntimeError("no PCI lookup in the fake")

    nv.nvmlInit = init
    nv.nvmlShutdown = shutdown
    nv.nvmlDeviceGetHandleByIndex = lambda i: ("gpu", i)
    nv.nvmlDeviceGetHandleByPciBusId = by_pci
    nv.nvmlDeviceGetClockInfo = clock
    nv.nvmlDeviceGetMaxClockInfo = lambda h, which: 1965
    nv.nvmlDeviceGetPowerUsage = lambda h: int(cur["s"][1] * 1000)
    nv.nvmlDeviceGetCurrentClocksEventReasons = lambda h: cur["s"][2]
    return nv


def sample(samples, seconds=0.2):
    s = bench.NvmlClockSampler(0)
    s.nv = fake_nvml(samples)
    with s:
        time.sleep(seconds)
    return s, s.summary()


def test_power_cap_is_reported_and_idle_samples_left_out():
    s, out = sample([(1965, 900.0, 0x4), (1800, 950.0, 0x4), (210, 80.0, 0x0)])
    assert out["source"] == "nvml"
    assert out["reasons"] == ["sw_power_cap"]
    assert out["sm_max_mhz"] == 1965
    assert out["samples"] == len(s.rows) >= 3  # one before, at least one during, one after
    # the median is over samples drawing more than 200 W only
    assert out["sm_mhz"] in (1800, 1965, (1800 + 1965) / 2)
    assert s.nv.calls == {"init": 1, "shutdown": 1}


def test_rejecting_reasons_are_named():
    _, out = sample([(1500, 700.0, 0x8 | 0x40), (1500, 700.0, 0x20)])
    assert out["reasons"] == ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown"]
    assert out["sm_mhz"] == 1500


def test_clean_run_has_no_reasons():
    _, out = sample([(1965, 600.0, 0x0)])
    assert out["reasons"] == [] and out["sm_mhz"] == 1965
