"""Host logic of bench.py on CPU: the clock record of the timed region (median SM
clock, highest max clock, the union of the throttle reasons seen) from NVML-style
samples and from parsed nvidia-smi lines."""
import subprocess

import bench


def test_clock_record_from_samples():
    c = bench.ClockSampler(0)
    c._nvml = None
    c.rows = [(1900.0, 1965.0, {"sw_power_cap"}), (1800.0, 1965.0, set()), (1850.0, 1965.0, set())]
    rec = c.stop()
    assert rec["sm_mhz"] == 1850.0 and rec["sm_max_mhz"] == 1965.0
    assert rec["reasons"] == ["sw_power_cap"] and rec["samples"] == 3


def test_clock_record_without_samples():
    c = bench.ClockSampler(0)
    c._nvml = None
    rec = c.stop()
    assert rec["sm_mhz"] is None and rec["reasons"] == [] and rec["samples"] == 0


def test_nvidia_smi_line_parsed(monkeypatch):
    line = "0, 1837, 1965, 812.40, 0x0000000000000004, Not Active, Not Active, Not Active, Active\n"

    class R:
        stdout = line

    monkeypatch.setattr(subprocess, "run", lambda *a, **k: R())
    c = bench.ClockSampler(0)
    c._nvml = None
    sm, mx, reasons = c._sample_smi()
    assert sm == 1837.0 and mx == 1965.0 and reasons == {"sw_power_cap"}
