"""Host logic of bench.py that needs no GPU: the clock sampler against a fake NVML (reads only) and
the reference arm's JSON line."""
from __future__ import annotations

import time

import bench


class FakeNVML:
    NVML_CLOCK_SM = 1

    def __init__(self, clocks, reasons):
        self.clocks = list(clocks)
        self.reasons = reasons
        self.k = 0

    def nvmlDeviceGetClockInfo(self, handle, kind):
        v = self.clocks[min(self.k, len(self.clocks) - 1)]
        self.k += 1
        return v

    def nvmlDeviceGetMaxClockInfo(self, handle, kind):
        return 1965

    def nvmlDeviceGetCurrentClocksEventReasons(self, handle):
        return self.reasons


def _sampler(fake):
    s = bench.ClockSampler(0)
    s._handle = lambda: (fake, None)
    return s


def test_short_region_still_has_entry_and_exit_samples():
    s = _sampler(FakeNVML([1965], 0))
    with s:
        pass
    out = s.summary()
    assert out["samples"] >= 2
    assert out["sm_mhz"] == 1965.0 and out["sm_max_mhz"] == 1965.0
    assert out["reasons"] == [] and out["source"] == "nvml"


def test_reasons_are_decoded_from_the_event_bits():
    s = _sampler(FakeNVML([1500, 1960, 1965], 0x4 | 0x8))
    with s:
        time.sleep(0.03)
    out = s.summary()
    assert out["reasons"] == ["hw_slowdown", "sw_power_cap"]
    assert out["samples"] >= 3


def test_idle_samples_do_not_pull_the_median_down():
    s = _sampler(FakeNVML([345, 1965, 1965, 1965], 0))
    with s:
        time.sleep(0.03)
    assert s.summary()["sm_mhz"] == 1965.0  # samples below half the max clock are idle, not load


def test_reference_arm_prints_the_contract_line():
    """`bench.py --impl reference` runs on host cores only and prints one JSON line with the keys the
    benchmark contract asks for."""
    import json
    import os
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "0", "--ref-seconds", "0.2"], capture_output=True, text=True, timeout=300,
                         cwd=root)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
