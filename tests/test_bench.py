"""bench.py's host-side bookkeeping that needs no GPU: the committed DRAM traffic per launch,
looked up by kernel kind and mesh family and scaled to the workload's cells."""

import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(REPO))

import bench  # noqa: E402


def test_traffic_is_per_mesh_family_and_scales_with_cells():
    tets = bench.committed_traffic("gradients", 1_016_064, "tets")
    channel = bench.committed_traffic("gradients", 994_600, "channel")
    assert tets == pytest.approx(452_191_659)
    assert channel == pytest.approx(626_937_259)  # the autotuned form's capture
    # the channel's longer stencils (about 23 entries per cell, 13.8 on the tets) read more
    assert channel / 994_600 > 1.4 * tets / 1_016_064
    assert bench.committed_traffic("gradients", 2 * 994_600, "channel") == pytest.approx(2 * channel)
    assert bench.committed_traffic("faces", 1000, "tets") is None
    assert bench.committed_traffic("gradients", 1000, "hex") is None


def test_nvml_clock_sampler_against_a_fake_nvml(monkeypatch):
    """The clock record of the timed region read through NVML (here a fake: 1900 MHz under a
    1965 MHz maximum with the power cap active): median clock, maximum, the active reasons by
    name, and samples taken through a short region."""
    import time
    import types

    fake = types.SimpleNamespace(
        nvmlInit=lambda: None, nvmlShutdown=lambda: None, NVML_CLOCK_SM=1,
        nvmlDeviceGetHandleByUUID=lambda uuid: "handle",
        nvmlDeviceGetMaxClockInfo=lambda h, c: 1965, nvmlDeviceGetClockInfo=lambda h, c: 1900,
        nvmlDeviceGetCurrentClocksEventReasons=lambda h: 0x4,
        nvmlClocksEventReasonHwSlowdown=0x8, nvmlClocksEventReasonHwThermalSlowdown=0x40,
        nvmlClocksEventReasonSwThermalSlowdown=0x20, nvmlClocksEventReasonSwPowerCap=0x4,
    )  # fmt: skip
    monkeypatch.setitem(sys.modules, "pynvml", fake)
    clocks = bench.clock_sampler("GPU-0")
    assert isinstance(clocks, bench.NvmlClockSampler)
    with clocks:
        time.sleep(0.03)
    s = clocks.summary()
    assert s["sm_mhz"] == 1900 and s["sm_max_mhz"] == 1965
    assert s["reasons"] == ["sw_power_cap"] and s["samples"] >= 3


def test_nvml_clock_sampler_survives_failed_reads(monkeypatch):
    """An NVML read that fails leaves the clock record short (here empty) without stopping the
    timed region."""
    import types

    def fail(*a):
        raise RuntimeError("NVML read failed")

    fake = types.SimpleNamespace(
        nvmlInit=lambda: None, nvmlShutdown=lambda: None, NVML_CLOCK_SM=1,
        nvmlDeviceGetHandleByUUID=lambda uuid: "handle", nvmlDeviceGetMaxClockInfo=lambda h, c: 1965,
        nvmlDeviceGetClockInfo=fail, nvmlDeviceGetCurrentClocksEventReasons=fail,
    )  # fmt: skip
    monkeypatch.setitem(sys.modules, "pynvml", fake)
    with bench.clock_sampler("GPU-0") as clocks:
        pass
    assert clocks.summary()["sm_mhz"] is None and clocks.summary()["samples"] == 0
