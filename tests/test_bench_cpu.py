"""The CPU arm of bench.py (``--impl reference``) prints one JSON line with the
contract's keys, and under several ranks only rank 0 prints."""

from __future__ import annotations

import json
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def _run(env_extra: dict) -> str:
    env = {**os.environ, **env_extra}
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "2",
                          "--warmup", "3"], capture_output=True, text=True, timeout=300, env=env, cwd=ROOT)
    assert out.returncode == 0, out.stderr
    return out.stdout


def test_reference_arm_prints_the_contract_line():
    lines = [ln for ln in _run({}).splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference" and line["value"] > 0 and line["steps"] == 2
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert line["e2e"]["value"] == line["value"] and line["cpu_baseline"]["value"] == line["value"]
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1


def test_reference_arm_prints_only_on_rank_0():
    assert _run({"RANK": "1", "WORLD_SIZE": "2"}).strip() == ""


def test_clock_sampler_records_only_inside_the_region(monkeypatch):
    """The sampler reads NVML (faked here) from a thread: set-up and a warm-up
    sample come before the region, samples are taken every millisecond inside
    it, and throttle reasons are decoded from the event-reason mask."""
    import time
    import types

    import bench

    calls = {"max": 0, "clock": 0}

    def max_clock(h, kind):
        calls["max"] += 1
        return 1965

    def clock(h, kind):
        calls["clock"] += 1
        return 1900 + calls["clock"] % 3

    fake = types.SimpleNamespace(
        nvmlInit=lambda: None, nvmlDeviceGetHandleByIndex=lambda i: "h", nvmlDeviceGetHandleByPciBusId=None,
        NVML_CLOCK_SM=0, nvmlDeviceGetMaxClockInfo=max_clock, nvmlDeviceGetClockInfo=clock,
        nvmlDeviceGetCurrentClocksEventReasons=lambda h: 0x4 | 0x8,
        nvmlClocksEventReasonHwSlowdown=0x8, nvmlClocksEventReasonHwThermalSlowdown=0x40,
        nvmlClocksEventReasonSwThermalSlowdown=0x20, nvmlClocksEventReasonSwPowerCap=0x4,
        nvmlClocksEventReasonHwPowerBrakeSlowdown=0x80)
    monkeypatch.setitem(sys.modules, "pynvml", fake)
    clk = bench.Clocks(types.SimpleNamespace(index=0))
    monkeypatch.setattr(clk, "_handle", lambda nvml: "h")
    with clk:
        before = calls["clock"]
        time.sleep(0.03)
    s = clk.summary()
    assert before >= 1 and calls["max"] == 1
    assert s["samples"] >= 5 and s["sm_max_mhz"] == 1965 and 1900 <= s["sm_mhz"] <= 1902
    assert s["reasons"] == ["hw_slowdown", "sw_power_cap"]
