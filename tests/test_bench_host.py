"""Host logic of bench.py that needs no GPU: the clock sampler keeps only the
nvidia-smi samples taken inside the timed region, and reads the throttle
reasons from them.  A stand-in nvidia-smi script prints idle lines until a
flag file appears, then loaded lines."""
from __future__ import annotations

import os
import stat
import time

import bench

FAKE = """#!/bin/bash
while true; do
  if [ -f "{flag}" ]; then
    echo "0, 1900, 1965, 700.0, 0x4, Not Active, Not Active, Not Active, Active"
  else
    echo "0, 1200, 1965, 100.0, 0x0, Not Active, Not Active, Not Active, Not Active"
  fi
  sleep 0.02
done
"""


def _fake_smi(tmp_path, monkeypatch):
    flag = tmp_path / "loaded"
    script = tmp_path / "nvidia-smi"
    script.write_text(FAKE.format(flag=flag))
    script.chmod(script.stat().st_mode | stat.S_IXUSR)
    monkeypatch.setenv("PATH", f"{tmp_path}{os.pathsep}{os.environ['PATH']}")
    return flag


def test_clock_samples_are_kept_only_inside_the_timed_region(tmp_path, monkeypatch):
    flag = _fake_smi(tmp_path, monkeypatch)
    with bench.ClockSampler(0) as clk:
        assert clk.lines, "the sampler is live before the caller's work starts"
        time.sleep(0.3)          # idle samples before the region
        flag.touch()
        time.sleep(0.1)
        clk.begin()
        time.sleep(0.3)          # the timed region: loaded samples only
        clk.end()
        flag.unlink()
        time.sleep(0.3)          # idle samples after the region
    s = clk.summary()
    assert s["timed_region_only"] is True
    assert s["samples"] >= 3
    assert s["sm_mhz"] == 1900.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"]
    # the idle samples were taken too, outside the region
    assert any(", 1200," in ln for _, ln in clk.lines)


def test_clock_summary_without_a_region_uses_every_sample(tmp_path, monkeypatch):
    _fake_smi(tmp_path, monkeypatch)
    with bench.ClockSampler(0) as clk:
        time.sleep(0.2)
    s = clk.summary()
    assert s["timed_region_only"] is False
    assert s["sm_mhz"] == 1200.0 and s["reasons"] == []


def test_clock_sampler_without_nvidia_smi_reports_no_samples(tmp_path, monkeypatch):
    monkeypatch.setenv("PATH", str(tmp_path))  # no nvidia-smi on the path
    with bench.ClockSampler(0) as clk:
        clk.begin()
        clk.end()
    assert clk.summary() == {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
