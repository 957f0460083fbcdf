"""bench.py's clock record, on the CPU, against a stand-in nvidia-smi.

The bench samples SM clocks and throttle reasons while it times and puts the
median clock and the reasons seen into its JSON line.  A stand-in
`nvidia-smi` on PATH prints lines in the real tool's CSV layout (its own
timestamp first, every 20 ms), so the windowing and the parsing run here.
"""
import os
import stat
import sys
import textwrap
import time

import pytest

import bench

FAKE = textwrap.dedent("""\
    #!{python}
    import datetime, sys, time
    # fields after the timestamp: index, clocks.sm, clocks.max.sm, power.draw,
    # reasons.active, hw_slowdown, hw_thermal_slowdown, sw_thermal_slowdown, sw_power_cap
    end = time.time() + 20
    k = 0
    while time.time() < end:
        now = datetime.datetime.now().strftime("%Y/%m/%d %H:%M:%S.%f")[:-3]
        cap = "Active" if k % 4 == 1 else "Not Active"
        sm = 1965 if k % 2 else 1905
        print(f"{{now}}, 0, {{sm}}, 1965, 700.00, 0x0000000000000004, Not Active, Not Active, Not Active, {{cap}}",
              flush=True)
        k += 1
        time.sleep(0.02)
""")


@pytest.fixture
def fake_smi(tmp_path, monkeypatch):
    path = tmp_path / "nvidia-smi"
    path.write_text(FAKE.format(python=sys.executable))
    path.chmod(path.stat().st_mode | stat.S_IXUSR)
    monkeypatch.setenv("PATH", f"{tmp_path}{os.pathsep}{os.environ['PATH']}")
    return path


def test_samples_inside_the_timed_region(fake_smi):
    s = bench.ClockSampler(0)
    s.start()
    time.sleep(0.1)  # the warm-up
    s.begin()
    time.sleep(0.4)
    rec = s.stop()
    assert rec is not None and rec["window"] == "timed region"
    assert rec["samples"] >= 5
    assert rec["sm_max_mhz"] == 1965.0
    assert rec["sm_mhz"] in (1905.0, 1935.0, 1965.0)  # the median of alternating samples
    assert rec["reasons"] == ["sw_power_cap"]


def test_a_region_too_short_for_a_sample_takes_the_samples_after_it(fake_smi):
    s = bench.ClockSampler(0)
    s.start()
    s.begin()
    rec = s.stop()  # no time for a 20 ms sample inside
    assert rec is not None
    assert rec["window"].startswith("0.3 s after the timed region")
    assert rec["samples"] >= 1


def test_no_nvidia_smi_gives_no_record(tmp_path, monkeypatch):
    monkeypatch.setenv("PATH", str(tmp_path))  # an empty directory: no nvidia-smi
    s = bench.ClockSampler(0)
    s.start(ready_s=0.2)
    s.begin()
    assert s.stop() is None


def test_timestamps_are_nvidia_smis_own():
    line = "2026/12/04 01:07:17.123, 0, 1965, 1965, 700.00, 0x0, Not Active, Not Active, Not Active, Not Active"
    t = bench.ClockSampler._stamp(line)
    assert t is not None and abs(t - time.mktime((2026, 12, 4, 1, 7, 17, 0, 0, -1)) - 0.123) < 1e-3
    assert bench.ClockSampler._stamp("not a sample") is None
