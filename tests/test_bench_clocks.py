"""bench.py's clock sampler on the CPU, against a stand-in nvidia-smi that
prints CSV samples at an interval: start() returns only once the sampler is
up and drops the sample taken before the timed region; stop() reports the
median SM clock, the maximum, the sample count and every throttle reason seen
active."""
import os
import stat
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

FAKE = r"""#!{python}
import sys, time
time.sleep({delay})
rows = [
    "0, 1965, 1965, 700.1, 0x0, Not Active, Not Active, Not Active, Not Active",
    "0, 1800, 1965, 990.5, 0x4, Not Active, Not Active, Not Active, Active",
    "0, 1965, 1965, 720.0, 0x0, Not Active, Not Active, Not Active, Not Active",
]
sys.stdout.write("0, 900, 1965, 80.0, 0x0, Not Active, Not Active, Not Active, Not Active\n")  # before the region
sys.stdout.flush()
i = 0
while True:
    time.sleep(0.02)
    sys.stdout.write(rows[i % 3] + "\n")
    sys.stdout.flush()
    i += 1
"""


def _fake(tmp_path, delay=0.3):
    p = tmp_path / "fake-smi"
    p.write_text(FAKE.format(python=sys.executable, delay=delay))
    p.chmod(p.stat().st_mode | stat.S_IEXEC)
    return str(p)


def test_sampler_waits_for_first_sample_and_drops_it(tmp_path):
    import bench
    c = bench.Clocks(0, exe=_fake(tmp_path, delay=0.4))
    t0 = time.monotonic()
    c.start()
    assert time.monotonic() - t0 >= 0.35  # returned only once the sampler was up
    time.sleep(0.3)
    out = c.stop()
    assert out["samples"] >= 5
    assert out["sm_max_mhz"] == 1965.0
    assert out["sm_mhz"] == 1965.0  # the idle 900 MHz sample before the region is not counted
    assert out["reasons"] == ["sw_power_cap"]


def test_sampler_missing_tool(tmp_path):
    import bench
    c = bench.Clocks(0, exe=str(tmp_path / "no-such-tool"))
    c.start()
    assert c.stop()["reasons"] == ["nvidia-smi unavailable"]


def test_sampler_tool_that_fails(tmp_path):
    import bench
    p = tmp_path / "failing-smi"
    p.write_text(f"#!{sys.executable}\nimport sys\nsys.stderr.write('NVIDIA-SMI has failed\\n')\nsys.exit(9)\n")
    p.chmod(p.stat().st_mode | stat.S_IEXEC)
    c = bench.Clocks(0, exe=str(p))
    t0 = time.monotonic()
    c.start(ready_timeout_s=5.0)
    assert time.monotonic() - t0 < 4.0  # end of output ends the wait
    out = c.stop()
    assert out["sm_mhz"] is None and out["reasons"][0].startswith("nvidia-smi: NVIDIA-SMI has failed")
