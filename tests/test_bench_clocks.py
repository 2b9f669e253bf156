"""The bench's clock record: nvidia-smi rows taken inside the timed region.

A stand-in nvidia-smi on PATH prints idle rows (300 MHz) for its first
0.4 s and loaded rows (1965 MHz, sw_power_cap active) after that, so the
summary must hold only the loaded rows that arrived after mark()."""
import importlib.util
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

FAKE = """#!{python}
import sys, time
i = 0
while True:
    mhz = 300 if i < 4 else 1965
    print(f"0, {{mhz}}, 1965, 650.0, 0x4, Not Active, Not Active, Not Active, Active", flush=True)
    time.sleep(0.1)
    i += 1
"""


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_clock_record_covers_only_the_timed_region(tmp_path, monkeypatch):
    fake = tmp_path / "nvidia-smi"
    fake.write_text(FAKE.format(python=sys.executable))
    fake.chmod(0o755)
    monkeypatch.setenv("PATH", f"{tmp_path}{os.pathsep}{os.environ.get('PATH', '')}")
    bench = _bench()
    c = bench.ClockSampler(0)
    c.start()
    assert c.rows, "start() returns once the first row has arrived"
    time.sleep(0.7)
    c.mark()
    time.sleep(0.5)
    rec = c.stop()
    assert rec["samples"] >= 3
    assert rec["sm_mhz"] == 1965.0 and rec["sm_max_mhz"] == 1965.0
    assert rec["reasons"] == ["sw_power_cap"]


def test_clock_record_without_nvidia_smi(tmp_path, monkeypatch):
    monkeypatch.setenv("PATH", str(tmp_path))
    bench = _bench()
    c = bench.ClockSampler(0)
    c.start()
    c.mark()
    rec = c.stop()
    assert rec == {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
