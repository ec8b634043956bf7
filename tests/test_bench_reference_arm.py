"""bench.py --impl reference on the CPU: for every workload it prints one JSON line with the
metric and unit of our own arm for that workload, "impl": "reference", a cpu_baseline that
describes the run and an e2e entry with no host-device traffic.  Tiny samples (--cpu-steps)
keep each run to seconds."""
import json
import subprocess
import sys

import pytest

from conftest import ROOT

CASES = [
    (["--workload", "rtm"], "RTM shots/s", "shots/s"),
    (["--workload", "afor"], "modelling shots/s", "shots/s"),
    (["--workload", "lsrtm"], "LSRTM gradient shots/s", "shots/s"),
    (["--workload", "batch"], "RTM shots/s", "shots/s"),
    (["--workload", "decon", "--config", "c2"], "decon windows/s", "windows/s"),
    (["--workload", "c5flow"], "RTM shots/s", "shots/s"),
]


@pytest.mark.parametrize("extra,metric,unit", CASES, ids=[c[0][1] for c in CASES])
def test_reference_arm_line(extra, metric, unit):
    cmd = [sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1", "--warmup", "0",
           "--cpu-steps", "16"] + extra
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [line for line in r.stdout.splitlines() if line.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert (d["metric"], d["unit"]) == (metric, unit)
    assert d["value"] > 0 and d["steps"] == 1 and d["warmup"] == 0
    assert d["higher_is_better"] is True
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["value"] == pytest.approx(d["value"])
    assert d["e2e"] == {"value": d["value"], "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["config"]["workload"]


def test_reference_arm_maps_no_product_library_and_times_what_it_ran():
    """The reference arm runs the oracle only: the process maps no libswd, and its steps x
    ms_per_step is time it actually spent (each step one bounded sample), so it fits inside
    the run's own wall clock."""
    code = ("import runpy, sys, time; t = time.perf_counter(); "
            "sys.argv = ['bench.py', '--impl', 'reference', '--steps', '2', '--warmup', '1', '--cpu-steps', '16']; "
            "runpy.run_path('bench.py', run_name='__main__'); "
            "maps = open('/proc/self/maps').read(); "
            "print('WALL', time.perf_counter() - t); print('LIBSWD', maps.count('libswd'))")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    out = r.stdout.splitlines()
    d = json.loads([line for line in out if line.startswith("{")][0])
    wall = float([line for line in out if line.startswith("WALL")][0].split()[1])
    assert int([line for line in out if line.startswith("LIBSWD")][0].split()[1]) == 0
    assert d["steps"] * d["ms_per_step"] / 1e3 <= wall
    assert "oracle" in d["cpu_baseline"]["sample"] or d["cpu_baseline"]["kind"] == "port"
