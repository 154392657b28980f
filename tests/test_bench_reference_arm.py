"""bench.py's reference arm (--impl reference) times the CPU oracle alone:
its JSON line has the contract's keys, and the process maps none of this
repository's native libraries (only the oracle's)."""

from __future__ import annotations

import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent

PROBE = r"""
import json, runpy, sys
sys.argv = ["bench.py", "--impl", "reference", "--workload", "{workload}", "--steps", "1", "--warmup", "0",
            "--particles", "{particles}", "--cpu-sample", "{sample}"]
try:
    runpy.run_path("bench.py", run_name="__main__")
finally:
    maps = open("/proc/self/maps").read()
    print(json.dumps({{"drift_ext": "astrodrift_b200._drift" in sys.modules,
                       "libdrift": "libdrift_b200" in maps, "oracle": "liboracle" in maps}}))
"""


def _run(workload, particles, sample):
    code = PROBE.format(workload=workload, particles=particles, sample=sample)
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=600,
                         check=True).stdout.strip().splitlines()
    return json.loads(out[-2]), json.loads(out[-1])


def test_reference_arm_line_and_native_libraries():
    line, maps = _run("kepler", 64, 16)
    assert line["impl"] == "reference" and line["metric"] == "accepted steps/s"
    assert line["value"] > 0 and line["higher_is_better"] is True
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert line["config"]["workload"] == "kepler-dopr54"
    assert maps == {"drift_ext": False, "libdrift": False, "oracle": True}


def test_reference_arm_times_the_default_bovy_workload():
    line, maps = _run("bovy", 4096, 8)
    assert line["config"]["workload"] == "bovy-uneven-dop853" and line["config"]["rtol"] == 1e-10
    assert line["value"] > 0
    assert not maps["libdrift"] and not maps["drift_ext"]
