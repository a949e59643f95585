"""The bench's reference arm on the CPU: `bench.py --impl reference` times the
reference's own SMCSampler (compiled from its headers into oracle/_ref) on a
bounded sample, prints the contract's JSON line, and never loads this
package's library (the arm must measure the reference alone)."""
import json
import os
import subprocess
import sys

import pytest

import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

_RUN = r"""
import runpy, sys
sys.argv = ["bench.py", "--impl", "reference", "--steps", "2", "--warmup", "0", "--filters", "32", "--obs", "20"]
try:
    runpy.run_path("bench.py", run_name="__main__")
finally:
    maps = open("/proc/self/maps").read()
    print("LIBRARY_MAPPED=%d MODULE_IMPORTED=%d" % ("libmckl_b200" in maps, "mckl_b200" in sys.modules))
"""


def test_reference_arm_line_and_isolation():
    if not O.have_ref():
        pytest.skip("oracle/_ref is not built on this host")
    r = subprocess.run([sys.executable, "-c", _RUN], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = r.stdout.strip().splitlines()
    assert lines[-1] == "LIBRARY_MAPPED=0 MODULE_IMPORTED=0", lines[-1]
    line = json.loads(lines[-2])
    assert line["impl"] == "reference"
    assert line["unit"] == "particle-steps/s" and line["value"] > 0
    assert line["steps"] == 2 and line["warmup"] == 0 and line["ms_per_step"] > 0
    assert line["higher_is_better"] is True
    cb = line["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == line["value"] and cb["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
