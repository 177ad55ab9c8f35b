"""bench.py's host side on CPU.  The reference arm times the oracle (the CPU restatement
of the reference's rayon step) through the same command line as the product's arm,
prints the contract's JSON line with "impl": "reference", and never loads the product
library (libphysph.so) into its process, so the measured baseline contains none of this
library's code.  The flop side of the roofline follows from the device counters."""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent

# Runs bench.py as its own __main__ on a small scene, then reports which shared
# objects of the repository the process mapped.
_DRIVER = r"""
import json, runpy, sys
sys.argv = ["bench.py", "--impl", "reference", "--steps", "3", "--warmup", "3", "--dims", "8", "16", "8"]
runpy.run_path("bench.py", run_name="__main__")
paths = {l.split()[-1] for l in open("/proc/self/maps").read().splitlines() if l.endswith(".so")}
print("MAPPED " + json.dumps(sorted(p for p in paths if "physph" in p or "liboracle" in p)))
"""


def test_reference_arm_prints_its_line_without_the_product_library():
    out = subprocess.run([sys.executable, "-c", _DRIVER], cwd=ROOT, capture_output=True,
                         text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout
    line = json.loads(lines[0])
    assert line["impl"] == "reference"
    assert line["steps"] == 3 and line["warmup"] == 3
    assert line["value"] > 0 and line["unit"] == "particle-steps/s" and line["higher_is_better"] is True
    assert line["config"]["particles"] == 8 * 16 * 8
    cb = line["cpu_baseline"]
    assert cb["value"] == line["value"] and cb["kind"] == "port" and cb["cores"] >= 1
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    mapped = [l for l in out.stdout.splitlines() if l.startswith("MAPPED ")]
    assert len(mapped) == 1
    libs = json.loads(mapped[0][len("MAPPED "):])
    assert any(p.endswith("liboracle.so") for p in libs), libs
    assert not any("libphysph" in p for p in libs), libs


def test_flop_rate_from_counters():
    sys.path.insert(0, str(ROOT))
    import bench
    n = 1000
    r = bench.flop_rate({"candidates": 219 * n, "pairs": 30 * n, "particles": n, "cells": 0}, n, 2.0)
    assert r["candidates_per_particle"] == 219.0 and r["pairs_per_particle"] == 30.0
    assert r["flops_per_particle_step"] == 2 * 8 * 219 + 72 * 30
    assert abs(r["achieved_tflops"] - r["flops_per_particle_step"] * n / 2e-3 / 1e12) < 1e-15
    assert r["peak"] is None
