"""bench.py pieces that need no GPU: the reference arm (the oracle's residual on the host cores)
prints one JSON line for the bench workload without loading the product library, and the
committed algorithmic FLOP counts are what the roofline reads."""
import json
import os
import subprocess
import sys

import bench

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROBE = r"""
import sys
sys.argv = ["bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0"]
sys.path.insert(0, ".")
import bench
bench.main()
maps = open("/proc/self/maps").read()
print("LOADED" if "libflowgpu.so" in maps else "NOT_LOADED")
"""


def test_reference_arm_line_without_the_product_library():
    r = subprocess.run([sys.executable, "-c", PROBE], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert lines[-1] == "NOT_LOADED"
    line = json.loads(lines[-2])
    assert line["impl"] == "reference" and line["metric"] == bench.METRIC and line["unit"] == "DOF/s"
    assert line["config"]["workload"] == bench.WORKLOAD
    assert line["value"] > 0 and line["ms_per_step"] > 0
    assert line["e2e"]["value"] == line["value"] and line["e2e"]["h2d_bytes_per_step"] == 0
    assert line["cpu_baseline"]["kind"] == "port"


def test_algorithmic_flops_read_by_the_roofline():
    d = json.load(open(os.path.join(ROOT, "tests", "golden", "residual_flops.json")))
    assert bench.algorithmic_flops("ns2_p2") == d["ns2_p2"]["flops"]
    assert bench.algorithmic_flops("euler3_p2") == d["euler3_p2"]["flops"]
    assert bench.algorithmic_flops("no_such_workload") is None
