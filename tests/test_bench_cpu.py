"""bench.py's reference arm on CPU: it times the reference's own code
(oracle/_ref, compiled from the reference's sources) and loads nothing of the
product library."""
import json
import os
import subprocess
import sys

import pytest

import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")
def test_reference_arm_loads_no_product_library():
    code = (
        "import json, sys; sys.path.insert(0, %r); import bench\n"
        "class A: steps, warmup = 1, 0\n"
        "line = bench.run_reference(A(), 0)\n"
        "maps = open('/proc/self/maps').read()\n"
        "print(json.dumps({'line': line, 'libvct': 'virtualct_b200/lib/' in maps, 'ref': 'libvct_ref_mb' in maps}))\n" % ROOT)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert out["ref"] and not out["libvct"]
    line = out["line"]
    assert line["impl"] == "reference" and line["value"] > 0 and line["unit"] == "rays*bins/s"
    cb = line["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["cpu_model"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0
