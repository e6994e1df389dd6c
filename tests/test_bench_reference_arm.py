"""bench.py's reference arm times only the reference's own code.

`bench.py --impl reference` runs the reference's Host vectorProduct
(oracle/_ref, else the oracle's C port) on the host cores.  Its speed is the
denominator of every ratio against this library, so the process must not
load this library's CUDA code at all, not even as a side effect of an
import.  The arm runs here in a subprocess (CPU only), which then reports
what it has mapped.
"""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent

PROBE = r"""
import contextlib, io, json, runpy, sys
sys.argv = ["bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0", "--no-solver"]
out = io.StringIO()
code = 0
try:
    with contextlib.redirect_stdout(out):
        runpy.run_path("bench.py", run_name="__main__")
except SystemExit as e:
    code = e.code or 0
maps = open("/proc/self/maps").read()
print(json.dumps({"exit": code, "line": out.getvalue().strip().splitlines()[-1],
                  "libtnlb200": "libtnlb200" in maps, "torch": "torch" in sys.modules}))
"""


def test_reference_arm_runs_without_the_library():
    p = subprocess.run([sys.executable, "-c", PROBE], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    r = json.loads(p.stdout.strip().splitlines()[-1])
    assert r["exit"] == 0
    assert not r["libtnlb200"], "the reference arm mapped libtnlb200.so"
    assert not r["torch"], "the reference arm imported torch"
    line = json.loads(r["line"])
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] in ("reference", "port")
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
