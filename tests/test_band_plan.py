"""The staging plan of the bulk-copy band products, checked on the CPU.

The reliable-update PCG's FSAI factor products stage their operands in
shared memory with bulk copies (cp.async.bulk), which need 16-byte-aligned
addresses and sizes; an unaligned copy is an illegal instruction on the GPU.
band_plan_check.cu compiles the host-side planner of tnl_b200/csrc/band.cuh
with nvcc (no GPU needed) and checks, for 4000 random diagonal patterns and
tiles of eight matrix sizes, the alignment of every copy band_issue would
issue, that every run fits its slot of the stage and covers the columns its
rows read, the interior-tile offsets, and the stages' fit in one block's
shared memory.
"""
import shutil
import subprocess
from pathlib import Path

import pytest

HERE = Path(__file__).resolve().parent
CSRC = HERE.parent / "tnl_b200" / "csrc"


def _nvcc():
    for cand in ("/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    return None


def test_band_plan_copies_are_aligned_and_fit(tmp_path):
    nvcc = _nvcc()
    if nvcc is None:
        pytest.skip("no nvcc")
    exe = tmp_path / "band_plan_check"
    p = subprocess.run([nvcc, "-std=c++17", "-O2", "-Wno-deprecated-gpu-targets", f"-I{CSRC}",
                        str(HERE / "band_plan_check.cu"), "-o", str(exe)], capture_output=True, text=True,
                       timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.startswith("ok "), r.stdout + r.stderr
    assert int(r.stdout.split()[1]) > 1_000_000
