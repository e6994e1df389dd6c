"""The C++ drop-in layer (include/tnlb/tnlb.hpp) run on the GPU: a program
written against the reference's API (SparseMatrix, vectorProduct, CG with
Diagonal) links libtnlb200.so and checks a known answer and a solve."""
import shutil
import subprocess
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]


def test_cpp_dropin_program():
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    out = ROOT / "tests" / "cpp" / "_build"
    out.mkdir(exist_ok=True)
    lib = ROOT / "tnl_b200" / "_lib"
    exe = out / "dropin"
    r = subprocess.run([nvcc, "-std=c++17", str(ROOT / "tests" / "cpp" / "dropin.cpp"), "-I", str(ROOT / "include"),
                        "-L", str(lib), "-ltnlb200", f"-Xlinker=-rpath={lib}", "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120, cwd=str(out))
    assert r.returncode == 0 and r.stdout.startswith("OK"), r.stdout + r.stderr


def test_cpp_device_assembly_program():
    """SparseMatrix::forAllElements with a device lambda (CSR storage) and
    the library's compiled Laplace assembler (SlicedEllpack storage) build
    the operator of the reference's sparse set-up benchmark; the program
    checks both by a product against a host-built CSR."""
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    out = ROOT / "tests" / "cpp" / "_build"
    out.mkdir(exist_ok=True)
    lib = ROOT / "tnl_b200" / "_lib"
    exe = out / "assembly"
    r = subprocess.run([nvcc, "-std=c++17", "--extended-lambda", "-gencode", "arch=compute_100a,code=sm_100a",
                        str(ROOT / "tests" / "cpp" / "assembly.cu"), "-I", str(ROOT / "include"), "-L", str(lib),
                        "-ltnlb200", f"-Xlinker=-rpath={lib}", "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120, cwd=str(out))
    assert r.returncode == 0 and r.stdout.startswith("OK"), r.stdout + r.stderr
