"""The C-ABI library: it loads without a GPU and exports every entry point
that include/tnlb200.h declares; host-side argument checks."""
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(tnlb_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_library_loads_and_exports_declared_symbols():
    from tnl_b200 import _capi

    exported = set(_capi.exported_symbols())
    declared = declared_functions()
    assert declared, "no declarations found"
    missing = [n for n in declared if n not in exported]
    assert not missing, f"declared in include/*.h but not exported: {missing}"
    assert _capi.tnlb_version().decode().startswith("tnlb200")


def test_launch_configuration_rejects_non_power_of_two():
    import tnl_b200

    with pytest.raises(ValueError):
        tnl_b200.LaunchConfiguration("Fixed", 3)
    assert tnl_b200.LaunchConfiguration("Fixed", 1).kernel() == (tnl_b200.capi.KERNEL_SCALAR, 1)
    assert tnl_b200.LaunchConfiguration("Warp").kernel() == (tnl_b200.capi.KERNEL_VECTOR, 32)


def test_error_status_without_gpu():
    """A null handle is rejected on the host before any CUDA call."""
    from tnl_b200 import _capi

    assert _capi.tnlb_spmv(None, 1, None, None, 0, None, None, 1.0, 0.0, 0, 0, 0, 0, None) == _capi.ERR_INVALID_ARGUMENT
    assert b"null" in _capi.tnlb_last_error()
    with pytest.raises(ValueError):
        _capi.check(_capi.ERR_INVALID_ARGUMENT)
    with pytest.raises(OverflowError):
        _capi.check(_capi.ERR_OVERFLOW)


def test_cpp_dropin_header_compiles():
    """The C++ drop-in header compiles against the C ABI without a GPU."""
    import shutil
    import subprocess

    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    out = ROOT / "tests" / "cpp" / "_build"
    out.mkdir(exist_ok=True)
    r = subprocess.run([nvcc, "-std=c++17", "-c", str(ROOT / "tests" / "cpp" / "dropin.cpp"), "-I", str(ROOT / "include"),
                        "-o", str(out / "dropin.o")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
