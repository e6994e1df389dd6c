"""The C-ABI library: it loads without a GPU and exports every entry point
that include/tnlb200.h declares; host-side argument checks."""
import re
from pathlib import Path

import numpy as np
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


MTX_CASES = {
    "general": "%%MatrixMarket matrix coordinate real general\n% a comment\n4 5 6\n1 1 2.5\n2 3 -1\n4 5 1e-3\n"
               "3 2 7\n1 4 0\n2 3 4.25\n",
    "symmetric": "%%MatrixMarket matrix coordinate real symmetric\n3 3 4\n1 1 4\n2 1 -1\n3 3 2\n3 1 0.5\n",
    "pattern": "%%MatrixMarket matrix coordinate pattern general\n3 3 3\n1 2\n3 1\n2 2\n",
    "integer_spaces": "%%MatrixMarket   matrix coordinate integer general\n%\n  2   2   2\n 1  1   3\n\n2 2 -4\n",
}


@pytest.mark.parametrize("case", list(MTX_CASES))
@pytest.mark.parametrize("symmetric", [False, True])
def test_mtx_read_matches_reference(tmp_path, reference, case, symmetric):
    """tnlb_mtx_read (host code of the library, no GPU needed) against the
    reference's own MatrixReader::readMtx: same CSR arrays, or the same error."""
    import tnl_b200

    f = tmp_path / f"{case}.mtx"
    f.write_text(MTX_CASES[case])
    try:
        r = reference.mtx_read(f, symmetric)
    except RuntimeError as e:
        with pytest.raises(RuntimeError) as got:
            tnl_b200.read_mtx(f, symmetric)
        assert str(got.value) == str(e)
        return
    A = tnl_b200.read_mtx(f, symmetric)
    assert (A.n, A.ncols) == (r[0], r[1])
    assert np.array_equal(A.rowptr, r[2]) and np.array_equal(A.cols, r[3]) and np.array_equal(A.vals, r[4])


def test_mtx_errors_match_reference(tmp_path, reference):
    import tnl_b200

    bad = {"header": "%%MatrixMarket matrix array real general\n2 2\n1 2\n3 4\n",
           "size": "%%MatrixMarket matrix coordinate real general\n2 2\n",
           "outside": "%%MatrixMarket matrix coordinate real general\n2 2 1\n3 1 1.0\n",
           "words": "%%MatrixMarket matrix coordinate real general\n2 2 1\n1 1\n"}
    for name, text in bad.items():
        f = tmp_path / f"{name}.mtx"
        f.write_text(text)
        with pytest.raises(RuntimeError) as e_ref:
            reference.mtx_read(f, False)
        with pytest.raises(RuntimeError) as e_ours:
            tnl_b200.read_mtx(f, False)
        assert str(e_ours.value) == str(e_ref.value), name


@pytest.mark.parametrize("line", ["0 1 1.0", "1 0 1.0", "-3 1 1.0", "1 -1 2.0", "x 1 1.0", "1 y 1.0",
                                  "99999999999 1 1.0"])
def test_mtx_rejects_positions_below_one_and_non_numbers(tmp_path, line):
    """A row or column below 1, a word that is not a number, or one beyond
    the int range is an I/O error, never a negative index into the CSR
    arrays (x[-1] on the device, or a write before the row pointer)."""
    import tnl_b200

    f = tmp_path / "bad.mtx"
    f.write_text(f"%%MatrixMarket matrix coordinate real general\n2 2 2\n1 1 4.0\n{line}\n")
    with pytest.raises(RuntimeError) as e:
        tnl_b200.read_mtx(f, False)
    assert "out of the matrix dimensions" in str(e.value) or "not an integer" in str(e.value)


def test_mtx_write_matches_reference_bytes(tmp_path, reference):
    """tnlb_mtx_write writes the bytes of the reference's MatrixWriter::writeMtx."""
    import tnl_b200
    from tnl_b200 import generators as g

    A = g.power_law(300, 1.73, 40, 3)
    A.vals[::7] = 0.0  # zero values are skipped by both
    ours, ref = tmp_path / "ours.mtx", tmp_path / "ref.mtx"
    tnl_b200.write_mtx(ours, A)
    reference.mtx_write(ref, A)
    assert ours.read_bytes() == ref.read_bytes()
    B = tnl_b200.read_mtx(ours)
    assert B.n == A.n and B.ncols == A.ncols


def test_matrix_file_header_of_reference_files(tmp_path):
    """tnlb_matrix_file_info_read (host only) on files the reference's own
    SparseMatrix::save wrote: type string, dimensions and storage of every
    format; a file that is no TNL object is an I/O error with the reason."""
    import ctypes as C

    from oracle.oracle import REF_SO, Reference
    from tnl_b200 import _capi, generators as g

    if not REF_SO.exists():
        pytest.skip("the reference driver oracle/_ref is not built")
    R = Reference()
    A = g.laplacian_2d(7)
    names = {0: "CSR< int >", 1: "Ellpack< int, ColumnMajorOrder, 32 >", 2: "SlicedEllpack< int, ColumnMajorOrder, 32 >",
             3: "ChunkedEllpack< int, ColumnMajorOrder >", 4: "BiEllpack< int, ColumnMajorOrder, 32 >",
             5: "AdaptiveCSR< int >"}
    for fmt, seg in names.items():
        for real64 in (True, False):
            path = tmp_path / f"m{fmt}{int(real64)}.tnl"
            R.save(fmt, A, path, colmajor=True, real64=real64)
            info = _capi.MatrixFileInfo()
            assert _capi.tnlb_matrix_file_info_read(str(path).encode(), C.byref(info)) == _capi.OK
            real = "double" if real64 else "float"
            assert info.type.decode() == (f"Matrices::SparseMatrix< {real}, {seg}, [any_device], int, General, "
                                          "[any_allocator], [any_allocator] >")
            assert info.rows == A.n and info.columns == A.ncols
            assert info.real == (_capi.F64 if real64 else _capi.F32) and info.format == fmt
            assert info.storage >= A.nnz
    bad = tmp_path / "bad.tnl"
    bad.write_bytes(b"not a tnl file")
    info = _capi.MatrixFileInfo()
    assert _capi.tnlb_matrix_file_info_read(str(bad).encode(), C.byref(info)) == _capi.ERR_IO
    assert b"magic number" in _capi.tnlb_last_error()


def test_ctypes_structs_match_the_c_header(tmp_path):
    """Every struct the Python layer mirrors with ctypes has the size and
    field offsets that a C compiler gives the declaration in
    include/tnlb200.h (gcc on a generated probe)."""
    import ctypes as C
    import shutil
    import subprocess

    from tnl_b200 import _capi

    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    mirrors = {
        "tnlb_solver_params": _capi.SolverParams,
        "tnlb_solve_result": _capi.SolveResult,
        "tnlb_segments_info": _capi.SegmentsInfo,
        "tnlb_acsr_block": _capi.AcsrBlock,
        "tnlb_host_csr": _capi.HostCSR,
        "tnlb_matrix_file_info": _capi.MatrixFileInfo,
    }
    lines = ['#include "tnlb200.h"', "#include <stdio.h>", "#include <stddef.h>", "int main(void) {"]
    expected = []
    for cname, py in mirrors.items():
        lines.append(f'   printf("%zu\\n", sizeof({cname}));')
        expected.append(C.sizeof(py))
        for field, _ in py._fields_:
            lines.append(f'   printf("%zu\\n", offsetof({cname}, {field}));')
            expected.append(getattr(py, field).offset)
    lines += ["   return 0;", "}"]
    src = tmp_path / "abi_probe.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "abi_probe"
    subprocess.run(["gcc", "-std=c99", f"-I{ROOT / 'include'}", str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    assert got == expected
