"""ctypes binding of libtnlb200.so (the C ABI declared in include/tnlb200.h).

The library is loaded from tnl_b200/_lib/libtnlb200.so.  There is no
fallback: if the library is missing, importing this module raises
ImportError telling how to build it.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libtnlb200.so"

if not LIB_PATH.exists():
    raise ImportError(
        f"{LIB_PATH} is missing: build the CUDA library with `python tnl_b200/build.py` "
        "(or __graft_entry__.build()); there is no CPU fallback"
    )

lib = C.CDLL(str(LIB_PATH))

# status codes (tnlb_status)
OK, ERR_INVALID_ARGUMENT, ERR_OVERFLOW, ERR_CUDA, ERR_NOT_IMPLEMENTED, ERR_BREAKDOWN, ERR_TIMEOUT, ERR_OOM, ERR_IO = range(9)
F32, F64 = 0, 1
CSR, ELLPACK, SLICED_ELLPACK, CHUNKED_ELLPACK, BIELLPACK, ADAPTIVE_CSR = range(6)
COLUMN_MAJOR, ROW_MAJOR = 0, 1
KERNEL_DEFAULT, KERNEL_SCALAR, KERNEL_VECTOR, KERNEL_LIGHT, KERNEL_ADAPTIVE, KERNEL_TILE = range(6)
(META_OFFSETS, META_SLICE_OFFSETS, META_SLICE_SEGMENT_SIZES, META_CH_SLICE_SIZE, META_CH_SLICE_CHUNK_SIZE,
 META_CH_SLICE_FIRST, META_CH_SLICE_POINTER, META_CH_SEGMENT_TO_CHUNK, META_CH_SEGMENT_TO_SLICE,
 META_CH_SEGMENT_POINTERS, META_CH_CHUNKS_TO_SEGMENTS, META_BI_PERMUTATION, META_BI_GROUP_POINTERS) = range(13)


class BackendRuntimeError(RuntimeError):
    """A CUDA error (the reference's Exceptions::BackendRuntimeError)."""


class BreakdownError(RuntimeError):
    """A zero pivot in the GMRES least-squares update (the reference throws 1)."""


class DeviceTimeoutError(RuntimeError):
    """A bounded device-side wait gave up."""


class SegmentsInfo(C.Structure):
    _fields_ = [
        ("format", C.c_int32), ("organization", C.c_int32), ("segments", C.c_int32), ("reserved0", C.c_int32),
        ("elements", C.c_int64), ("storage", C.c_int64), ("segment_size", C.c_int32), ("aligned_size", C.c_int32),
        ("slices", C.c_int32), ("chunks_in_slice", C.c_int32), ("acsr_blocks", C.c_int64 * 6),
    ]


class AcsrBlock(C.Structure):
    _fields_ = [
        ("type", C.c_uint8), ("warp_idx", C.c_uint8), ("warps_count", C.c_uint8), ("reserved", C.c_uint8),
        ("first_segment", C.c_int32), ("block_size", C.c_int32), ("segments_in_block", C.c_int32),
    ]


class SolverParams(C.Structure):
    _fields_ = [
        ("max_iterations", C.c_int32), ("min_iterations", C.c_int32), ("convergence_residue", C.c_double),
        ("divergence_residue", C.c_double), ("gmres_variant", C.c_int32), ("gmres_restarting_min", C.c_int32),
        ("gmres_restarting_max", C.c_int32), ("gmres_restarting_step_min", C.c_int32),
        ("gmres_restarting_step_max", C.c_int32), ("bicgstab_exact_residue", C.c_int32), ("spmv_kernel", C.c_int32),
        ("bicgstab_ell", C.c_int32), ("idr_s", C.c_int32), ("idr_residual_smoothing", C.c_int32),
        ("reliable_layout", C.c_int32), ("reliable_operator", C.c_int32),
    ]


class HostCSR(C.Structure):
    _fields_ = [("rows", C.c_int32), ("columns", C.c_int32), ("nnz", C.c_int64), ("rowptr", C.POINTER(C.c_int32)),
                ("cols", C.POINTER(C.c_int32)), ("values", C.POINTER(C.c_double))]


class MatrixFileInfo(C.Structure):
    _fields_ = [("format", C.c_int32), ("organization", C.c_int32), ("real", C.c_int32), ("symmetric", C.c_int32),
                ("rows", C.c_int64), ("columns", C.c_int64), ("storage", C.c_int64), ("type", C.c_char * 512)]


class SolveResult(C.Structure):
    _fields_ = [("converged", C.c_int32), ("iterations", C.c_int32), ("residue", C.c_double),
                ("status_detail", C.c_int32), ("fallback_iterations", C.c_int32)]


SOLVER_CG, SOLVER_BICGSTAB, SOLVER_GMRES, SOLVER_FGMRES, SOLVER_TFQMR, SOLVER_BICGSTABL, SOLVER_IDRS = range(7)
PRECOND_NONE, PRECOND_JACOBI, PRECOND_ILU0, PRECOND_FSAI, PRECOND_FSAI2, PRECOND_ILUT = range(6)
GMRES_CGS, GMRES_CGSR, GMRES_MGS, GMRES_MGSR, GMRES_CWY = range(5)

_p = C.c_void_p
_i32, _i64, _f64 = C.c_int32, C.c_int64, C.c_double


def _sig(name, argtypes, restype=C.c_int):
    f = getattr(lib, name)
    f.argtypes = argtypes
    f.restype = restype
    return f


tnlb_last_error = _sig("tnlb_last_error", [], C.c_char_p)
tnlb_version = _sig("tnlb_version", [], C.c_char_p)
tnlb_segments_create = _sig("tnlb_segments_create", [C.c_int, C.c_int, _p, _i32, _p, C.POINTER(_p)])
tnlb_segments_destroy = _sig("tnlb_segments_destroy", [_p])
tnlb_segments_get_info = _sig("tnlb_segments_get_info", [_p, C.POINTER(SegmentsInfo)])
tnlb_segments_read_metadata = _sig("tnlb_segments_read_metadata", [_p, C.c_int, _p, _i64])
tnlb_segments_read_acsr_blocks = _sig("tnlb_segments_read_acsr_blocks", [_p, _i32, _p, _i64])
tnlb_segments_global_index = _sig("tnlb_segments_global_index", [_p, _p, _p, _i64, _p, _p])
tnlb_matrix_fill_from_csr = _sig("tnlb_matrix_fill_from_csr", [_p, C.c_int, _p, _p, _p, _p, _p, _p])
tnlb_spmv = _sig("tnlb_spmv", [_p, C.c_int, _p, _p, _i32, _p, _p, _f64, _f64, _i32, _i32, C.c_int, _i32, _p])
tnlb_spmv_last_launch_count = _sig("tnlb_spmv_last_launch_count", [], _i32)
tnlb_mtx_read = _sig("tnlb_mtx_read", [C.c_char_p, _i32, C.POINTER(HostCSR)])
tnlb_mtx_write = _sig("tnlb_mtx_write", [C.c_char_p, _i32, _i32, _p, _p, _p])
tnlb_host_csr_free = _sig("tnlb_host_csr_free", [C.POINTER(HostCSR)], None)
tnlb_matrix_to_host_csr = _sig("tnlb_matrix_to_host_csr", [_p, C.c_int, _p, _p, _i32, C.POINTER(HostCSR)])
tnlb_spmv_symmetric = _sig("tnlb_spmv_symmetric", [_p, C.c_int, _p, _p, _p, _p, _f64, _f64, _i32, _i32, _p])
tnlb_spmv_transposed = _sig("tnlb_spmv_transposed", [_p, C.c_int, _p, _p, _i32, _p, _p, _f64, _f64, _i32, _i32, _p])
tnlb_spmv_csr_noalloc = _sig("tnlb_spmv_csr_noalloc",
                             [C.c_int, _i32, _i32, C.c_int64, _p, _p, _p, _p, _p, _f64, _f64, _p])
tnlb_dot = _sig("tnlb_dot", [C.c_int, _i64, _p, _p, _p, _p])
tnlb_axpby = _sig("tnlb_axpby", [C.c_int, _i64, _f64, _p, _f64, _p, _p])
tnlb_bench_stream_gather = _sig("tnlb_bench_stream_gather", [C.c_int, _i32, _i32, _i64, _p, _p, _p, _p, _p, _p])
tnlb_matrix_assemble_laplace_2d = _sig("tnlb_matrix_assemble_laplace_2d", [_p, C.c_int, _i32, _p, _p, _p])
tnlb_segments_offsets_view = _sig("tnlb_segments_offsets_view", [_p, C.POINTER(_p)])
tnlb_solver_params_default = _sig("tnlb_solver_params_default", [C.POINTER(SolverParams)], None)
tnlb_solve = _sig("tnlb_solve", [C.c_int, C.c_int, C.POINTER(SolverParams), _p, C.c_int, _p, _p, _p, _p, _p,
                                 C.POINTER(SolveResult)])
tnlb_true_residual = _sig("tnlb_true_residual", [_p, C.c_int, _p, _p, _p, _p, _p, C.POINTER(_f64)])
tnlb_solve_mixed = _sig("tnlb_solve_mixed", [C.POINTER(SolverParams), _p, _p, _p, _p, _p, _f64, _i32, C.c_int,
                                             C.c_int, _p, _p, C.POINTER(SolveResult), C.POINTER(_i32)])
tnlb_matrix_save = _sig("tnlb_matrix_save", [C.c_char_p, _p, C.c_int, _p, _p, _i32, _i32, _i32])
tnlb_matrix_file_info_read = _sig("tnlb_matrix_file_info_read", [C.c_char_p, C.POINTER(MatrixFileInfo)])
tnlb_matrix_load = _sig("tnlb_matrix_load", [C.c_char_p, C.POINTER(_p), _p, _p, _i64])
tnlb_matrix_transpose_rowptr = _sig("tnlb_matrix_transpose_rowptr", [_p, _p, _i32, _p, C.POINTER(_i64), _p])
tnlb_matrix_transpose_fill = _sig("tnlb_matrix_transpose_fill", [_p, C.c_int, _p, _p, _i32, _f64, _p, _p, _p])
tnlb_solve_mixed_reliable = _sig("tnlb_solve_mixed_reliable", [C.POINTER(SolverParams), _p, _p, _p, _p, _p, _f64,
                                                               C.c_int, C.c_int, _p, _p, C.POINTER(SolveResult),
                                                               C.POINTER(_i32)])
tnlb_precond_create_ilut = _sig("tnlb_precond_create_ilut", [_p, C.c_int, _p, _p, _i32, _f64, _p, C.POINTER(_p)])
tnlb_precond_create_fsai = _sig("tnlb_precond_create_fsai", [_p, C.c_int, _p, _p, _i32, _p, C.POINTER(_p)])
tnlb_precond_create = _sig("tnlb_precond_create", [C.c_int, _p, C.c_int, _p, _p, _p, C.POINTER(_p)])
tnlb_precond_solve = _sig("tnlb_precond_solve", [_p, _p, _p, _p])
tnlb_precond_destroy = _sig("tnlb_precond_destroy", [_p])
tnlb_precond_read_factor = _sig("tnlb_precond_read_factor", [_p, _i32, _p, _p, _p, _i64])
tnlb_solve_preconditioned = _sig("tnlb_solve_preconditioned", [C.c_int, _p, C.POINTER(SolverParams), _p, C.c_int, _p,
                                                               _p, _p, _p, _p, C.POINTER(SolveResult)])
tnlb_lfsai_num_params = _sig("tnlb_lfsai_num_params", [], _i64)
tnlb_lfsai_create = _sig("tnlb_lfsai_create", [C.c_uint64, _p, C.POINTER(_p)])
tnlb_lfsai_destroy = _sig("tnlb_lfsai_destroy", [_p])
tnlb_lfsai_get_params = _sig("tnlb_lfsai_get_params", [_p, _p, _i64])
tnlb_lfsai_set_params = _sig("tnlb_lfsai_set_params", [_p, _p, _i64])
tnlb_lfsai_get_grad = _sig("tnlb_lfsai_get_grad", [_p, _p, _i64])
tnlb_lfsai_set_tensor_cores = _sig("tnlb_lfsai_set_tensor_cores", [_p, _i32])
tnlb_lfsai_set_level = _sig("tnlb_lfsai_set_level", [_p, _i32])
tnlb_lfsai_set_two_factor = _sig("tnlb_lfsai_set_two_factor", [_p, _i32])
tnlb_lfsai_gradient = _sig("tnlb_lfsai_gradient", [_p, _i32, _p, C.c_int, _p, _p, _p, _i32, _p, C.POINTER(_f64)])
tnlb_lfsai_adam_step = _sig("tnlb_lfsai_adam_step", [_p, _f64, _p])
tnlb_lfsai_precond_create = _sig("tnlb_lfsai_precond_create", [_p, _p, C.c_int, _p, _p, _p, C.POINTER(_p)])
tnlb_lfsai_eval = _sig("tnlb_lfsai_eval", [_p, _p, C.c_int, _p, _p, _p, _p, _p])
tnlb_ilu0_factors = _sig("tnlb_ilu0_factors", [_p, C.c_int, _p, _p, _p, _p, _p, _i64, _p])


def check(status: int) -> None:
    """Raise the exception the reference would throw for this status."""
    if status == OK:
        return
    msg = (tnlb_last_error() or b"").decode(errors="replace")
    if status == ERR_INVALID_ARGUMENT:
        raise ValueError(msg)
    if status == ERR_OVERFLOW:
        raise OverflowError(msg)
    if status == ERR_NOT_IMPLEMENTED:
        raise NotImplementedError(msg)
    if status == ERR_BREAKDOWN:
        raise BreakdownError(msg)
    if status == ERR_TIMEOUT:
        raise DeviceTimeoutError(msg)
    if status == ERR_OOM:
        raise MemoryError(msg)
    if status == ERR_IO:
        raise RuntimeError(msg)
    raise BackendRuntimeError(msg)


def exported_symbols() -> list[str]:
    """Names of every tnlb_* function the library exports (checked against the header)."""
    import subprocess

    out = subprocess.run(["nm", "-D", "--defined-only", str(LIB_PATH)], capture_output=True, text=True).stdout
    return sorted({ln.split()[-1] for ln in out.splitlines() if " T " in ln and ln.split()[-1].startswith("tnlb_")})
