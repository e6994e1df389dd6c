"""tnl_b200 -- TNL's sparse formats, SpMV and Krylov solvers on NVIDIA B200.

A Python host layer over the C ABI of libtnlb200.so (include/tnlb200.h),
mirroring the reference's class names and argument meanings:

* segments formats ``CSR``, ``Ellpack``, ``SlicedEllpack``, ``ChunkedEllpack``,
  ``BiEllpack``, ``AdaptiveCSR`` (TNL::Algorithms::Segments) with
  ``setSegmentsSizes``, ``getSegmentCount``, ``getElementCount``,
  ``getStorageSize`` and the metadata getters;
* ``SparseMatrix`` (TNL::Matrices::SparseMatrix, general matrices) with
  ``setDimensions``, ``setRowCapacities``, ``assign`` (the cross-format
  ``operator=``), ``vectorProduct``;
* ``LaunchConfiguration`` (TNL::Algorithms::Segments::LaunchConfiguration).

Device memory comes from PyTorch (CUDA tensors); all arithmetic runs in the
library's CUDA kernels.  Errors raise the Python counterparts of the
reference's exceptions (ValueError for std::invalid_argument,
OverflowError for std::overflow_error, BackendRuntimeError for CUDA errors).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _capi as capi
from ._capi import BackendRuntimeError, BreakdownError, DeviceTimeoutError, check  # noqa: F401
from .generators import CSRMatrix  # noqa: F401

__all__ = [
    "CSR", "Ellpack", "SlicedEllpack", "ChunkedEllpack", "BiEllpack", "AdaptiveCSR", "SparseMatrix",
    "LaunchConfiguration", "ColumnMajorOrder", "RowMajorOrder", "CSRMatrix", "check", "BackendRuntimeError",
    "CG", "BICGStab", "GMRES", "FGMRES", "TFQMR", "BICGStabL", "IDRs", "Diagonal", "ILU0", "FSAI", "FSAI2",
    "solve_mixed", "solve_mixed_reliable", "true_residual", "ILUT", "read_mtx", "write_mtx", "assemble_laplace_2d",
]

ColumnMajorOrder = capi.COLUMN_MAJOR
RowMajorOrder = capi.ROW_MAJOR


def _stream(stream=None) -> int:
    s = torch.cuda.current_stream() if stream is None else stream
    return s.cuda_stream


def _real_code(dtype) -> int:
    if dtype == torch.float64:
        return capi.F64
    if dtype == torch.float32:
        return capi.F32
    raise TypeError(f"unsupported real type {dtype}")


def _device_i32(a) -> torch.Tensor:
    if isinstance(a, torch.Tensor):
        return a.to(device="cuda", dtype=torch.int32).contiguous()
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.int32)).cuda()


class LaunchConfiguration:
    """Segments::LaunchConfiguration (Algorithms/Segments/LaunchConfiguration.h:18-86).

    ``mapping`` is one of the ThreadsToSegmentsMapping names ("Fixed",
    "Warp", "Block", "BlockMerged", "DynamicGrouping") or one of the kernel
    names of SegmentsReductionKernels ("Scalar", "Vector", "Light",
    "Adaptive", "Default"), or "Tile" (CSR: the merge-path tile kernel
    whatever the row lengths).  ``threadsPerSegmentCount`` must be a positive
    power of two (std::invalid_argument otherwise, as in the reference).
    """

    def __init__(self, mapping: str = "Default", threadsPerSegmentCount: int = 0):
        if threadsPerSegmentCount and (threadsPerSegmentCount < 0 or threadsPerSegmentCount & (threadsPerSegmentCount - 1)):
            raise ValueError("Threads per segment count must be a positive power of two.")
        self.mapping = mapping
        self.tps = int(threadsPerSegmentCount)

    def kernel(self) -> tuple[int, int]:
        m = self.mapping
        if m in ("Default", "DynamicGrouping", "BlockMerged"):
            return capi.KERNEL_DEFAULT, self.tps
        if m == "Scalar" or (m == "Fixed" and self.tps in (0, 1)):
            return capi.KERNEL_SCALAR, 1
        if m in ("Fixed", "Vector"):
            return capi.KERNEL_VECTOR, self.tps or 32
        if m == "Warp":
            return capi.KERNEL_VECTOR, 32
        if m == "Block":
            return capi.KERNEL_VECTOR, self.tps or 256
        if m == "Light":
            return capi.KERNEL_LIGHT, self.tps
        if m == "Adaptive":
            return capi.KERNEL_ADAPTIVE, 0
        if m == "Tile":
            return capi.KERNEL_TILE, 0
        raise ValueError(f"unknown launch mapping {m}")


class _Segments:
    FORMAT = -1
    DEFAULT_ORGANIZATION = ColumnMajorOrder

    def __init__(self, organization: int | None = None):
        self.organization = self.DEFAULT_ORGANIZATION if organization is None else organization
        self._h = C.c_void_p()
        self._info = capi.SegmentsInfo()

    def __del__(self):
        try:
            if self._h:
                capi.tnlb_segments_destroy(self._h)
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def setSegmentsSizes(self, sizes) -> None:
        d = _device_i32(sizes)
        if self._h:
            capi.tnlb_segments_destroy(self._h)
            self._h = C.c_void_p()
        h = C.c_void_p()
        check(capi.tnlb_segments_create(self.FORMAT, self.organization, d.data_ptr() if d.numel() else None,
                                        d.numel(), _stream(), C.byref(h)))
        self._h = h
        check(capi.tnlb_segments_get_info(self._h, C.byref(self._info)))

    def _adopt(self, handle) -> None:
        """Take ownership of a segments handle built elsewhere (a loaded file)."""
        if self._h:
            capi.tnlb_segments_destroy(self._h)
        self._h = C.c_void_p(handle)
        check(capi.tnlb_segments_get_info(self._h, C.byref(self._info)))
        self.organization = self._info.organization

    def getSegmentCount(self) -> int:
        return self._info.segments

    def getElementCount(self) -> int:
        return self._info.elements

    def getStorageSize(self) -> int:
        return self._info.storage

    @property
    def info(self) -> capi.SegmentsInfo:
        return self._info

    def _meta(self, which: int, count: int) -> np.ndarray:
        out = np.zeros(max(count, 1), dtype=np.int32)
        check(capi.tnlb_segments_read_metadata(self._h, which, out.ctypes.data, out.size))
        return out[:count]

    def getGlobalIndex(self, segment, local) -> np.ndarray:
        s = _device_i32(np.atleast_1d(segment))
        l = _device_i32(np.atleast_1d(local))
        out = torch.empty(s.numel(), dtype=torch.int64, device="cuda")
        check(capi.tnlb_segments_global_index(self._h, s.data_ptr(), l.data_ptr(), s.numel(), out.data_ptr(), _stream()))
        return out.cpu().numpy()


class CSR(_Segments):
    """Algorithms::Segments::CSR."""
    FORMAT = capi.CSR

    def getOffsets(self) -> np.ndarray:
        return self._meta(capi.META_OFFSETS, self._info.segments + 1)


class AdaptiveCSR(CSR):
    """Algorithms::Segments::AdaptiveCSR (CSR offsets + block descriptors)."""
    FORMAT = capi.ADAPTIVE_CSR

    def getBlocks(self, size_log: int) -> np.ndarray:
        cnt = self._info.acsr_blocks[size_log]
        buf = (capi.AcsrBlock * max(cnt, 1))()
        check(capi.tnlb_segments_read_acsr_blocks(self._h, size_log, buf, cnt))
        dt = np.dtype([("type", np.uint8), ("warp_idx", np.uint8), ("warps_count", np.uint8), ("reserved", np.uint8),
                       ("first_segment", np.int32), ("block_size", np.int32), ("segments_in_block", np.int32)])
        return np.frombuffer(bytes(buf), dtype=dt)[:cnt].copy()


class Ellpack(_Segments):
    """Algorithms::Segments::Ellpack (Alignment 32)."""
    FORMAT = capi.ELLPACK

    def getSegmentSize(self) -> int:
        return self._info.segment_size

    def getAlignedSize(self) -> int:
        return self._info.aligned_size


class SlicedEllpack(_Segments):
    """Algorithms::Segments::SlicedEllpack (SliceSize 32)."""
    FORMAT = capi.SLICED_ELLPACK

    def getSliceOffsets(self) -> np.ndarray:
        return self._meta(capi.META_SLICE_OFFSETS, self._info.slices + 1)

    def getSliceSegmentSizes(self) -> np.ndarray:
        return self._meta(capi.META_SLICE_SEGMENT_SIZES, self._info.slices)


class ChunkedEllpack(_Segments):
    """Algorithms::Segments::ChunkedEllpack (256 chunks per slice, desired chunk size 16)."""
    FORMAT = capi.CHUNKED_ELLPACK

    def getNumberOfSlices(self) -> int:
        return self._info.slices

    def getSlices(self) -> dict[str, np.ndarray]:
        ns = self._info.slices
        return {
            "size": self._meta(capi.META_CH_SLICE_SIZE, ns),
            "chunkSize": self._meta(capi.META_CH_SLICE_CHUNK_SIZE, ns),
            "firstSegment": self._meta(capi.META_CH_SLICE_FIRST, ns),
            "pointer": self._meta(capi.META_CH_SLICE_POINTER, ns),
        }

    def getSegmentToChunkMapping(self) -> np.ndarray:
        return self._meta(capi.META_CH_SEGMENT_TO_CHUNK, self._info.segments)

    def getSegmentToSliceMapping(self) -> np.ndarray:
        return self._meta(capi.META_CH_SEGMENT_TO_SLICE, self._info.segments)

    def getSegmentPointers(self) -> np.ndarray:
        return self._meta(capi.META_CH_SEGMENT_POINTERS, self._info.segments + 1)

    def getChunksToSegmentsMapping(self) -> np.ndarray:
        return self._meta(capi.META_CH_CHUNKS_TO_SEGMENTS, self._info.slices * self._info.chunks_in_slice)


class BiEllpack(_Segments):
    """Algorithms::Segments::BiEllpack (strips of 32)."""
    FORMAT = capi.BIELLPACK

    def getSegmentsPermutation(self) -> np.ndarray:
        return self._meta(capi.META_BI_PERMUTATION, self._info.segments)

    def getGroupPointers(self) -> np.ndarray:
        return self._meta(capi.META_BI_GROUP_POINTERS, self._info.slices * 6 + 1)


FORMATS = {c.__name__: c for c in (CSR, Ellpack, SlicedEllpack, ChunkedEllpack, BiEllpack, AdaptiveCSR)}


class SparseMatrix:
    """Matrices::SparseMatrix<Real, Devices::Cuda, int, GeneralMatrix, Segments>.

    ``segments`` is one of the format classes, ``real`` torch.float64 or
    torch.float32.  Values and column indexes are CUDA tensors of length
    getStorageSize(); padding slots hold column -1 and value 0.  With
    ``symmetric=True`` it is SparseMatrix<..., SymmetricMatrix, ...>: one
    triangle is stored and vectorProduct adds the mirrored entries.
    """

    def __init__(self, segments=CSR, real=torch.float64, organization: int | None = None, symmetric: bool = False):
        self.symmetric = bool(symmetric)
        self.segments_cls = segments
        self.real = real
        self.organization = organization
        self.rows = 0
        self.columns = 0
        self.segments = segments(organization)
        self.values = torch.zeros(0, dtype=real, device="cuda")
        self.columnIndexes = torch.zeros(0, dtype=torch.int32, device="cuda")

    # -- construction ------------------------------------------------------
    def setDimensions(self, rows: int, columns: int) -> None:
        if rows < 0 or columns < 0:
            raise ValueError("negative matrix dimensions")
        self.rows, self.columns = int(rows), int(columns)

    def setRowCapacities(self, capacities) -> None:
        """SparseMatrix::setRowCapacities (SparseMatrix.hpp:303-325)."""
        caps = _device_i32(capacities)
        if caps.numel() != self.rows:
            raise ValueError("setRowCapacities: the number of capacities does not match the number of rows")
        self.segments.setSegmentsSizes(caps)
        st = self.segments.getStorageSize()
        self.values = torch.zeros(st, dtype=self.real, device="cuda")
        self.columnIndexes = torch.full((st,), -1, dtype=torch.int32, device="cuda")

    def assign(self, rowptr, cols, vals, columns: int | None = None) -> "SparseMatrix":
        """Cross-format ``operator=`` from a CSR matrix (SparseOperations.hpp:106-186).

        Row capacities are the source row lengths; elements with value 0 or
        column -1 are dropped, the rest packed into each row's slots.
        """
        rp = _device_i32(rowptr)
        n = rp.numel() - 1
        c = _device_i32(cols)
        v = (vals if isinstance(vals, torch.Tensor) else torch.as_tensor(np.ascontiguousarray(vals)))
        v = v.to(device="cuda", dtype=self.real).contiguous()
        self.setDimensions(n, n if columns is None else columns)
        self.setRowCapacities(rp[1:] - rp[:-1])
        check(capi.tnlb_matrix_fill_from_csr(self.segments.handle, _real_code(self.real), rp.data_ptr(),
                                             c.data_ptr() if c.numel() else None, v.data_ptr() if v.numel() else None,
                                             self.columnIndexes.data_ptr() if self.columnIndexes.numel() else None,
                                             self.values.data_ptr() if self.values.numel() else None, _stream()))
        return self

    @classmethod
    def from_csr(cls, A: CSRMatrix, segments=CSR, real=torch.float64, organization: int | None = None,
                 symmetric: bool = False) -> "SparseMatrix":
        M = cls(segments, real, organization, symmetric)
        return M.assign(A.rowptr, A.cols, A.vals, A.ncols)

    # -- queries -------------------------------------------------------------
    def getRows(self) -> int:
        return self.rows

    def getColumns(self) -> int:
        return self.columns

    def getValues(self) -> torch.Tensor:
        return self.values

    def getColumnIndexes(self) -> torch.Tensor:
        return self.columnIndexes

    def getSegments(self):
        return self.segments

    # -- products ------------------------------------------------------------
    def vectorProduct(self, inVector: torch.Tensor, outVector: torch.Tensor, matrixMultiplicator: float = 1.0,
                      outVectorMultiplicator: float = 0.0, begin: int = 0, end: int = 0,
                      launchConfig: LaunchConfiguration | None = None, stream=None, synchronize: bool = True) -> None:
        """outVector = matrixMultiplicator * A * inVector + outVectorMultiplicator * outVector.

        SparseMatrixBase::vectorProduct (SparseMatrixBase.hpp:270-393);
        synchronous on return like the reference unless synchronize=False.
        """
        if inVector.numel() != self.columns:
            raise ValueError("vectorProduct: size of the input vector does not match the number of matrix columns")
        if outVector.numel() != self.rows:
            raise ValueError("vectorProduct: size of the output vector does not match the number of matrix rows")
        if inVector.dtype != self.real or outVector.dtype != self.real:
            raise TypeError("vector real type must match the matrix real type")
        if not (inVector.is_cuda and outVector.is_cuda and inVector.is_contiguous() and outVector.is_contiguous()):
            raise ValueError("vectors must be contiguous CUDA tensors")
        st = _stream(stream)
        if self.symmetric:
            # SparseMatrixBase.hpp:296-330: beta scales y, mirrored entries added atomically
            check(capi.tnlb_spmv_symmetric(self.segments.handle, _real_code(self.real),
                                           self.columnIndexes.data_ptr() if self.columnIndexes.numel() else None,
                                           self.values.data_ptr() if self.values.numel() else None,
                                           inVector.data_ptr() if inVector.numel() else None,
                                           outVector.data_ptr() if outVector.numel() else None,
                                           float(matrixMultiplicator), float(outVectorMultiplicator), int(begin),
                                           int(end), st))
            if synchronize:
                torch.cuda.current_stream().synchronize() if stream is None else stream.synchronize()
            return
        k, tps = (launchConfig or LaunchConfiguration()).kernel()
        check(capi.tnlb_spmv(self.segments.handle, _real_code(self.real),
                             self.columnIndexes.data_ptr() if self.columnIndexes.numel() else None,
                             self.values.data_ptr() if self.values.numel() else None, self.columns,
                             inVector.data_ptr() if inVector.numel() else None,
                             outVector.data_ptr() if outVector.numel() else None,
                             float(matrixMultiplicator), float(outVectorMultiplicator), int(begin), int(end), k, tps, st))
        if synchronize:
            torch.cuda.current_stream().synchronize() if stream is None else stream.synchronize()


    def toHostCSR(self) -> CSRMatrix:
        """The stored elements as host CSR (segment order, padding dropped, FP64 values)."""
        h = capi.HostCSR()
        check(capi.tnlb_matrix_to_host_csr(self.segments.handle, _real_code(self.real),
                                           self.columnIndexes.data_ptr() if self.columnIndexes.numel() else None,
                                           self.values.data_ptr() if self.values.numel() else None, self.columns,
                                           C.byref(h)))
        try:
            return _host_csr_to_numpy(h)
        finally:
            capi.tnlb_host_csr_free(C.byref(h))

    # -- files -----------------------------------------------------------------
    def save(self, fileName) -> None:
        """SparseMatrix::save (SparseMatrix.hpp:632-643): TNL's binary matrix
        file, byte for byte what the reference writes for this matrix."""
        check(capi.tnlb_matrix_save(str(fileName).encode(), self.segments.handle, _real_code(self.real),
                                    self.columnIndexes.data_ptr() if self.columnIndexes.numel() else None,
                                    self.values.data_ptr() if self.values.numel() else None, self.rows,
                                    self.columns, int(self.symmetric)))

    def getSerializationType(self) -> str:
        """The matrix type string of a TNL file (SparseMatrixBase.hpp:46-53)."""
        org = "RowMajorOrder" if self.segments.organization == RowMajorOrder else "ColumnMajorOrder"
        seg = {CSR: "CSR< int >", AdaptiveCSR: "AdaptiveCSR< int >", Ellpack: f"Ellpack< int, {org}, 32 >",
               SlicedEllpack: f"SlicedEllpack< int, {org}, 32 >", ChunkedEllpack: f"ChunkedEllpack< int, {org} >",
               BiEllpack: f"BiEllpack< int, {org}, 32 >"}[self.segments_cls]
        real = "double" if self.real == torch.float64 else "float"
        kind = "Symmetric" if self.symmetric else "General"
        return (f"Matrices::SparseMatrix< {real}, {seg}, [any_device], int, {kind}, [any_allocator], "
                "[any_allocator] >")

    def load(self, fileName) -> "SparseMatrix":
        """SparseMatrix::load (SparseMatrix.hpp:646-694): the file's type must
        be this matrix's type, else the reference's FileDeserializationError
        message is raised (as RuntimeError); the segments come from the
        stored metadata."""
        info = capi.MatrixFileInfo()
        check(capi.tnlb_matrix_file_info_read(str(fileName).encode(), C.byref(info)))
        found, expected = info.type.decode(), self.getSerializationType()
        if found != expected:
            raise RuntimeError(f"{fileName}: object type does not match (expected {expected}, found {found}).")
        cols = torch.empty(max(info.storage, 1), dtype=torch.int32, device="cuda")
        vals = torch.empty(max(info.storage, 1), dtype=self.real, device="cuda")
        h = C.c_void_p()
        check(capi.tnlb_matrix_load(str(fileName).encode(), C.byref(h), cols.data_ptr(), vals.data_ptr(),
                                    max(info.storage, 1)))
        self.segments._adopt(h.value)
        self.rows, self.columns = int(info.rows), int(info.columns)
        self.columnIndexes, self.values = cols[:info.storage], vals[:info.storage]
        return self

    def getTransposition(self, matrixMultiplicator: float = 1.0, segments=None) -> "SparseMatrix":
        """B = matrixMultiplicator * A^T as a new matrix (SparseMatrix::getTransposition,
        SparseMatrix.hpp:495-551), in ``segments`` (default: this matrix's
        format) with this matrix's real type; rows of B in ascending column
        order.  B is filled through the cross-format assignment, so an
        explicitly stored zero of A (or a zero multiplicator) leaves a
        padding slot in B where the reference stores a zero."""
        n_t = self.columns
        trp = torch.zeros(n_t + 1, dtype=torch.int32, device="cuda")
        nnz = C.c_int64()
        cols = self.columnIndexes.data_ptr() if self.columnIndexes.numel() else None
        check(capi.tnlb_matrix_transpose_rowptr(self.segments.handle, cols, n_t, trp.data_ptr(), C.byref(nnz),
                                                _stream()))
        tc = torch.empty(max(nnz.value, 1), dtype=torch.int32, device="cuda")
        tv = torch.empty(max(nnz.value, 1), dtype=self.real, device="cuda")
        check(capi.tnlb_matrix_transpose_fill(self.segments.handle, _real_code(self.real), cols,
                                              self.values.data_ptr() if self.values.numel() else None, n_t,
                                              float(matrixMultiplicator), tc.data_ptr(), tv.data_ptr(), _stream()))
        B = SparseMatrix(segments if segments is not None else self.segments_cls, self.real, self.organization)
        return B.assign(trp, tc[:nnz.value], tv[:nnz.value], self.rows)

    def transposedVectorProduct(self, inVector: torch.Tensor, outVector: torch.Tensor, matrixMultiplicator: float = 1.0,
                            outVectorMultiplicator: float = 0.0, begin: int = 0, end: int = 0, stream=None,
                            synchronize: bool = True) -> None:
        """outVector = matrixMultiplicator * A^T * inVector + outVectorMultiplicator * outVector.

        SparseMatrixBase::transposedVectorProduct (SparseMatrixBase.hpp:542-588);
        a symmetric matrix uses vectorProduct, as the reference does."""
        if inVector.numel() != self.rows:
            raise ValueError("transposedVectorProduct: size of the input vector does not match the number of matrix rows")
        if outVector.numel() != self.columns:
            raise ValueError(
                "transposedVectorProduct: size of the output vector does not match the number of matrix columns")
        if self.symmetric:
            return self.vectorProduct(inVector, outVector, matrixMultiplicator, outVectorMultiplicator, begin, end,
                                      stream=stream, synchronize=synchronize)
        if inVector.dtype != self.real or outVector.dtype != self.real:
            raise TypeError("vector real type must match the matrix real type")
        check(capi.tnlb_spmv_transposed(self.segments.handle, _real_code(self.real),
                                        self.columnIndexes.data_ptr() if self.columnIndexes.numel() else None,
                                        self.values.data_ptr() if self.values.numel() else None, self.columns,
                                        inVector.data_ptr() if inVector.numel() else None,
                                        outVector.data_ptr() if outVector.numel() else None, float(matrixMultiplicator),
                                        float(outVectorMultiplicator), int(begin), int(end), _stream(stream)))
        if synchronize:
            torch.cuda.current_stream().synchronize() if stream is None else stream.synchronize()


def _host_csr_to_numpy(h: "capi.HostCSR") -> CSRMatrix:
    nnz = int(h.nnz)
    rp = np.ctypeslib.as_array(h.rowptr, shape=(h.rows + 1,)).copy()
    cols = np.ctypeslib.as_array(h.cols, shape=(max(nnz, 1),))[:nnz].copy()
    vals = np.ctypeslib.as_array(h.values, shape=(max(nnz, 1),))[:nnz].copy()
    return CSRMatrix(rp, cols, vals, h.columns)


def assemble_laplace_2d(grid_size: int, segments=None, real=torch.float64, organization: int | None = None,
                        capacity: int = 5) -> "SparseMatrix":
    """The 2D Laplace operator of a grid_size x grid_size grid assembled on
    the GPU (identity rows on the boundary, 1, 1, -4, 1, 1 inside), as the
    reference's sparse set-up benchmark builds it with forElements
    (SparseMatrixSetup_Benchmark.cpp): row capacities `capacity` (5 in the
    benchmark), then one thread per row writes its stencil into the
    storage of the chosen format."""
    seg = CSR if segments is None else segments
    n = grid_size * grid_size
    M = SparseMatrix(seg, real, organization)
    M.setDimensions(n, n)
    M.setRowCapacities(torch.full((n,), capacity, dtype=torch.int32, device="cuda"))
    check(capi.tnlb_matrix_assemble_laplace_2d(M.segments.handle, _real_code(real), grid_size,
                                               M.columnIndexes.data_ptr(), M.values.data_ptr(), _stream()))
    return M


def read_mtx(path, symmetric: bool = False) -> CSRMatrix:
    """MatrixReader::readMtx (Matrices/MatrixReader.hpp): a MatrixMarket file as
    host CSR.  ``symmetric=True`` reads into symmetric storage (the lower
    triangle), as for a SymmetricMatrix; RuntimeError carries the reader's
    messages."""
    h = capi.HostCSR()
    check(capi.tnlb_mtx_read(str(path).encode(), int(bool(symmetric)), C.byref(h)))
    try:
        return _host_csr_to_numpy(h)
    finally:
        capi.tnlb_host_csr_free(C.byref(h))


def write_mtx(path, A) -> None:
    """MatrixWriter::writeMtx (Matrices/MatrixWriter.hpp): a CSRMatrix or a
    SparseMatrix written as "coordinate real general"."""
    if isinstance(A, SparseMatrix):
        A = A.toHostCSR()
    rp = np.ascontiguousarray(A.rowptr, np.int32)
    cols = np.ascontiguousarray(A.cols, np.int32)
    vals = np.ascontiguousarray(A.vals, np.float64)
    check(capi.tnlb_mtx_write(str(path).encode(), len(rp) - 1, int(A.ncols), rp.ctypes.data,
                              cols.ctypes.data if cols.size else None, vals.ctypes.data if vals.size else None))


def dot(a: torch.Tensor, b: torch.Tensor) -> torch.Tensor:
    """(a, b) computed by the library into a device scalar (float64)."""
    out = torch.empty(1, dtype=torch.float64, device="cuda")
    check(capi.tnlb_dot(_real_code(a.dtype), a.numel(), a.data_ptr(), b.data_ptr(), out.data_ptr(), _stream()))
    return out


# ----------------------------------------------------------------- solvers

class _Preconditioner:
    KIND = capi.PRECOND_NONE

    def __init__(self):
        self.matrix = None
        self._h = C.c_void_p()

    def __del__(self):
        try:
            if self._h:
                capi.tnlb_precond_destroy(self._h)
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def update(self, matrix: SparseMatrix) -> None:
        """Preconditioner::update (Preconditioners/Preconditioner.h:96-110)."""
        if matrix.getRows() == 0:
            raise ValueError(f"{type(self).__name__}::update: the matrix is empty")
        if matrix.getRows() != matrix.getColumns():
            raise ValueError(f"{type(self).__name__}::update: matrix must be square")
        if self._h:
            capi.tnlb_precond_destroy(self._h)
            self._h = C.c_void_p()
        h = C.c_void_p()
        check(capi.tnlb_precond_create(self.KIND, matrix.segments.handle, _real_code(matrix.real),
                                       matrix.columnIndexes.data_ptr(), matrix.values.data_ptr(), _stream(),
                                       C.byref(h)))
        self._h = h
        self.matrix = matrix

    def solve(self, b: torch.Tensor, x: torch.Tensor) -> None:
        """Preconditioner::solve: x = M^{-1} b."""
        check(capi.tnlb_precond_solve(self._h, b.data_ptr(), x.data_ptr(), _stream()))

    def factor(self, which: int = 0):
        """(rowptr, cols, values) of an FSAI factor: 0 = G (G_L), 1 = the second
        factor as applied (G^T, or G_U)."""
        n = self.matrix.getRows()
        cap = max(self.matrix.getValues().numel(), 32 * n)  # a level-1 FSAI factor outgrows A
        rp = np.zeros(n + 1, np.int32)
        cols = np.zeros(max(cap, 1), np.int32)
        vals = np.zeros(max(cap, 1), np.float64 if self.matrix.real == torch.float64 else np.float32)
        check(capi.tnlb_precond_read_factor(self._h, which, rp.ctypes.data, cols.ctypes.data, vals.ctypes.data, cap))
        return rp, cols[:rp[-1]], vals[:rp[-1]]


class Diagonal(_Preconditioner):
    """Solvers::Linear::Preconditioners::Diagonal (Jacobi)."""
    KIND = capi.PRECOND_JACOBI


class FSAI2(_Preconditioner):
    """Two-factor FSAI for nonsymmetric matrices, M^-1 = G_U G_L (no
    counterpart in the reference)."""
    KIND = capi.PRECOND_FSAI2


class FSAI(_Preconditioner):
    """Factorised sparse approximate inverse M^-1 = G^T G with
    Kolotilina-Yeremin values (no counterpart in the reference); G on the
    lower triangle of A's pattern (``level=0``, the default) or of the
    pattern of A^2 (``level=1``: one level of fill)."""
    KIND = capi.PRECOND_FSAI

    def __init__(self, level: int = 0):
        super().__init__()
        if level not in (0, 1):
            raise ValueError("FSAI: the pattern level must be 0 or 1")
        self.level = level

    def update(self, matrix: SparseMatrix) -> None:
        if self.level == 0:
            return super().update(matrix)
        if matrix.getRows() == 0:
            raise ValueError("FSAI::update: the matrix is empty")
        if matrix.getRows() != matrix.getColumns():
            raise ValueError("FSAI::update: matrix must be square")
        if self._h:
            capi.tnlb_precond_destroy(self._h)
            self._h = C.c_void_p()
        h = C.c_void_p()
        check(capi.tnlb_precond_create_fsai(matrix.segments.handle, _real_code(matrix.real),
                                            matrix.columnIndexes.data_ptr(), matrix.values.data_ptr(), self.level,
                                            _stream(), C.byref(h)))
        self._h = h
        self.matrix = matrix


class ILUT(_Preconditioner):
    """Solvers::Linear::Preconditioners::ILUT (ILUT.hpp:27-258): dual-threshold
    ILU factorised on the host with the reference's arithmetic and selection
    (the reference has no CUDA ILUT), applied on the GPU by the level-
    scheduled triangular solves.  Setup keys "ilut-p" (default 0) and
    "ilut-threshold" (default 1e-4)."""
    KIND = capi.PRECOND_ILUT

    def __init__(self):
        super().__init__()
        self.p = 0
        self.tau = 1e-4

    def setup(self, parameters: dict, prefix: str = "") -> bool:
        if prefix + "ilut-p" in parameters:
            self.p = int(parameters[prefix + "ilut-p"])
        if prefix + "ilut-threshold" in parameters:
            self.tau = float(parameters[prefix + "ilut-threshold"])
        return True

    def update(self, matrix: SparseMatrix) -> None:
        if matrix.getRows() == 0:
            raise ValueError("ILUT::update: the matrix is empty")
        if matrix.getRows() != matrix.getColumns():
            raise ValueError("ILUT::update: matrix must be square")
        if self._h:
            capi.tnlb_precond_destroy(self._h)
            self._h = C.c_void_p()
        h = C.c_void_p()
        check(capi.tnlb_precond_create_ilut(matrix.segments.handle, _real_code(matrix.real),
                                            matrix.columnIndexes.data_ptr(), matrix.values.data_ptr(), self.p,
                                            self.tau, _stream(), C.byref(h)))
        self._h = h
        self.matrix = matrix

    def factors(self):
        """The factors as one CSR (rowptr, cols, values): row i holds its L
        entries (columns < i, unit diagonal implied) then its U entries, the
        first U entry the pivot."""
        n = self.matrix.getRows()
        cap = max(self.matrix.getValues().numel(), 32 * n)  # a level-1 FSAI factor outgrows A * (3 + 2 * self.p) + 2 * n * (self.p + 1) + 16
        rp = np.zeros(n + 1, np.int32)
        cols = np.zeros(cap, np.int32)
        vals = np.zeros(cap, np.float64 if self.matrix.real == torch.float64 else np.float32)
        check(capi.tnlb_precond_read_factor(self._h, 0, rp.ctypes.data, cols.ctypes.data, vals.ctypes.data, cap))
        return rp, cols[:rp[-1]], vals[:rp[-1]]


class ILU0(_Preconditioner):
    """Solvers::Linear::Preconditioners::ILU0 (on the GPU)."""
    KIND = capi.PRECOND_ILU0

    def factors(self):
        """(rowptr, cols, values) of L (strictly lower, unit diagonal implied) and U on A's pattern."""
        M = self.matrix
        n = M.getRows()
        cap = M.getValues().numel()
        rp = np.zeros(n + 1, np.int32)
        cols = np.zeros(max(cap, 1), np.int32)
        vals = np.zeros(max(cap, 1), np.float64 if M.real == torch.float64 else np.float32)
        check(capi.tnlb_ilu0_factors(M.segments.handle, _real_code(M.real), M.columnIndexes.data_ptr(),
                                     M.values.data_ptr(), rp.ctypes.data, cols.ctypes.data, vals.ctypes.data, cap,
                                     _stream()))
        nnz = int(rp[-1])
        return rp, cols[:nnz], vals[:nnz]


class _LinearSolver:
    """LinearSolver + IterativeSolver (Solvers/Linear/LinearSolver.h, Solvers/IterativeSolver.h)."""
    KIND = capi.SOLVER_CG

    def __init__(self):
        self.params = capi.SolverParams()
        capi.tnlb_solver_params_default(C.byref(self.params))
        self.matrix = None
        self.preconditioner = None
        self.iterations = 0
        self.residue = 0.0

    def setMatrix(self, matrix: SparseMatrix) -> None:
        if matrix.getRows() != matrix.getColumns():
            raise ValueError("LinearSolver::setMatrix: matrix must be square")
        self.matrix = matrix

    def setPreconditioner(self, preconditioner) -> None:
        self.preconditioner = preconditioner

    def setConvergenceResidue(self, r: float) -> None:
        self.params.convergence_residue = r

    def setDivergenceResidue(self, r: float) -> None:
        self.params.divergence_residue = r

    def setMaxIterations(self, n: int) -> None:
        self.params.max_iterations = n

    def setMinIterations(self, n: int) -> None:
        self.params.min_iterations = n

    def getIterations(self) -> int:
        return self.iterations

    def getResidue(self) -> float:
        return self.residue

    def setup(self, parameters: dict, prefix: str = "") -> bool:
        """setup(ParameterContainer) with the reference's keys (IterativeSolver.hpp:14-36,
        GMRES.hpp:20-37, BICGStab.hpp:14-21, BICGStabL.hpp:14-33, IDRs.hpp:18-34)."""
        p = self.params
        g = lambda k: parameters.get(prefix + k)  # noqa: E731
        if g("max-iterations") is not None:
            p.max_iterations = int(g("max-iterations"))
        if g("min-iterations") is not None:
            p.min_iterations = int(g("min-iterations"))
        if g("convergence-residue") is not None:
            p.convergence_residue = float(g("convergence-residue"))
        if g("divergence-residue") is not None:
            p.divergence_residue = float(g("divergence-residue"))
        if g("gmres-variant") is not None:
            p.gmres_variant = {"CGS": 0, "CGSR": 1, "MGS": 2, "MGSR": 3, "CWY": 4}[g("gmres-variant")]
        for key, field in (("gmres-restarting-min", "gmres_restarting_min"),
                           ("gmres-restarting-max", "gmres_restarting_max"),
                           ("gmres-restarting-step-min", "gmres_restarting_step_min"),
                           ("gmres-restarting-step-max", "gmres_restarting_step_max")):
            if g(key) is not None:
                setattr(p, field, int(g(key)))
        if g("bicgstab-exact-residue") is not None:
            p.bicgstab_exact_residue = int(bool(g("bicgstab-exact-residue")))
        if g("bicgstab-ell") is not None:
            p.bicgstab_ell = int(g("bicgstab-ell"))
        if g("idr-s") is not None:
            p.idr_s = int(g("idr-s"))
        if g("idr-residual-smoothing") is not None:
            p.idr_residual_smoothing = int(bool(g("idr-residual-smoothing")))
        return True

    def solve(self, b: torch.Tensor, x: torch.Tensor) -> bool:
        """LinearSolver::solve(b, x): x holds the initial guess; returns the convergence flag."""
        M = self.matrix
        if M is None:
            raise RuntimeError("No matrix was set. Call setMatrix() before solve().")
        if b.numel() != M.getRows() or x.numel() != M.getRows():
            raise ValueError("solve: vector sizes do not match the matrix")
        ph = self.preconditioner.handle if self.preconditioner is not None else None
        r = capi.SolveResult()
        check(capi.tnlb_solve_preconditioned(self.KIND, ph, C.byref(self.params), M.segments.handle,
                                             _real_code(M.real), M.columnIndexes.data_ptr(), M.values.data_ptr(),
                                             b.data_ptr(), x.data_ptr(), _stream(), C.byref(r)))
        self.iterations = r.iterations
        self.residue = r.residue
        return bool(r.converged)


class CG(_LinearSolver):
    """Solvers::Linear::CG."""
    KIND = capi.SOLVER_CG


class BICGStab(_LinearSolver):
    """Solvers::Linear::BICGStab."""
    KIND = capi.SOLVER_BICGSTAB


class GMRES(_LinearSolver):
    """Solvers::Linear::GMRES (restarted, left-preconditioned; CGS, CGSR, MGS, MGSR)."""
    KIND = capi.SOLVER_GMRES


class TFQMR(_LinearSolver):
    """Solvers::Linear::TFQMR (left-preconditioned; the stopping residue is
    the quasi-residual bound of TFQMR.hpp:86)."""
    KIND = capi.SOLVER_TFQMR


class BICGStabL(_LinearSolver):
    """Solvers::Linear::BICGStabL: BiCGStab(ell), keys "bicgstab-ell" and
    "bicgstab-exact-residue"."""
    KIND = capi.SOLVER_BICGSTABL


class IDRs(_LinearSolver):
    """Solvers::Linear::IDRs: IDR(s), keys "idr-s" and "idr-residual-smoothing";
    residues are unpreconditioned, as in the reference."""
    KIND = capi.SOLVER_IDRS


class FGMRES(_LinearSolver):
    """Restarted GMRES with right, flexible preconditioning (no counterpart in
    the reference): the stopping residue is the unpreconditioned one."""
    KIND = capi.SOLVER_FGMRES


def true_residual(M: SparseMatrix, b: torch.Tensor, x: torch.Tensor) -> float:
    """||b - A x|| / ||b|| in FP64 on the GPU (Utils/LinearResidueGetter.hpp:11-23)."""
    out = C.c_double()
    check(capi.tnlb_true_residual(M.segments.handle, _real_code(M.real), M.columnIndexes.data_ptr(),
                                  M.values.data_ptr(), b.data_ptr(), x.data_ptr(), _stream(), C.byref(out)))
    return out.value


def solve_mixed_reliable(M: SparseMatrix, b: torch.Tensor, x: torch.Tensor, tol: float = 1e-8, delta: float = 0.3,
                         max_iterations: int = 1000000, inner: str | _Preconditioner = "jacobi",
                         vectors: torch.dtype = torch.float32, layout: str = "auto",
                         operator: str = "excess") -> dict:
    """Mixed-precision PCG with reliable updates (SPD matrices, FP64 matrix
    and vectors): CG iterations on FP32 values (FP32 or FP64 ``vectors``)
    whose correction is folded into the FP64 x, with the residual recomputed
    in FP64, each time the recursive residual has fallen below ``delta``
    times its value at the last update (0.3: the fewest iterations on the
    2048^2 diffusion matrix among 0.02 ... 0.7); the search direction is
    kept across updates.  When the FP32 iteration stalls (the true residual
    no longer halves, or a breakdown) the solve finishes with FP64 Jacobi
    PCG: ``fallback`` and ``fallback_iterations`` in the result.

    ``inner`` is "jacobi", "fsai", "none", or an FP32 Jacobi / FSAI
    preconditioner object built for an FP32 copy of the matrix (e.g. a
    learned FSAI).  Stops on the true FP64 residual ``tol``.

    ``layout`` picks the internal FP32 copies of short-row matrices: "auto"
    stores a matrix with few diagonals by diagonal (the products of FSAI
    factors of more than 5 diagonals staging their operands in shared
    memory by bulk copies), others as CSR with 16-bit column offsets;
    "offsets" always the latter; "diagonal" the diagonal copies read by
    ordinary loads throughout.  All give the same row sums bit for bit
    (their FP64 dot products group rows differently).

    ``operator`` "excess" stores, in the FP32 copy of A, each row's FP64
    sum in place of its diagonal entry and sums a row as
    s_i x_i + sum_j a_ij (x_j - x_i): on high-contrast diffusion operators
    the FP32 copy then keeps the small eigenvalues that FP32 rounding of
    a_ii destroys; "plain" keeps the values as they are.
    """
    if M.real != torch.float64:
        raise TypeError("solve_mixed_reliable takes an FP64 matrix")
    layouts = {"auto": 0, "offsets": 1, "diagonal": 2}
    if layout not in layouts:
        raise ValueError(f"solve_mixed_reliable: unknown layout {layout!r}")
    operators = {"excess": 0, "plain": 1}
    if operator not in operators:
        raise ValueError(f"solve_mixed_reliable: unknown operator form {operator!r}")
    p = capi.SolverParams()
    capi.tnlb_solver_params_default(C.byref(p))
    p.reliable_layout = layouts[layout]
    p.reliable_operator = operators[operator]
    p.convergence_residue = tol
    p.max_iterations = max_iterations
    r = capi.SolveResult()
    upd = C.c_int32()
    kinds = {"none": capi.PRECOND_NONE, "jacobi": capi.PRECOND_JACOBI, "fsai": capi.PRECOND_FSAI}
    if isinstance(inner, str) and inner not in kinds:
        raise ValueError(f"solve_mixed_reliable: unknown preconditioner {inner!r}")
    kind = kinds[inner] if isinstance(inner, str) else capi.PRECOND_NONE
    handle = None if isinstance(inner, str) else inner.handle
    check(capi.tnlb_solve_mixed_reliable(C.byref(p), M.segments.handle, M.columnIndexes.data_ptr(),
                                         M.values.data_ptr(), b.data_ptr(), x.data_ptr(), delta,
                                         _real_code(vectors), kind, handle, _stream(), C.byref(r), C.byref(upd)))
    return {"converged": bool(r.converged), "iterations": r.iterations, "reliable_updates": upd.value,
            "true_residual": r.residue, "fallback": r.status_detail == 2,
            "fallback_iterations": r.fallback_iterations, "stalled": r.status_detail != 0}


def solve_mixed(M: SparseMatrix, b: torch.Tensor, x: torch.Tensor, tol: float = 1e-8, inner_tol: float = 1e-4,
                max_outer: int = 50, max_iterations: int = 1000000000, inner: str | _Preconditioner = "jacobi",
                solver: str = "cg", gmres_restart: int = 30) -> dict:
    """FP32 PCG inside FP64 iterative refinement (SPD matrices, FP64 matrix and vectors).

    ``inner`` is "jacobi", "fsai", "ilu0", "none", or an FP32 preconditioner
    object built for an FP32 copy of the matrix (e.g. a learned FSAI).
    """
    if M.real != torch.float64:
        raise TypeError("solve_mixed takes an FP64 matrix")
    p = capi.SolverParams()
    capi.tnlb_solver_params_default(C.byref(p))
    p.convergence_residue = tol
    p.max_iterations = max_iterations
    p.gmres_restarting_min = p.gmres_restarting_max = gmres_restart
    skind = {"cg": capi.SOLVER_CG, "bicgstab": capi.SOLVER_BICGSTAB, "gmres": capi.SOLVER_GMRES,
             "fgmres": capi.SOLVER_FGMRES}[solver]
    r = capi.SolveResult()
    outer = C.c_int32()
    kinds = {"none": capi.PRECOND_NONE, "jacobi": capi.PRECOND_JACOBI, "ilu0": capi.PRECOND_ILU0,
             "fsai": capi.PRECOND_FSAI, "fsai2": capi.PRECOND_FSAI2}
    kind = kinds.get(inner, capi.PRECOND_JACOBI) if isinstance(inner, str) else capi.PRECOND_NONE
    handle = None if isinstance(inner, str) else inner.handle
    check(capi.tnlb_solve_mixed(C.byref(p), M.segments.handle, M.columnIndexes.data_ptr(), M.values.data_ptr(),
                                b.data_ptr(), x.data_ptr(), inner_tol, max_outer, skind, kind, handle, _stream(),
                                C.byref(r), C.byref(outer)))
    return {"converged": bool(r.converged), "inner_iterations": r.iterations, "outer_iterations": outer.value,
            "true_residual": r.residue}
