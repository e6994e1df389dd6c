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
    "Adaptive", "Default").  ``threadsPerSegmentCount`` must be a positive
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
    getStorageSize(); padding slots hold column -1 and value 0.
    """

    def __init__(self, segments=CSR, real=torch.float64, organization: int | None = None):
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
    def from_csr(cls, A: CSRMatrix, segments=CSR, real=torch.float64, organization: int | None = None) -> "SparseMatrix":
        M = cls(segments, real, organization)
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
        k, tps = (launchConfig or LaunchConfiguration()).kernel()
        st = _stream(stream)
        check(capi.tnlb_spmv(self.segments.handle, _real_code(self.real),
                             self.columnIndexes.data_ptr() if self.columnIndexes.numel() else None,
                             self.values.data_ptr() if self.values.numel() else None, self.columns,
                             inVector.data_ptr() if inVector.numel() else None,
                             outVector.data_ptr() if outVector.numel() else None,
                             float(matrixMultiplicator), float(outVectorMultiplicator), int(begin), int(end), k, tps, st))
        if synchronize:
            torch.cuda.current_stream().synchronize() if stream is None else stream.synchronize()


def dot(a: torch.Tensor, b: torch.Tensor) -> torch.Tensor:
    """(a, b) computed by the library into a device scalar (float64)."""
    out = torch.empty(1, dtype=torch.float64, device="cuda")
    check(capi.tnlb_dot(_real_code(a.dtype), a.numel(), a.data_ptr(), b.data_ptr(), out.data_ptr(), _stream()))
    return out
