"""Python access to the checker libraries -- TEST INFRASTRUCTURE ONLY.

* ``Oracle`` wraps _build/liboracle.so, the plain-C restatement of the
  reference's builders, index maps, fill, SpMV and solvers (tnl_oracle.c).
* ``Reference`` wraps _ref/libtnlref.so, the reference's own Host/OpenMP
  code compiled from its headers (ref_tnl.cpp), when it was built.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use
this module; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "_build" / "liboracle.so"
REF_SO = HERE / "_ref" / "libtnlref.so"
REF_CUDA_SO = HERE / "_ref" / "libtnlref_cuda.so"

CSR, ELLPACK, SLICED_ELLPACK, CHUNKED_ELLPACK, BIELLPACK, ADAPTIVE_CSR = range(6)


def build() -> None:
    """Build the oracle (and the reference driver when its sources are present)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _ptr(a):
    return a.ctypes.data if a is not None else None


class OrcSegments(C.Structure):
    _fields_ = [
        ("kind", C.c_int32), ("colmajor", C.c_int32), ("n", C.c_int32), ("storage", C.c_int32),
        ("offsets", C.c_void_p), ("segmentSize", C.c_int32), ("alignedSize", C.c_int32),
        ("sliceOffsets", C.c_void_p), ("sliceSegmentSizes", C.c_void_p),
        ("chunksInSlice", C.c_int32), ("segmentToChunk", C.c_void_p), ("segmentToSlice", C.c_void_p),
        ("sliceChunkSize", C.c_void_p), ("sliceFirst", C.c_void_p), ("slicePointer", C.c_void_p),
        ("perm", C.c_void_p), ("groupPointers", C.c_void_p),
    ]


class SolverState(C.Structure):
    _fields_ = [
        ("maxIterations", C.c_int32), ("minIterations", C.c_int32), ("convergenceResidue", C.c_double),
        ("divergenceResidue", C.c_double), ("iterations", C.c_int32), ("residue", C.c_double),
        ("history", C.c_void_p), ("historyCap", C.c_int32),
    ]


class Segments:
    """Metadata of one format built by the oracle, plus the C view for index maps."""

    def __init__(self, kind: int, n: int, colmajor: bool, storage: int, **meta):
        self.kind, self.n, self.colmajor, self.storage = kind, n, colmajor, storage
        self.meta = meta
        self._keep = [v for v in meta.values() if isinstance(v, np.ndarray)]

    def cview(self) -> OrcSegments:
        m = self.meta
        s = OrcSegments()
        s.kind = CSR if self.kind == ADAPTIVE_CSR else self.kind
        s.colmajor = int(self.colmajor)
        s.n = self.n
        s.storage = self.storage
        s.offsets = _ptr(m.get("offsets"))
        s.segmentSize = m.get("segmentSize", 0)
        s.alignedSize = m.get("alignedSize", 0)
        s.sliceOffsets = _ptr(m.get("sliceOffsets"))
        s.sliceSegmentSizes = _ptr(m.get("sliceSegmentSizes"))
        s.chunksInSlice = 256
        s.segmentToChunk = _ptr(m.get("segmentToChunk"))
        s.segmentToSlice = _ptr(m.get("segmentToSlice"))
        s.sliceChunkSize = _ptr(m.get("chunkSize"))
        s.sliceFirst = _ptr(m.get("firstSegment"))
        s.slicePointer = _ptr(m.get("pointer"))
        s.perm = _ptr(m.get("perm"))
        s.groupPointers = _ptr(m.get("groupPointers"))
        return s


class Oracle:
    def __init__(self):
        if not ORACLE_SO.exists():
            build()
        L = self.L = C.CDLL(str(ORACLE_SO))
        p, i32, i64, f64 = C.c_void_p, C.c_int32, C.c_int64, C.c_double
        for name, args, res in [
            ("orc_csr_build", [p, i32, p], None),
            ("orc_ellpack_build", [p, i32, C.c_int, p, p], C.c_int),
            ("orc_sell_build", [p, i32, p, p], i64),
            ("orc_chell_slices", [p, i32, i32, i32, p, p, p], i32),
            ("orc_chell_build", [p, i32, i32, i32, i32, p, p, p, p, p, p, p, p, p], C.c_int),
            ("orc_biell_build", [p, i32, p, p], i64),
            ("orc_acsr_blocks", [p, i32, i32, p, p, p, p, p, p], i64),
            ("orc_segment_capacity", [C.POINTER(OrcSegments), i32], i32),
            ("orc_global_index", [C.POINTER(OrcSegments), i32, i32], i64),
            ("orc_fill_f64", [C.POINTER(OrcSegments), p, p, p, p, p], None),
            ("orc_fill_f32", [C.POINTER(OrcSegments), p, p, p, p, p], None),
            ("orc_spmv_f64", [C.POINTER(OrcSegments), p, p, p, p, f64, f64, i32, i32], None),
            ("orc_spmv_f32", [C.POINTER(OrcSegments), p, p, p, p, f64, f64, i32, i32], None),
            ("orc_spmv_symmetric_f64", [C.POINTER(OrcSegments), p, p, p, p, f64, f64, i32, i32], None),
            ("orc_spmv_symmetric_f32", [C.POINTER(OrcSegments), p, p, p, p, f64, f64, i32, i32], None),
            ("orc_spmv_transposed_f64", [C.POINTER(OrcSegments), p, p, i32, p, p, f64, f64, i32, i32], None),
            ("orc_spmv_transposed_f32", [C.POINTER(OrcSegments), p, p, i32, p, p, f64, f64, i32, i32], None),
            ("orc_cg", [i32, p, p, p, C.c_int, p, p, C.POINTER(SolverState)], C.c_int),
            ("orc_bicgstab", [i32, p, p, p, C.c_int, C.c_int, p, p, C.POINTER(SolverState)], C.c_int),
            ("orc_gmres", [i32, p, p, p, C.c_int, i32, C.c_int, p, p, C.POINTER(SolverState)], C.c_int),
            ("orc_fgmres", [i32, p, p, p, C.c_int, i32, C.c_int, p, p, C.POINTER(SolverState)], C.c_int),
            ("orc_gmres_cwy", [i32, p, p, p, C.c_int, i32, p, p, C.POINTER(SolverState)], C.c_int),
            ("orc_tfqmr", [i32, p, p, p, C.c_int, p, p, C.POINTER(SolverState)], C.c_int),
            ("orc_bicgstabl", [i32, p, p, p, C.c_int, C.c_int, C.c_int, p, p, C.POINTER(SolverState)], C.c_int),
            ("orc_idrs", [i32, p, p, p, C.c_int, C.c_int, C.c_int, p, p, p, C.POINTER(SolverState)], C.c_int),
            ("orc_idrs_shadow", [i32, i32, p], None),
            ("orc_true_residual", [i32, p, p, p, p, p], f64),
            ("orc_pcg_reliable", [i32, p, p, p, C.c_int, p, p, f64, f64, i32, C.c_int, C.c_int, p, p, p], C.c_int),
            ("orc_pcg_reliable_fsai", [i32, p, p, p, p, p, p, p, p, p, p, p, f64, f64, i32, C.c_int, C.c_int, p, p, p],
             C.c_int),
            ("orc_ilut_factor", [i32, p, p, p, i32, f64, p, p, p], C.c_long),
            ("orc_lu_apply", [i32, p, p, p, p, p], None),
            ("orc_ilu0_factor", [i32, p, p, p, p, p, p, p, p, p], C.c_int),
            ("orc_prec_apply", [i32, p, p, p, C.c_int, p, p], C.c_int),
        ]:
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res

    # ------------------------------------------------------------ builders
    def build(self, kind: int, sizes, colmajor: bool = True) -> Segments:
        sizes = _i32(sizes)
        n = len(sizes)
        L = self.L
        if kind in (CSR, ADAPTIVE_CSR):
            off = np.zeros(n + 1, np.int32)
            L.orc_csr_build(sizes.ctypes.data, n, off.ctypes.data)
            return Segments(kind, n, colmajor, int(off[-1]), offsets=off)
        if kind == ELLPACK:
            ss, al = C.c_int32(), C.c_int32()
            rc = L.orc_ellpack_build(sizes.ctypes.data, n, int(colmajor), C.byref(ss), C.byref(al))
            if rc == 2:
                raise OverflowError("Ellpack: multiplication overflow")
            return Segments(kind, n, colmajor, ss.value * al.value, segmentSize=ss.value, alignedSize=al.value)
        if kind == SLICED_ELLPACK:
            slices = (n + 31) // 32
            so = np.zeros(slices + 1, np.int32)
            sw = np.zeros(max(slices, 1), np.int32)
            st = L.orc_sell_build(sizes.ctypes.data, n, so.ctypes.data, sw.ctypes.data)
            if st < 0:
                raise OverflowError("SlicedEllpack storage overflow")
            return Segments(kind, n, colmajor, int(st), sliceOffsets=so, sliceSegmentSizes=sw[:slices])
        if kind == CHUNKED_ELLPACK:
            ns = L.orc_chell_slices(sizes.ctypes.data, n, 256, 16, None, None, None)
            a = {k: np.zeros(max(ns, 1), np.int32) for k in ("size", "chunkSize", "firstSegment", "pointer")}
            s2c = np.zeros(max(n, 1), np.int32)
            s2s = np.zeros(max(n, 1), np.int32)
            sp = np.zeros(n + 1, np.int32)
            c2s = np.zeros(max(ns * 256, 1), np.int32)
            st = C.c_int32()
            rc = L.orc_chell_build(sizes.ctypes.data, n, 256, 16, ns, a["size"].ctypes.data, a["chunkSize"].ctypes.data,
                                   a["firstSegment"].ctypes.data, a["pointer"].ctypes.data, s2c.ctypes.data,
                                   s2s.ctypes.data, sp.ctypes.data, c2s.ctypes.data, C.byref(st))
            if rc != 0:
                raise OverflowError("ChunkedEllpack build failed")
            meta = {k: v[:ns] for k, v in a.items()}
            return Segments(kind, n, colmajor, st.value, segmentToChunk=s2c[:n], segmentToSlice=s2s[:n],
                            segmentPointers=sp, chunksToSegments=c2s[:ns * 256], numberOfSlices=ns, **meta)
        if kind == BIELLPACK:
            strips = (n + 31) // 32
            perm = np.zeros(max(n, 1), np.int32)
            gp = np.zeros(strips * 6 + 1, np.int32)
            st = L.orc_biell_build(sizes.ctypes.data, n, perm.ctypes.data, gp.ctypes.data)
            if st < 0:
                raise OverflowError("BiEllpack storage overflow")
            return Segments(kind, n, colmajor, int(st), perm=perm[:n], groupPointers=gp)
        raise ValueError(kind)

    def acsr_blocks(self, offsets, size_log: int) -> np.ndarray:
        off = _i32(offsets)
        n = len(off) - 1
        cnt = self.L.orc_acsr_blocks(off.ctypes.data, n, 1 << size_log, None, None, None, None, None, None)
        t = np.zeros(max(cnt, 1), np.uint8)
        f = np.zeros(max(cnt, 1), np.int32)
        bs = np.zeros(max(cnt, 1), np.int32)
        sib = np.zeros(max(cnt, 1), np.int32)
        wi = np.zeros(max(cnt, 1), np.uint8)
        wc = np.zeros(max(cnt, 1), np.uint8)
        self.L.orc_acsr_blocks(off.ctypes.data, n, 1 << size_log, t.ctypes.data, f.ctypes.data, bs.ctypes.data,
                               sib.ctypes.data, wi.ctypes.data, wc.ctypes.data)
        return {"type": t[:cnt], "first": f[:cnt], "blockSize": bs[:cnt], "segmentsInBlock": sib[:cnt],
                "warpIdx": wi[:cnt], "warpsCount": wc[:cnt]}

    # --------------------------------------------------------- index maps
    def global_index(self, seg: Segments, segment: int, local: int) -> int:
        v = seg.cview()
        return self.L.orc_global_index(C.byref(v), segment, local)

    def capacity(self, seg: Segments, segment: int) -> int:
        v = seg.cview()
        return self.L.orc_segment_capacity(C.byref(v), segment)

    def fill(self, seg: Segments, rowptr, cols, vals):
        rowptr, cols = _i32(rowptr), _i32(cols)
        vals = np.ascontiguousarray(vals)
        oc = np.zeros(max(seg.storage, 1), np.int32)
        ov = np.zeros(max(seg.storage, 1), vals.dtype)
        v = seg.cview()
        f = self.L.orc_fill_f64 if vals.dtype == np.float64 else self.L.orc_fill_f32
        f(C.byref(v), rowptr.ctypes.data, cols.ctypes.data, vals.ctypes.data, oc.ctypes.data, ov.ctypes.data)
        return oc[:seg.storage], ov[:seg.storage]

    def spmv(self, seg: Segments, cols, vals, x, y=None, alpha=1.0, beta=0.0, begin=0, end=0):
        cols = _i32(cols)
        vals = np.ascontiguousarray(vals)
        x = np.ascontiguousarray(x, dtype=vals.dtype)
        y = np.zeros(seg.n, vals.dtype) if y is None else np.array(y, dtype=vals.dtype, copy=True)
        v = seg.cview()
        f = self.L.orc_spmv_f64 if vals.dtype == np.float64 else self.L.orc_spmv_f32
        f(C.byref(v), cols.ctypes.data, vals.ctypes.data, x.ctypes.data, y.ctypes.data, alpha, beta, begin, end)
        return y

    def spmv_symmetric(self, seg: Segments, cols, vals, x, y=None, alpha=1.0, beta=0.0, begin=0, end=0):
        """vectorProduct of a symmetric matrix stored as one triangle."""
        cols = _i32(cols)
        vals = np.ascontiguousarray(vals)
        x = np.ascontiguousarray(x, dtype=vals.dtype)
        y = np.zeros(seg.n, vals.dtype) if y is None else np.array(y, dtype=vals.dtype, copy=True)
        v = seg.cview()
        f = self.L.orc_spmv_symmetric_f64 if vals.dtype == np.float64 else self.L.orc_spmv_symmetric_f32
        f(C.byref(v), cols.ctypes.data, vals.ctypes.data, x.ctypes.data, y.ctypes.data, alpha, beta, begin, end)
        return y

    def spmv_transposed(self, seg: Segments, cols, vals, columns: int, x, y=None, alpha=1.0, beta=0.0, begin=0,
                        end=0):
        """transposedVectorProduct: y (length `columns`) = alpha A^T x + beta y."""
        cols = _i32(cols)
        vals = np.ascontiguousarray(vals)
        x = np.ascontiguousarray(x, dtype=vals.dtype)
        y = np.zeros(columns, vals.dtype) if y is None else np.array(y, dtype=vals.dtype, copy=True)
        v = seg.cview()
        f = self.L.orc_spmv_transposed_f64 if vals.dtype == np.float64 else self.L.orc_spmv_transposed_f32
        f(C.byref(v), cols.ctypes.data, vals.ctypes.data, columns, x.ctypes.data, y.ctypes.data, alpha, beta, begin,
          end)
        return y

    # ------------------------------------------------------------ solvers
    def _state(self, tol, maxit, history):
        S = SolverState()
        S.maxIterations = maxit
        S.minIterations = 0
        S.convergenceResidue = tol
        S.divergenceResidue = np.finfo(np.float64).max
        hist = np.zeros(history, np.float64) if history else None
        S.history = hist.ctypes.data if hist is not None else None
        S.historyCap = history
        return S, hist

    def idrs_shadow(self, n: int, s: int) -> np.ndarray:
        """The IDR(s) shadow space (n x s, column-major) as the reference draws it."""
        P = np.zeros(n * s)
        self.L.orc_idrs_shadow(n, s, P.ctypes.data)
        return P

    def solve(self, solver: str, A, b, x0=None, precond: int = 1, tol=1e-8, maxit=100000, gmres_m=30,
              gmres_reorth=2, bicgstab_exact=False, history=0, ell=1, idr_s=4, idr_smoothing=False):
        rowptr, cols, vals = _i32(A.rowptr), _i32(A.cols), np.ascontiguousarray(A.vals, np.float64)
        b = np.ascontiguousarray(b, np.float64)
        x = np.zeros(A.n) if x0 is None else np.array(x0, np.float64, copy=True)
        S, hist = self._state(tol, maxit, history)
        args = (A.n, rowptr.ctypes.data, cols.ctypes.data, vals.ctypes.data)
        if solver == "cg":
            ok = self.L.orc_cg(*args, precond, b.ctypes.data, x.ctypes.data, C.byref(S))
        elif solver == "bicgstab":
            ok = self.L.orc_bicgstab(*args, precond, int(bicgstab_exact), b.ctypes.data, x.ctypes.data, C.byref(S))
        elif solver == "gmres":
            ok = self.L.orc_gmres(*args, precond, gmres_m, gmres_reorth, b.ctypes.data, x.ctypes.data, C.byref(S))
        elif solver == "tfqmr":
            ok = self.L.orc_tfqmr(*args, precond, b.ctypes.data, x.ctypes.data, C.byref(S))
        elif solver == "bicgstabl":
            ok = self.L.orc_bicgstabl(*args, precond, ell, int(bicgstab_exact), b.ctypes.data, x.ctypes.data,
                                      C.byref(S))
        elif solver == "idrs":
            P = self.idrs_shadow(A.n, idr_s)
            ok = self.L.orc_idrs(*args, precond, idr_s, int(idr_smoothing), P.ctypes.data, b.ctypes.data,
                                 x.ctypes.data, C.byref(S))
        elif solver == "gmres_cwy":
            ok = self.L.orc_gmres_cwy(*args, precond, gmres_m, b.ctypes.data, x.ctypes.data, C.byref(S))
        elif solver == "fgmres":
            ok = self.L.orc_fgmres(*args, precond, gmres_m, gmres_reorth, b.ctypes.data, x.ctypes.data, C.byref(S))
        else:
            raise ValueError(solver)
        return {"x": x, "converged": ok == 1, "status": ok, "iterations": S.iterations, "residue": S.residue,
                "history": hist}

    def ilut_factor(self, A, p=0, tau=1e-4):
        """The ILUT factors (ILUT.hpp:27-258 restated) as one CSR: row i holds
        its L entries then its U entries.  Returns (rowptr, cols, vals)."""
        rowptr, cols, vals = _i32(A.rowptr), _i32(A.cols), np.ascontiguousarray(A.vals, np.float64)
        nnz = self.L.orc_ilut_factor(A.n, rowptr.ctypes.data, cols.ctypes.data, vals.ctypes.data, p, tau, None, None,
                                     None)
        frp = np.zeros(A.n + 1, np.int32)
        fc = np.zeros(max(nnz, 1), np.int32)
        fv = np.zeros(max(nnz, 1), np.float64)
        self.L.orc_ilut_factor(A.n, rowptr.ctypes.data, cols.ctypes.data, vals.ctypes.data, p, tau, frp.ctypes.data,
                               fc.ctypes.data, fv.ctypes.data)
        return frp, fc[:nnz], fv[:nnz]

    def lu_apply(self, frp, fc, fv, b):
        """x = U^-1 L^-1 b for factors in the layout of ilut_factor."""
        frp, fc = _i32(frp), _i32(fc)
        fv = np.ascontiguousarray(fv, np.float64)
        b = np.ascontiguousarray(b, np.float64)
        x = np.zeros(len(frp) - 1)
        self.L.orc_lu_apply(len(frp) - 1, frp.ctypes.data, fc.ctypes.data, fv.ctypes.data, b.ctypes.data,
                            x.ctypes.data)
        return x

    @staticmethod
    def transpose(A, mult=1.0, real=np.float64):
        """getTransposition (Matrices/SparseMatrix.hpp:495-551) restated:
        the entries of A stably sorted by column, so each row of B = mult * A^T
        holds its entries in ascending column order (the reference's
        single-threaded order); values multiplied by mult in `real`.
        Returns (rowptr, cols, vals) with ncols rows."""
        rowptr, cols = np.asarray(A.rowptr, np.int64), np.asarray(A.cols, np.int64)
        rows = np.repeat(np.arange(A.n, dtype=np.int64), np.diff(rowptr))
        keep = cols != -1
        rows, cols, vals = rows[keep], cols[keep], np.asarray(A.vals, real)[keep]
        order = np.argsort(cols, kind="stable")
        trp = np.zeros(A.ncols + 1, np.int64)
        np.add.at(trp, cols + 1, 1)
        return (np.cumsum(trp).astype(np.int32), rows[order].astype(np.int32),
                (vals[order] * real(mult)).astype(real))

    def pcg_reliable(self, A, b, precond: int = 1, tol=1e-8, delta=0.1, maxit=100000, x0=None, vec64=False,
                     excess=None):
        """The library's mixed-precision PCG with reliable updates (FP32
        values, FP32 or FP64 vectors, FP64 updates); precond 0 none, 1 Jacobi.
        ``excess`` (default: with FP32 vectors, as the library's compact
        copies do) sums the FP32 product in the row-excess form."""
        if excess is None:
            excess = not vec64
        rowptr, cols, vals = _i32(A.rowptr), _i32(A.cols), np.ascontiguousarray(A.vals, np.float64)
        b = np.ascontiguousarray(b, np.float64)
        x = np.zeros(A.n) if x0 is None else np.array(x0, np.float64, copy=True)
        it, upd, res = C.c_int32(), C.c_int32(), C.c_double()
        ok = self.L.orc_pcg_reliable(A.n, rowptr.ctypes.data, cols.ctypes.data, vals.ctypes.data, precond,
                                     b.ctypes.data, x.ctypes.data, tol, delta, maxit, int(vec64), int(excess),
                                     C.byref(it), C.byref(upd), C.byref(res))
        return {"x": x, "converged": ok == 1, "stalled": ok == 2, "iterations": it.value, "updates": upd.value,
                "residue": res.value}

    def pcg_reliable_fsai(self, A, b, G, GT, tol=1e-8, delta=0.1, maxit=100000, vec64=False, excess=None):
        """pcg_reliable with the FSAI preconditioner z = G^T (G r): G and GT
        are (rowptr, cols, FP32 values) of the factor and of its transpose
        in the entry order the solver applies them."""
        if excess is None:
            excess = not vec64
        rowptr, cols, vals = _i32(A.rowptr), _i32(A.cols), np.ascontiguousarray(A.vals, np.float64)
        grp, gc, gv = _i32(G[0]), _i32(G[1]), np.ascontiguousarray(G[2], np.float32)
        trp, tc, tv = _i32(GT[0]), _i32(GT[1]), np.ascontiguousarray(GT[2], np.float32)
        b = np.ascontiguousarray(b, np.float64)
        x = np.zeros(A.n)
        it, upd, res = C.c_int32(), C.c_int32(), C.c_double()
        ok = self.L.orc_pcg_reliable_fsai(A.n, rowptr.ctypes.data, cols.ctypes.data, vals.ctypes.data,
                                          grp.ctypes.data, gc.ctypes.data, gv.ctypes.data, trp.ctypes.data,
                                          tc.ctypes.data, tv.ctypes.data, b.ctypes.data, x.ctypes.data, tol, delta,
                                          maxit, int(vec64), int(excess), C.byref(it), C.byref(upd), C.byref(res))
        return {"x": x, "converged": ok == 1, "iterations": it.value, "updates": upd.value, "residue": res.value}

    def true_residual(self, A, b, x) -> float:
        rowptr, cols, vals = _i32(A.rowptr), _i32(A.cols), np.ascontiguousarray(A.vals, np.float64)
        b = np.ascontiguousarray(b, np.float64)
        x = np.ascontiguousarray(x, np.float64)
        return self.L.orc_true_residual(A.n, rowptr.ctypes.data, cols.ctypes.data, vals.ctypes.data, b.ctypes.data,
                                        x.ctypes.data)

    def ilu0(self, A):
        n, nnz = A.n, A.nnz
        rowptr, cols, vals = _i32(A.rowptr), _i32(A.cols), np.ascontiguousarray(A.vals, np.float64)
        Lp, Up = np.zeros(n + 1, np.int32), np.zeros(n + 1, np.int32)
        Lc, Uc = np.zeros(nnz, np.int32), np.zeros(nnz, np.int32)
        Lv, Uv = np.zeros(nnz), np.zeros(nnz)
        self.L.orc_ilu0_factor(n, rowptr.ctypes.data, cols.ctypes.data, vals.ctypes.data, Lp.ctypes.data,
                               Lc.ctypes.data, Lv.ctypes.data, Up.ctypes.data, Uc.ctypes.data, Uv.ctypes.data)
        return Lp, Lc[:Lp[-1]], Lv[:Lp[-1]], Up, Uc[:Up[-1]], Uv[:Up[-1]]

    def prec_apply(self, A, kind: int, b):
        rowptr, cols, vals = _i32(A.rowptr), _i32(A.cols), np.ascontiguousarray(A.vals, np.float64)
        b = np.ascontiguousarray(b, np.float64)
        x = np.zeros(A.n)
        self.L.orc_prec_apply(A.n, rowptr.ctypes.data, cols.ctypes.data, vals.ctypes.data, kind, b.ctypes.data,
                              x.ctypes.data)
        return x


class Reference:
    """The reference's own Host code (oracle/_ref/libtnlref.so), when built."""

    def __init__(self, threads: int | None = None):
        if not REF_SO.exists():
            raise FileNotFoundError(f"{REF_SO} not built (needs the reference sources)")
        if threads is not None:
            os.environ["OMP_NUM_THREADS"] = str(threads)
        L = self.L = C.CDLL(str(REF_SO))
        p, i32, f64 = C.c_void_p, C.c_int, C.c_double
        for name, args, res in [
            ("ref_csr_build", [p, i32, p], C.c_int),
            ("ref_ellpack_build", [p, i32, i32, p, p], C.c_int),
            ("ref_sell_build", [p, i32, p, p], C.c_long),
            ("ref_chell_build", [p, i32, p, p, p, p, p, p, p, p, p], C.c_int),
            ("ref_biell_build", [p, i32, p, p], C.c_long),
            ("ref_acsr_blocks", [p, i32, i32, p, p, p, p, p, p], C.c_long),
            ("ref_fill_f64", [i32, i32, i32, i32, p, p, p, p, p], C.c_long),
            ("ref_fill_f32", [i32, i32, i32, i32, p, p, p, p, p], C.c_long),
            ("ref_spmv_f64", [i32, i32, i32, i32, p, p, p, p, p, f64, f64, i32, i32, i32], f64),
            ("ref_spmv_f32", [i32, i32, i32, i32, p, p, p, p, p, f64, f64, i32, i32, i32], f64),
            ("ref_solve", [i32, i32, i32, p, p, p, p, p, f64, i32, i32, i32, i32, p, p, p], C.c_int),
            ("ref_solve_ext", [i32, i32, i32, p, p, p, p, p, f64, i32, i32, i32, p, p, p], C.c_int),
            ("ref_spmv_symmetric_f64", [i32, p, p, p, p, p, f64, f64, i32, i32], None),
            ("ref_mtx_read", [C.c_char_p, i32, p, p, p, p, p, p, C.c_char_p, i32], C.c_int),
            ("ref_mtx_write", [C.c_char_p, i32, i32, p, p, p], None),
            ("ref_spmv_transposed_f64", [i32, i32, p, p, p, p, p, f64, f64, i32, i32], None),
            ("ref_transpose_f64", [i32, i32, p, p, p, f64, p, p, p], C.c_long),
            ("ref_save", [C.c_int, C.c_int, C.c_int, i32, i32, p, p, p, C.c_char_p], C.c_int),
            ("ref_ilut_factor", [i32, p, p, p, i32, f64, C.POINTER(C.c_long), C.POINTER(C.c_long), p, p, p, p, p, p],
             C.c_int),
            ("ref_ilut_apply", [i32, p, p, p, i32, f64, p, p], C.c_int),
            ("ref_set_ilut", [i32, f64], None),
            ("ref_prec_apply", [i32, p, p, p, i32, p, p], C.c_int),
            ("ref_omp_threads", [], C.c_int),
            ("ref_set_threads", [C.c_int], None),
        ]:
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res

    def threads(self) -> int:
        return self.L.ref_omp_threads()

    def set_threads(self, n: int) -> None:
        self.L.ref_set_threads(n)

    def build(self, kind: int, sizes) -> dict:
        """Metadata of the reference's Host builders (column-major where it matters)."""
        sizes = _i32(sizes)
        n = len(sizes)
        L = self.L
        if kind in (CSR, ADAPTIVE_CSR):
            off = np.zeros(n + 1, np.int32)
            L.ref_csr_build(sizes.ctypes.data, n, off.ctypes.data)
            return {"offsets": off}
        if kind == ELLPACK:
            ss, al = C.c_int(), C.c_int()
            rc = L.ref_ellpack_build(sizes.ctypes.data, n, 1, C.byref(ss), C.byref(al))
            if rc == 2:
                raise OverflowError("Ellpack: multiplication overflow")
            return {"segmentSize": ss.value, "alignedSize": al.value}
        if kind == SLICED_ELLPACK:
            slices = (n + 31) // 32
            so = np.zeros(slices + 1, np.int32)
            sw = np.zeros(max(slices, 1), np.int32)
            st = L.ref_sell_build(sizes.ctypes.data, n, so.ctypes.data, sw.ctypes.data)
            return {"sliceOffsets": so, "sliceSegmentSizes": sw[:slices], "storage": st}
        if kind == CHUNKED_ELLPACK:
            ns = L.ref_chell_build(sizes.ctypes.data, n, *([None] * 9))
            a = {k: np.zeros(max(ns, 1), np.int32) for k in ("size", "chunkSize", "firstSegment", "pointer")}
            s2c = np.zeros(max(n, 1), np.int32)
            s2s = np.zeros(max(n, 1), np.int32)
            sp = np.zeros(n + 1, np.int32)
            c2s = np.zeros(max(ns * 256, 1), np.int32)
            st = C.c_int()
            L.ref_chell_build(sizes.ctypes.data, n, a["size"].ctypes.data, a["chunkSize"].ctypes.data,
                              a["firstSegment"].ctypes.data, a["pointer"].ctypes.data, s2c.ctypes.data,
                              s2s.ctypes.data, sp.ctypes.data, c2s.ctypes.data, C.byref(st))
            out = {k: v[:ns] for k, v in a.items()}
            out.update(segmentToChunk=s2c[:n], segmentToSlice=s2s[:n], segmentPointers=sp,
                       chunksToSegments=c2s[:ns * 256], storage=st.value, numberOfSlices=ns)
            return out
        if kind == BIELLPACK:
            strips = (n + 31) // 32
            perm = np.zeros(max(n, 1), np.int32)
            gp = np.zeros(strips * 6 + 1, np.int32)
            st = L.ref_biell_build(sizes.ctypes.data, n, perm.ctypes.data, gp.ctypes.data)
            return {"perm": perm[:n], "groupPointers": gp, "storage": st}
        raise ValueError(kind)

    def acsr_blocks(self, sizes, size_log: int) -> dict:
        sizes = _i32(sizes)
        n = len(sizes)
        cnt = self.L.ref_acsr_blocks(sizes.ctypes.data, n, size_log, None, None, None, None, None, None)
        if cnt < 0:
            return None  # needs a GPU backend (LONG blocks)
        t = np.zeros(max(cnt, 1), np.uint8)
        f = np.zeros(max(cnt, 1), np.int32)
        bs = np.zeros(max(cnt, 1), np.int32)
        sib = np.zeros(max(cnt, 1), np.int32)
        wi = np.zeros(max(cnt, 1), np.uint8)
        wc = np.zeros(max(cnt, 1), np.uint8)
        self.L.ref_acsr_blocks(sizes.ctypes.data, n, size_log, t.ctypes.data, f.ctypes.data, bs.ctypes.data,
                               sib.ctypes.data, wi.ctypes.data, wc.ctypes.data)
        return {"type": t[:cnt], "first": f[:cnt], "blockSize": bs[:cnt], "segmentsInBlock": sib[:cnt],
                "warpIdx": wi[:cnt], "warpsCount": wc[:cnt]}

    def fill(self, kind: int, A, real=np.float64, colmajor: bool = True):
        rowptr, cols = _i32(A.rowptr), _i32(A.cols)
        vals = np.ascontiguousarray(A.vals, dtype=real)
        f = self.L.ref_fill_f64 if real == np.float64 else self.L.ref_fill_f32
        st = f(kind, int(colmajor), A.n, A.ncols, rowptr.ctypes.data, cols.ctypes.data, vals.ctypes.data, None, None)
        if st == -2:
            raise OverflowError("Ellpack: multiplication overflow")
        oc = np.zeros(max(st, 1), np.int32)
        ov = np.zeros(max(st, 1), real)
        f(kind, int(colmajor), A.n, A.ncols, rowptr.ctypes.data, cols.ctypes.data, vals.ctypes.data, oc.ctypes.data,
          ov.ctypes.data)
        return oc[:st], ov[:st]

    def spmv(self, kind: int, A, x, y=None, alpha=1.0, beta=0.0, begin=0, end=0, reps=1, real=np.float64,
             colmajor: bool = False):
        """Returns (y, best seconds of `reps` calls)."""
        rowptr, cols = _i32(A.rowptr), _i32(A.cols)
        vals = np.ascontiguousarray(A.vals, dtype=real)
        x = np.ascontiguousarray(x, dtype=real)
        y = np.zeros(A.n, real) if y is None else np.array(y, dtype=real, copy=True)
        f = self.L.ref_spmv_f64 if real == np.float64 else self.L.ref_spmv_f32
        t = f(kind, int(colmajor), A.n, A.ncols, rowptr.ctypes.data, cols.ctypes.data, vals.ctypes.data, x.ctypes.data,
              y.ctypes.data, alpha, beta, begin, end, reps)
        return y, t

    def mtx_read(self, path, symmetric: bool = False):
        """The reference's MatrixReader::readMtx: (rows, columns, rowptr, cols, vals) or RuntimeError."""
        rows, columns, nnz = C.c_int(), C.c_int(), C.c_long()
        err = C.create_string_buffer(512)
        p = str(path).encode()
        if self.L.ref_mtx_read(p, int(symmetric), C.byref(rows), C.byref(columns), C.byref(nnz), None, None, None,
                               err, 512):
            raise RuntimeError(err.value.decode())
        rp = np.zeros(rows.value + 1, np.int32)
        cols = np.zeros(max(nnz.value, 1), np.int32)
        vals = np.zeros(max(nnz.value, 1))
        self.L.ref_mtx_read(p, int(symmetric), C.byref(rows), C.byref(columns), C.byref(nnz), rp.ctypes.data,
                            cols.ctypes.data, vals.ctypes.data, err, 512)
        return rows.value, columns.value, rp, cols[:nnz.value], vals[:nnz.value]

    def mtx_write(self, path, A):
        rowptr, cols = _i32(A.rowptr), _i32(A.cols)
        vals = np.ascontiguousarray(A.vals, np.float64)
        self.L.ref_mtx_write(str(path).encode(), A.n, A.ncols, rowptr.ctypes.data, cols.ctypes.data, vals.ctypes.data)

    def spmv_symmetric(self, A, x, y=None, alpha=1.0, beta=0.0, begin=0, end=0):
        """The reference's vectorProduct of a SymmetricMatrix CSR matrix (A holds one triangle)."""
        rowptr, cols = _i32(A.rowptr), _i32(A.cols)
        vals = np.ascontiguousarray(A.vals, np.float64)
        x = np.ascontiguousarray(x, np.float64)
        y = np.zeros(A.n) if y is None else np.array(y, np.float64, copy=True)
        self.L.ref_spmv_symmetric_f64(A.n, rowptr.ctypes.data, cols.ctypes.data, vals.ctypes.data, x.ctypes.data,
                                      y.ctypes.data, alpha, beta, begin, end)
        return y

    def spmv_transposed(self, A, x, y=None, alpha=1.0, beta=0.0, begin=0, end=0):
        """The reference's transposedVectorProduct of a general CSR matrix."""
        rowptr, cols = _i32(A.rowptr), _i32(A.cols)
        vals = np.ascontiguousarray(A.vals, np.float64)
        x = np.ascontiguousarray(x, np.float64)
        y = np.zeros(A.ncols) if y is None else np.array(y, np.float64, copy=True)
        self.L.ref_spmv_transposed_f64(A.n, A.ncols, rowptr.ctypes.data, cols.ctypes.data, vals.ctypes.data,
                                       x.ctypes.data, y.ctypes.data, alpha, beta, begin, end)
        return y

    def ilut_factor(self, A, p=0, tau=1e-4):
        """The reference's ILUT::update: (L rowptr, cols, vals), (U rowptr,
        cols, vals) with their padding; U's rows stored reversed."""
        rowptr, cols = _i32(A.rowptr), _i32(A.cols)
        vals = np.ascontiguousarray(A.vals, np.float64)
        ln, un = C.c_long(), C.c_long()
        args = (A.n, rowptr.ctypes.data, cols.ctypes.data, vals.ctypes.data, p, tau, C.byref(ln), C.byref(un))
        if self.L.ref_ilut_factor(*args, None, None, None, None, None, None) != 0:
            raise RuntimeError("reference ILUT failed")
        lrp, urp = np.zeros(A.n + 1, np.int32), np.zeros(A.n + 1, np.int32)
        lc, uc = np.zeros(max(ln.value, 1), np.int32), np.zeros(max(un.value, 1), np.int32)
        lv, uv = np.zeros(max(ln.value, 1)), np.zeros(max(un.value, 1))
        self.L.ref_ilut_factor(*args, lrp.ctypes.data, lc.ctypes.data, lv.ctypes.data, urp.ctypes.data,
                               uc.ctypes.data, uv.ctypes.data)
        return (lrp, lc[:ln.value], lv[:ln.value]), (urp, uc[:un.value], uv[:un.value])

    def ilut_apply(self, A, b, p=0, tau=1e-4):
        rowptr, cols = _i32(A.rowptr), _i32(A.cols)
        vals = np.ascontiguousarray(A.vals, np.float64)
        b = np.ascontiguousarray(b, np.float64)
        x = np.zeros(A.n)
        if self.L.ref_ilut_apply(A.n, rowptr.ctypes.data, cols.ctypes.data, vals.ctypes.data, p, tau, b.ctypes.data,
                                 x.ctypes.data) != 0:
            raise RuntimeError("reference ILUT failed")
        return x

    def save(self, fmt: int, A, path, colmajor=True, real64=True) -> None:
        """The reference's SparseMatrix::save of A in format `fmt` (built by
        its cross-format operator= from CSR)."""
        rowptr, cols = _i32(A.rowptr), _i32(A.cols)
        vals = np.ascontiguousarray(A.vals, np.float64)
        rc = self.L.ref_save(fmt, int(colmajor), int(real64), A.n, A.ncols, rowptr.ctypes.data, cols.ctypes.data,
                             vals.ctypes.data, str(path).encode())
        if rc != 0:
            raise RuntimeError("reference save failed")

    def transpose(self, A, mult=1.0):
        """The reference's getTransposition of a general CSR matrix into CSR:
        (rowptr, cols, vals) of mult * A^T, padding included."""
        rowptr, cols = _i32(A.rowptr), _i32(A.cols)
        vals = np.ascontiguousarray(A.vals, np.float64)
        size = self.L.ref_transpose_f64(A.n, A.ncols, rowptr.ctypes.data, cols.ctypes.data, vals.ctypes.data, mult,
                                        None, None, None)
        trp = np.zeros(A.ncols + 1, np.int32)
        tc = np.zeros(max(size, 1), np.int32)
        tv = np.zeros(max(size, 1), np.float64)
        self.L.ref_transpose_f64(A.n, A.ncols, rowptr.ctypes.data, cols.ctypes.data, vals.ctypes.data, mult,
                                 trp.ctypes.data, tc.ctypes.data, tv.ctypes.data)
        return trp, tc[:size], tv[:size]

    def solve(self, solver: str, A, b, x0=None, precond: int = 1, tol=1e-8, maxit=100000, gmres_m=30,
              gmres_variant: int = 3, bicgstab_exact=False, ell=1, idr_s=4, idr_smoothing=False):
        rowptr, cols, vals = _i32(A.rowptr), _i32(A.cols), np.ascontiguousarray(A.vals, np.float64)
        b = np.ascontiguousarray(b, np.float64)
        x = np.zeros(A.n) if x0 is None else np.array(x0, np.float64, copy=True)
        it, res, sec = C.c_int(), C.c_double(), C.c_double()
        if solver in ("tfqmr", "bicgstabl", "idrs"):
            kind = {"tfqmr": 3, "bicgstabl": 4, "idrs": 5}[solver]
            param = ell if solver == "bicgstabl" else idr_s
            flag = int(bicgstab_exact) if solver == "bicgstabl" else int(idr_smoothing)
            ok = self.L.ref_solve_ext(kind, precond, A.n, rowptr.ctypes.data, cols.ctypes.data, vals.ctypes.data,
                                      b.ctypes.data, x.ctypes.data, tol, maxit, param, flag, C.byref(it),
                                      C.byref(res), C.byref(sec))
            return {"x": x, "converged": ok == 1, "status": ok, "iterations": it.value, "residue": res.value,
                    "seconds": sec.value}
        kind = {"cg": 0, "bicgstab": 1, "gmres": 2}[solver]
        ok = self.L.ref_solve(kind, precond, A.n, rowptr.ctypes.data, cols.ctypes.data, vals.ctypes.data, b.ctypes.data,
                              x.ctypes.data, tol, maxit, gmres_m, gmres_variant, int(bicgstab_exact), C.byref(it),
                              C.byref(res), C.byref(sec))
        return {"x": x, "converged": ok == 1, "iterations": it.value, "residue": res.value, "seconds": sec.value}

    def prec_apply(self, A, kind: int, b):
        rowptr, cols, vals = _i32(A.rowptr), _i32(A.cols), np.ascontiguousarray(A.vals, np.float64)
        b = np.ascontiguousarray(b, np.float64)
        x = np.zeros(A.n)
        self.L.ref_prec_apply(A.n, rowptr.ctypes.data, cols.ctypes.data, vals.ctypes.data, kind, b.ctypes.data,
                              x.ctypes.data)
        return x


class ReferenceCuda:
    """The reference's own CUDA vectorProduct (oracle/_ref/libtnlref_cuda.so,
    TNL's Devices::Cuda backend compiled for sm_100a), for the secondary GPU
    comparison.  Needs a GPU."""

    def __init__(self):
        if not REF_CUDA_SO.exists():
            raise FileNotFoundError(f"{REF_CUDA_SO} not built (needs the reference sources)")
        L = self.L = C.CDLL(str(REF_CUDA_SO))
        p, i32 = C.c_void_p, C.c_int
        L.ref_cuda_spmv.argtypes = [i32, i32, i32, i32, p, p, p, p, p, i32, C.POINTER(C.c_double),
                                    C.POINTER(C.c_double), C.c_char_p, i32, p, i32, C.c_char_p, i32]
        L.ref_cuda_spmv.restype = C.c_int

    def spmv(self, fmt: int, A, x, real=np.float64, reps: int = 20) -> dict:
        """y = A x by the reference's CUDA vectorProduct (fmt 0: CSR, 2:
        column-major SlicedEllpack); mean ms per synchronous call under the
        default launch configuration and under each of the reference's
        reductionLaunchConfigurations."""
        rowptr, cols = _i32(A.rowptr), _i32(A.cols)
        vals = np.ascontiguousarray(A.vals, real)
        x = np.ascontiguousarray(x, real)
        y = np.zeros(A.n, real)
        md, mb = C.c_double(), C.c_double()
        name = C.create_string_buffer(64)
        err = C.create_string_buffer(512)
        allms = np.zeros(32)
        k = self.L.ref_cuda_spmv(fmt, int(real == np.float64), A.n, A.ncols, rowptr.ctypes.data, cols.ctypes.data,
                                 vals.ctypes.data, x.ctypes.data, y.ctypes.data, reps, C.byref(md), C.byref(mb), name,
                                 64, allms.ctypes.data, 32, err, 512)
        if k < 0:
            raise RuntimeError(err.value.decode())
        return {"y": y, "ms_default": md.value, "ms_best": mb.value, "best": name.value.decode(),
                "ms_all": allms[:k].tolist()}
