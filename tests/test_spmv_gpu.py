"""GPU parity of the segment builders, the matrix fill and SpMV.

Everything is called through the C ABI (tnl_b200 is a ctypes layer over
libtnlb200.so) and compared with the oracle restatement and the golden
fixtures produced by the reference:
  * builder metadata and AdaptiveCSR descriptors: bit-exact;
  * cross-format fill (column indexes, values): bit-exact;
  * SpMV: |y - y_ref| <= rtol * max(|y_ref|, sum_j |alpha a_ij x_j| + |beta y0_i|)
    with rtol = 1e-13 (FP64) and 2e-5 (FP32); the known answers exactly.
"""
import hashlib

import numpy as np
import pytest
import torch

from helpers import FORMATS, assert_spmv_close, row_abs_sums
from known_answers import cases as known_cases

pytestmark = pytest.mark.gpu

ORGS = {"col": 0, "row": 1}
RTOL = {np.float64: 1e-13, np.float32: 2e-5}


def tnl():
    import tnl_b200

    return tnl_b200


def gpu_segments(fmt, sizes, org="col"):
    t = tnl()
    s = t.FORMATS[fmt](ORGS[org])
    s.setSegmentsSizes(np.asarray(sizes, np.int32))
    return s


def oracle_segments(oracle, fmt, sizes, org="col"):
    return oracle.build(FORMATS[fmt], np.asarray(sizes, np.int32), colmajor=(org == "col"))


def gpu_meta(s, fmt):
    if fmt in ("CSR", "AdaptiveCSR"):
        return {"offsets": s.getOffsets()}
    if fmt == "Ellpack":
        return {"segmentSize": s.getSegmentSize(), "alignedSize": s.getAlignedSize()}
    if fmt == "SlicedEllpack":
        return {"sliceOffsets": s.getSliceOffsets(), "sliceSegmentSizes": s.getSliceSegmentSizes()}
    if fmt == "ChunkedEllpack":
        m = s.getSlices()
        m.update(segmentToChunk=s.getSegmentToChunkMapping(), segmentToSlice=s.getSegmentToSliceMapping(),
                 segmentPointers=s.getSegmentPointers(), chunksToSegments=s.getChunksToSegmentsMapping(),
                 numberOfSlices=s.getNumberOfSlices())
        return m
    if fmt == "BiEllpack":
        return {"perm": s.getSegmentsPermutation(), "groupPointers": s.getGroupPointers()}
    raise ValueError(fmt)


def size_vectors(golden):
    from tnl_b200 import generators as g

    out = {c: golden.get(f"sizes/{c}") for c in golden.size_cases()}
    rng = np.random.default_rng(99)
    out["zipf_100k"] = g.zipf_lengths(100_000, 1.73, 4096, 21)
    out["zipf15_50k"] = g.zipf_lengths(50_000, 1.5, 4096, 22)
    out["mixed_zero_rows"] = np.where(rng.random(20_000) < 0.4, 0, rng.integers(0, 2000, 20_000)).astype(np.int32)
    out["n31"] = rng.integers(0, 40, 31).astype(np.int32)
    out["n65"] = rng.integers(0, 40, 65).astype(np.int32)
    return out


@pytest.mark.parametrize("fmt", ["CSR", "Ellpack", "SlicedEllpack", "ChunkedEllpack", "BiEllpack"])
def test_builder_metadata_bit_exact(oracle, golden, fmt):
    for name, sizes in size_vectors(golden).items():
        if fmt == "ChunkedEllpack" and len(sizes) == 0:
            continue
        o = oracle_segments(oracle, fmt, sizes)
        s = gpu_segments(fmt, sizes)
        assert s.getStorageSize() == o.storage, (name, fmt)
        assert s.getSegmentCount() == len(sizes)
        assert s.getElementCount() == int(np.sum(sizes, dtype=np.int64))
        m = gpu_meta(s, fmt)
        for k, v in m.items():
            assert np.array_equal(np.asarray(v), np.asarray(o.meta[k])), (name, fmt, k)
        # and against the reference's own output where the fixture has it
        prefix = f"build/{name}/{fmt}/"
        for key in golden.arrays.files:
            if key.startswith(prefix):
                assert np.array_equal(np.asarray(m[key[len(prefix):]]), golden.get(key)), (name, fmt, key)


def test_adaptive_csr_descriptors_bit_exact(oracle, golden):
    for name, sizes in size_vectors(golden).items():
        s = gpu_segments("AdaptiveCSR", sizes)
        off = np.zeros(len(sizes) + 1, np.int32)
        off[1:] = np.cumsum(sizes)
        for sl in range(6):
            b = s.getBlocks(sl)
            o = oracle.acsr_blocks(off, sl)
            assert len(b) == len(o["type"]), (name, sl)
            assert np.array_equal(b["type"], o["type"]), (name, sl)
            assert np.array_equal(b["first_segment"], o["first"]), (name, sl)
            assert np.array_equal(b["warp_idx"], o["warpIdx"]), (name, sl)
            nonlong = o["type"] != 0
            nonlong[-1:] = False
            assert np.array_equal(b["block_size"][nonlong], o["blockSize"][nonlong]), (name, sl)
            assert np.array_equal(b["segments_in_block"][nonlong], o["segmentsInBlock"][nonlong]), (name, sl)
            wc = (o["type"] == 0)
            assert np.array_equal(b["warps_count"][wc], o["warpsCount"][wc]), (name, sl)
            if golden.meta["acsr"].get(f"{name}/{sl}") not in (None, "unavailable"):
                assert np.array_equal(b["type"], golden.get(f"acsr/{name}/{sl}/type")), (name, sl)
                assert np.array_equal(b["first_segment"], golden.get(f"acsr/{name}/{sl}/first")), (name, sl)


def test_global_index_matches_oracle(oracle):
    from tnl_b200 import generators as g

    sizes = g.zipf_lengths(3000, 1.6, 600, 5)
    rng = np.random.default_rng(3)
    for fmt in ("CSR", "Ellpack", "SlicedEllpack", "ChunkedEllpack", "BiEllpack"):
        for org in ("col", "row"):
            o = oracle_segments(oracle, fmt, sizes, org)
            s = gpu_segments(fmt, sizes, org)
            segs = rng.integers(0, len(sizes), 2000).astype(np.int32)
            locs = np.array([rng.integers(0, max(1, oracle.capacity(o, int(r)))) for r in segs], np.int32)
            got = s.getGlobalIndex(segs, locs)
            exp = np.array([oracle.global_index(o, int(r), int(l)) for r, l in zip(segs, locs)])
            ok = np.array([l < oracle.capacity(o, int(r)) for r, l in zip(segs, locs)])
            assert np.array_equal(got[ok], exp[ok]), (fmt, org)


def _digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("fmt", list(FORMATS))
@pytest.mark.parametrize("org", ["col", "row"])
def test_fill_bit_exact(oracle, golden, fmt, org):
    t = tnl()
    for mname in ("powerlaw2000", "laplacian32"):
        rp = golden.get(f"mat/{mname}/rowptr")
        cols = golden.get(f"mat/{mname}/cols")
        vals = golden.get(f"mat/{mname}/vals")
        for real, tdt in ((np.float64, torch.float64), (np.float32, torch.float32)):
            M = t.SparseMatrix(t.FORMATS[fmt], tdt, ORGS[org]).assign(rp, cols, vals.astype(real))
            gc = M.getColumnIndexes().cpu().numpy()
            gv = M.getValues().cpu().numpy()
            ref = golden.meta["fill"][f"{mname}/{fmt}/{org}/{np.dtype(real).name}"]
            assert len(gc) == ref["storage"]
            assert _digest(gc) == ref["cols"] and _digest(gv) == ref["vals"], (mname, fmt, org, real)


def kernel_variants(fmt, org):
    t = tnl()
    L = t.LaunchConfiguration
    if fmt == "CSR":
        return [L("Default"), L("Tile"), L("Scalar"), L("Light"), L("Adaptive")] + [L("Fixed", k) for k in (2, 4, 8, 16, 32)] + [
            L("Block", k) for k in (64, 128, 256)]
    if fmt == "AdaptiveCSR":
        return [L("Default"), L("Adaptive"), L("Light"), L("Fixed", 8)]
    if fmt == "Ellpack" and org == "row":
        return [L("Default")] + [L("Fixed", k) for k in (1, 2, 8, 32)]
    if fmt == "SlicedEllpack":
        return [L("Default")] + [L("Fixed", k) for k in ((1, 2, 4, 8) if org == "col" else (1, 4, 32))]
    return [L("Default")]


@pytest.mark.parametrize("fmt", list(FORMATS))
@pytest.mark.parametrize("org", ["col", "row"])
def test_known_answers_gpu(fmt, org):
    t = tnl()
    for name, rp, c, v, nc, x, y0, expected in known_cases():
        M = t.SparseMatrix(t.FORMATS[fmt], torch.float64, ORGS[org]).assign(rp, c, v, nc)
        for lc in kernel_variants(fmt, org):
            xs = torch.tensor(x, device="cuda")
            ys = torch.tensor(y0, device="cuda")
            M.vectorProduct(xs, ys, launchConfig=lc)
            assert np.array_equal(ys.cpu().numpy(), expected), (name, fmt, org, lc.mapping, lc.tps)


def matrices():
    from tnl_b200 import generators as g

    rng = np.random.default_rng(5)
    A = g.power_law(20000, 1.73, 4096, 31)
    B = g.laplacian_2d(64)
    # rows of every length class, a third of them empty
    lens = np.where(rng.random(6000) < 0.33, 0, g.zipf_lengths(6000, 1.3, 5000, 9))
    rp = np.zeros(6001, np.int64)
    rp[1:] = np.cumsum(lens)
    cols = g.distinct_sorted_columns(rp, 6000, 8)
    C = g.CSRMatrix(rp.astype(np.int32), cols, g.uniform_vector(int(rp[-1]), 4))
    return {"powerlaw20k": A, "laplacian64": B, "empty_rows": C}


@pytest.fixture(scope="module")
def mats():
    return matrices()


@pytest.mark.parametrize("fmt", list(FORMATS))
@pytest.mark.parametrize("org", ["col", "row"])
@pytest.mark.parametrize("real", [np.float64, np.float32])
def test_spmv_parity(oracle, mats, fmt, org, real):
    t = tnl()
    tdt = torch.float64 if real == np.float64 else torch.float32
    from tnl_b200 import generators as g

    for mname, A in mats.items():
        vals = A.vals.astype(real)
        M = t.SparseMatrix(t.FORMATS[fmt], tdt, ORGS[org]).assign(A.rowptr, A.cols, vals, A.ncols)
        seg = oracle.build(FORMATS["CSR"], A.row_lengths())
        x = g.uniform_vector(A.ncols, 0).astype(real)
        y0 = g.uniform_vector(A.n, 9).astype(real)
        absum = row_abs_sums(A.rowptr, A.cols, vals, x)
        for alpha, beta, begin, end in ((1.0, 0.0, 0, 0), (-2.5, 0.0, 0, 0), (1.0, 0.5, 0, 0), (0.75, -1.25, 0, 0),
                                        (1.0, 0.0, A.n // 3, 2 * A.n // 3)):
            yref = oracle.spmv(seg, A.cols, vals, x, y0, alpha, beta, begin, end)
            scale = abs(alpha) * absum + abs(beta) * np.abs(y0.astype(np.float64))
            for lc in kernel_variants(fmt, org):
                xs = torch.tensor(x, device="cuda")
                ys = torch.tensor(y0, device="cuda")
                M.vectorProduct(xs, ys, alpha, beta, begin, end, launchConfig=lc)
                y = ys.cpu().numpy()
                assert_spmv_close(y, yref, scale, RTOL[real])
                if end:
                    assert np.array_equal(y[:begin], y0[:begin]) and np.array_equal(y[end:], y0[end:])


def test_spmv_beta_zero_ignores_nan_in_y():
    """beta == 0 must not read y (SparseMatrixBase.hpp:346-365)."""
    t = tnl()
    from tnl_b200 import generators as g

    A = g.power_law(5000, 1.73, 1000, 3)
    for fmt in FORMATS:
        M = t.SparseMatrix(t.FORMATS[fmt], torch.float64).assign(A.rowptr, A.cols, A.vals)
        x = torch.tensor(g.uniform_vector(A.n, 0), device="cuda")
        y = torch.full((A.n,), float("nan"), dtype=torch.float64, device="cuda")
        M.vectorProduct(x, y)
        assert torch.isfinite(y).all(), fmt


def test_full_size_powerlaw_csr_against_oracle(oracle):
    """The benchmark matrix (4,194,304 rows, Zipf 1.73, cap 4096): every CSR
    kernel against the oracle's sequential per-row sums, FP64 and FP32."""
    t = tnl()
    from tnl_b200 import generators as g

    A = g.power_law(4_194_304, 1.73, 4096, 2)
    x = g.uniform_vector(A.n, 0)
    seg = oracle.build(FORMATS["CSR"], A.row_lengths())
    for real, tdt in ((np.float64, torch.float64), (np.float32, torch.float32)):
        vals = A.vals.astype(real)
        xr = x.astype(real)
        yref = oracle.spmv(seg, A.cols, vals, xr)
        scale = row_abs_sums(A.rowptr, A.cols, vals, xr)
        M = t.SparseMatrix(t.CSR, tdt).assign(A.rowptr, A.cols, vals)
        xs = torch.tensor(xr, device="cuda")
        for lc in (t.LaunchConfiguration("Default"), t.LaunchConfiguration("Light"), t.LaunchConfiguration("Fixed", 32)):
            ys = torch.empty(A.n, dtype=tdt, device="cuda")
            M.vectorProduct(xs, ys, launchConfig=lc)
            assert_spmv_close(ys.cpu().numpy(), yref, scale, RTOL[real])


def test_full_size_powerlaw_ellpack_overflows():
    """Ellpack storage 4096 x 4,194,304 exceeds int32: std::overflow_error."""
    t = tnl()
    from tnl_b200 import generators as g

    lens = g.zipf_lengths(4_194_304, 1.73, 4096, 2)
    s = t.Ellpack()
    with pytest.raises(OverflowError):
        s.setSegmentsSizes(lens)


def test_size_mismatch_raises():
    t = tnl()
    from tnl_b200 import generators as g

    A = g.laplacian_2d(8)
    M = t.SparseMatrix(t.CSR, torch.float64).assign(A.rowptr, A.cols, A.vals)
    with pytest.raises(ValueError):
        M.vectorProduct(torch.zeros(A.n + 1, dtype=torch.float64, device="cuda"),
                        torch.zeros(A.n, dtype=torch.float64, device="cuda"))
    with pytest.raises(ValueError):
        M.vectorProduct(torch.zeros(A.n, dtype=torch.float64, device="cuda"),
                        torch.zeros(A.n - 1, dtype=torch.float64, device="cuda"))


def test_empty_matrix():
    t = tnl()
    for fmt in FORMATS:
        if fmt == "ChunkedEllpack":
            continue
        M = t.SparseMatrix(t.FORMATS[fmt], torch.float64).assign(np.zeros(1, np.int32), np.zeros(0, np.int32),
                                                                  np.zeros(0))
        M.vectorProduct(torch.zeros(0, dtype=torch.float64, device="cuda"),
                        torch.zeros(0, dtype=torch.float64, device="cuda"))


def test_dot():
    t = tnl()
    a = torch.randn(1_000_003, dtype=torch.float64, device="cuda")
    b = torch.randn(1_000_003, dtype=torch.float64, device="cuda")
    d = t.dot(a, b).item()
    assert d == pytest.approx(float((a * b).sum().item()), rel=1e-12, abs=1e-9)


def _lower_triangle(A):
    from tnl_b200 import generators as g

    rows = np.repeat(np.arange(A.n), np.diff(A.rowptr))
    keep = np.asarray(A.cols) <= rows
    lens = np.bincount(rows[keep], minlength=A.n)
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    return g.CSRMatrix(rp, A.cols[keep], A.vals[keep], A.ncols)


@pytest.mark.parametrize("fmt", list(FORMATS))
@pytest.mark.parametrize("org", ["col", "row"])
@pytest.mark.parametrize("real", [np.float64, np.float32])
def test_symmetric_and_transposed_products(oracle, mats, fmt, org, real):
    """vectorProduct of a symmetric matrix (one triangle stored) and
    transposedVectorProduct, every format, against the oracle (pinned to the
    reference): the GPU adds the scattered terms atomically, so only the
    order of the additions differs -- the same bound as the SpMV parity test,
    with the scale taken over the terms each output entry receives."""
    t = tnl()
    tdt = torch.float64 if real == np.float64 else torch.float32
    from tnl_b200 import generators as g

    for mname, A in mats.items():
        if mname == "laplacian64":
            S = _lower_triangle(A)
            vals = S.vals.astype(real)
            M = t.SparseMatrix(t.FORMATS[fmt], tdt, ORGS[org], symmetric=True).assign(S.rowptr, S.cols, vals, S.ncols)
            seg = oracle.build(FORMATS["CSR"], S.row_lengths())
            x = g.uniform_vector(S.n, 0).astype(real)
            y0 = g.uniform_vector(S.n, 9).astype(real)
            # scale: the full (mirrored) matrix's row sums of |a x|
            absum = row_abs_sums(A.rowptr, A.cols, A.vals.astype(real), x)
            for alpha, beta, begin, end in ((1.0, 0.0, 0, 0), (0.75, -1.25, 0, 0), (1.0, 1.0, S.n // 3, 2 * S.n // 3)):
                yref = oracle.spmv_symmetric(seg, S.cols, vals, x, y0, alpha, beta, begin, end)
                xs, ys = torch.tensor(x, device="cuda"), torch.tensor(y0, device="cuda")
                M.vectorProduct(xs, ys, alpha, beta, begin, end)
                assert_spmv_close(ys.cpu().numpy(), yref, abs(alpha) * absum + abs(beta) * np.abs(y0), RTOL[real])
        vals = A.vals.astype(real)
        M = t.SparseMatrix(t.FORMATS[fmt], tdt, ORGS[org]).assign(A.rowptr, A.cols, vals, A.ncols)
        seg = oracle.build(FORMATS["CSR"], A.row_lengths())
        x = g.uniform_vector(A.n, 4).astype(real)
        y0 = g.uniform_vector(A.ncols, 5).astype(real)
        # scale per output column: sum over rows of |a_rc x_r|
        import scipy.sparse as sp

        absT = np.abs(sp.csr_matrix((np.abs(vals.astype(np.float64)), A.cols, A.rowptr), shape=(A.n, A.ncols)).T
                      @ np.abs(x.astype(np.float64)))
        for alpha, beta, begin, end in ((1.0, 0.0, 0, 0), (-2.5, 0.5, 0, 0), (1.0, 1.0, A.ncols // 4, A.ncols // 2)):
            yref = oracle.spmv_transposed(seg, A.cols, vals, A.ncols, x, y0, alpha, beta, begin, end)
            xs, ys = torch.tensor(x, device="cuda"), torch.tensor(y0, device="cuda")
            M.transposedVectorProduct(xs, ys, alpha, beta, begin, end)
            assert_spmv_close(ys.cpu().numpy(), yref, abs(alpha) * absT + abs(beta) * np.abs(y0), RTOL[real])


@pytest.mark.parametrize("fmt", list(FORMATS))
@pytest.mark.parametrize("real", [np.float64, np.float32])
def test_transposition(oracle, mats, fmt, real):
    """getTransposition from every format: B's stored entries (host CSR
    export) equal the oracle's stable-sorted transposition bit for bit --
    row pointer, columns in ascending order, values times the multiplicator
    in the matrix's real type -- and B's product equals A's transposed
    product."""
    t = tnl()
    tdt = torch.float64 if real == np.float64 else torch.float32
    from tnl_b200 import generators as g

    for mname, A in mats.items():
        vals = A.vals.astype(real)
        M = t.SparseMatrix(t.FORMATS[fmt], tdt).assign(A.rowptr, A.cols, vals, A.ncols)
        for mult in (1.0, -2.5):
            B = M.getTransposition(mult, segments=t.CSR)
            assert B.getRows() == A.ncols and B.getColumns() == A.n
            h = B.toHostCSR()
            from tnl_b200.generators import CSRMatrix

            trp, tc, tv = oracle.transpose(CSRMatrix(A.rowptr, A.cols, vals, A.ncols), mult, real)
            assert np.array_equal(h.rowptr, trp), mname
            assert np.array_equal(h.cols, tc), mname
            assert np.array_equal(h.vals.astype(real), tv), mname
        # the same format as A, and its product against A^T x
        B = M.getTransposition(1.0)
        x = torch.tensor(g.uniform_vector(A.n, 4).astype(real), device="cuda")
        y1 = torch.zeros(A.ncols, dtype=tdt, device="cuda")
        y2 = torch.zeros(A.ncols, dtype=tdt, device="cuda")
        B.vectorProduct(x, y1)
        M.transposedVectorProduct(x, y2)
        tol = 1e-12 if real == np.float64 else 1e-4
        assert torch.allclose(y1, y2, rtol=tol, atol=tol * float(y2.abs().max())), mname
