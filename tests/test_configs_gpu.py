"""GPU parity at the full sizes of the benchmark configurations.

The other GPU tests check every kernel on matrices of at most some 20,000
rows; the speeds are quoted on these matrices, so they are checked here at
their full sizes, through the C ABI, against the oracle and against results
of the reference itself (tests/golden/config_golden.json, made by
tests/golden/make_config_golden.py from the reference's Host code):

* SpMV of every format (and the CSR kernel variants) on the 1024^2
  Laplacian (n = 1,048,576) and the 256^3 GRF diffusion operator
  (n = 16,777,216, 117M nonzeros), FP64 at 1e-13 and FP32 at 2e-5 per row
  (the rule of assert_spmv_close);
* CSR on the power-law matrix with Zipf 1.5 row lengths (n = 4,194,304,
  about 2.06e8 nonzeros);
* builder metadata at full size: CSR, SlicedEllpack and BiEllpack equal the
  reference's arrays bit for bit (SHA-256), ChunkedEllpack its storage
  size, AdaptiveCSR the oracle's descriptors; where the reference's int32
  storage count wraps around (ChunkedEllpack at Zipf 1.73, SlicedEllpack
  at Zipf 1.5) the GPU builder raises OverflowError;
* Jacobi-CG on the 1024^2 Laplacian to 1e-8 within 2 iterations of the
  reference's count, with its true residual;
* mixed-precision solves against a tightly converged FP64 solution: the
  256^3 diffusion problem to 1e-10 and the 2048^2 learned-preconditioner
  evaluation problem to 1e-8; the error of the mixed solution may not
  exceed four times the error of plain FP64 PCG stopped at the same true
  residual.
"""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest
import torch

from helpers import FORMATS, assert_spmv_close

pytestmark = pytest.mark.gpu

GOLDEN = json.loads((Path(__file__).resolve().parent / "golden" / "config_golden.json").read_text())
RTOL = {np.float64: 1e-13, np.float32: 2e-5}


def tnl():
    import tnl_b200

    return tnl_b200


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _gen():
    from tnl_b200 import generators as g

    return g


@pytest.fixture(scope="module")
def laplacian():
    return _gen().laplacian_2d(1024)


@pytest.fixture(scope="module")
def diffusion():
    return _gen().diffusion_3d(256)


def _variants(fmt):
    t = tnl()
    L = t.LaunchConfiguration
    if fmt == "CSR":
        return [("col", L("Default")), ("col", L("Tile")), ("col", L("Light")), ("col", L("Scalar")),
                ("col", L("Fixed", 8))]
    if fmt == "AdaptiveCSR":
        return [("col", L("Adaptive"))]
    if fmt in ("Ellpack", "SlicedEllpack"):
        return [("col", L("Default")), ("row", L("Default"))]
    return [("col", L("Default"))]


def _every_format_against_oracle(oracle, A, real):
    t = tnl()
    g = _gen()
    tdt = torch.float64 if real == np.float64 else torch.float32
    vals = A.vals.astype(real)
    x = g.uniform_vector(A.ncols, 0).astype(real)
    seg = oracle.build(FORMATS["CSR"], A.row_lengths())
    yref = oracle.spmv(seg, A.cols, vals, x)
    scale = oracle.spmv(seg, A.cols, np.abs(A.vals), np.abs(x.astype(np.float64)))
    xs = torch.tensor(x, device="cuda")
    for fmt in FORMATS:
        for org, lc in _variants(fmt):
            M = t.SparseMatrix(t.FORMATS[fmt], tdt, t.RowMajorOrder if org == "row" else t.ColumnMajorOrder)
            M.assign(A.rowptr, A.cols, vals, A.ncols)
            ys = torch.full((A.n,), float("nan"), dtype=tdt, device="cuda")
            M.vectorProduct(xs, ys, launchConfig=lc)
            assert_spmv_close(ys.cpu().numpy(), yref, scale, RTOL[real])
            del M, ys
            torch.cuda.empty_cache()


@pytest.mark.parametrize("real", [np.float64, np.float32])
def test_laplacian_1024_every_format_against_oracle(oracle, laplacian, real):
    _every_format_against_oracle(oracle, laplacian, real)


@pytest.mark.parametrize("real", [np.float64, np.float32])
def test_diffusion_256cubed_every_format_against_oracle(oracle, diffusion, real):
    _every_format_against_oracle(oracle, diffusion, real)


def test_laplacian_1024_alpha_beta_against_oracle(oracle, laplacian):
    """y = alpha A x + beta y with both multiplicators through the default
    (short-row) kernel and SlicedEllpack at full size."""
    t = tnl()
    g = _gen()
    A = laplacian
    x = g.uniform_vector(A.n, 0)
    y0 = g.uniform_vector(A.n, 9)
    seg = oracle.build(FORMATS["CSR"], A.row_lengths())
    yref = oracle.spmv(seg, A.cols, A.vals, x, y0, -0.75, 1.5)
    scale = 0.75 * oracle.spmv(seg, A.cols, np.abs(A.vals), np.abs(x)) + 1.5 * np.abs(y0)
    for fmt in ("CSR", "SlicedEllpack"):
        M = t.SparseMatrix(t.FORMATS[fmt], torch.float64).assign(A.rowptr, A.cols, A.vals)
        ys = torch.tensor(y0, device="cuda")
        M.vectorProduct(torch.tensor(x, device="cuda"), ys, -0.75, 1.5)
        assert_spmv_close(ys.cpu().numpy(), yref, scale, 1e-13)


def test_powerlaw_zipf15_csr_against_oracle(oracle):
    """The literal Zipf exponent 1.5 (cap 4096, mean about 49 nonzeros per
    row, 2.06e8 nonzeros): the default CSR kernel against the oracle, FP64."""
    t = tnl()
    g = _gen()
    A = g.power_law(4_194_304, 1.5, 4096, 2)
    assert A.nnz > 2.0e8
    x = g.uniform_vector(A.ncols, 0)
    seg = oracle.build(FORMATS["CSR"], A.row_lengths())
    yref = oracle.spmv(seg, A.cols, A.vals, x)
    scale = oracle.spmv(seg, A.cols, np.abs(A.vals), np.abs(x))
    M = t.SparseMatrix(t.CSR, torch.float64).assign(A.rowptr, A.cols, A.vals)
    ys = torch.empty(A.n, dtype=torch.float64, device="cuda")
    M.vectorProduct(torch.tensor(x, device="cuda"), ys)
    assert_spmv_close(ys.cpu().numpy(), yref, scale, 1e-13)


def _config_sizes(name):
    g = _gen()
    if name == "powerlaw_zipf173":
        return g.zipf_lengths(4_194_304, 1.73, 4096, 2)
    if name == "powerlaw_zipf15":
        return g.zipf_lengths(4_194_304, 1.5, 4096, 2)
    if name == "laplacian1024":
        return g.laplacian_2d(1024).row_lengths()
    return g.diffusion_3d(64).row_lengths() if name == "small" else None


@pytest.mark.parametrize("name", ["powerlaw_zipf173", "powerlaw_zipf15", "laplacian1024", "diffusion256"])
def test_builders_full_size_match_reference(name, diffusion):
    """Segment metadata of the GPU builders at full size, bit for bit against
    the digests of the reference's Host builders."""
    t = tnl()
    ref = GOLDEN["builders"][name]
    sizes = diffusion.row_lengths() if name == "diffusion256" else _config_sizes(name)
    assert digest(np.ascontiguousarray(sizes, np.int32)) == ref["sizes_digest"]
    s = t.CSR()
    s.setSegmentsSizes(sizes)
    assert digest(s.getOffsets()) == ref["CSR"]["offsets"]
    meta = {"SlicedEllpack": lambda s: {"sliceOffsets": s.getSliceOffsets(),
                                        "sliceSegmentSizes": s.getSliceSegmentSizes()},
            "BiEllpack": lambda s: {"perm": s.getSegmentsPermutation(), "groupPointers": s.getGroupPointers()},
            "ChunkedEllpack": lambda s: {}}
    for fmt, get in meta.items():
        s = t.FORMATS[fmt]()
        if ref[fmt]["storage"] < 0:
            # the reference's int32 storage count wraps around (a negative
            # size); the GPU builder refuses the matrix instead
            with pytest.raises(OverflowError):
                s.setSegmentsSizes(sizes)
            continue
        s.setSegmentsSizes(sizes)
        assert s.getStorageSize() == ref[fmt]["storage"], fmt
        for k, v in get(s).items():
            assert digest(v) == ref[fmt][k], (fmt, k)


@pytest.mark.parametrize("name", ["powerlaw_zipf173", "laplacian1024"])
def test_adaptive_csr_descriptors_full_size(oracle, name):
    """AdaptiveCSR descriptors at full size against the oracle (the
    reference's Host builder needs a CUDA backend for LONG descriptors,
    which the power-law rows produce)."""
    t = tnl()
    sizes = _config_sizes(name)
    s = t.AdaptiveCSR()
    s.setSegmentsSizes(sizes)
    off = np.zeros(len(sizes) + 1, np.int32)
    off[1:] = np.cumsum(sizes)
    for sl in range(6):
        b = s.getBlocks(sl)
        o = oracle.acsr_blocks(off, sl)
        assert len(b) == len(o["type"]), sl
        assert np.array_equal(b["type"], o["type"]), sl
        assert np.array_equal(b["first_segment"], o["first"]), sl
        assert np.array_equal(b["warp_idx"], o["warpIdx"]), sl
        nonlong = o["type"] != 0
        nonlong[-1:] = False
        assert np.array_equal(b["block_size"][nonlong], o["blockSize"][nonlong]), sl
        assert np.array_equal(b["segments_in_block"][nonlong], o["segmentsInBlock"][nonlong]), sl
        wc = o["type"] == 0
        assert np.array_equal(b["warps_count"][wc], o["warpsCount"][wc]), sl


def test_laplacian_1024_jacobi_cg_matches_reference(laplacian):
    """CG with the Diagonal preconditioner on the 1024^2 Laplacian to the
    reference's stopping rule at 1e-8: the iteration count within 2 of the
    reference's (one- and multi-threaded runs), the true residual of the
    same order as the reference's solution's."""
    t = tnl()
    g = _gen()
    A = laplacian
    b = torch.tensor(g.uniform_vector(A.n, 1), device="cuda")
    M = t.SparseMatrix(t.CSR, torch.float64).assign(A.rowptr, A.cols, A.vals)
    S = t.CG()
    S.setMatrix(M)
    P = t.Diagonal()
    P.update(M)
    S.setPreconditioner(P)
    S.setup({"convergence-residue": 1e-8, "max-iterations": 100000})
    x = torch.zeros(A.n, dtype=torch.float64, device="cuda")
    assert S.solve(b, x)
    refs = [v for k, v in GOLDEN["solves"].items() if k.startswith("laplacian1024/cg/jacobi/")]
    assert refs
    for r in refs:
        assert abs(S.getIterations() - r["iterations"]) <= 2, (S.getIterations(), r)
    tr = t.true_residual(M, b, x)
    assert tr < 1e-8 and tr < 2.0 * max(r["true_residual"] for r in refs), tr


def _fp64_pcg(M, b, tol, precond="jacobi", maxit=200000):
    t = tnl()
    S = t.CG()
    S.setMatrix(M)
    P = t.Diagonal() if precond == "jacobi" else t.FSAI()
    P.update(M)
    S.setPreconditioner(P)
    S.setConvergenceResidue(tol)
    S.setMaxIterations(maxit)
    x = torch.zeros(M.getRows(), dtype=torch.float64, device="cuda")
    S.solve(b, x)
    return x, S.getIterations()


def _fp64_to_true_residual(M, b, tol, precond="jacobi"):
    """FP64 PCG with its stopping residue halved until the true residual is
    below tol."""
    t = tnl()
    r = tol
    while True:
        x, it = _fp64_pcg(M, b, r, precond)
        if t.true_residual(M, b, x) < tol or r < tol * 1e-4:
            return x, it
        r *= 0.5


def _rel_err(x, xref):
    return float(torch.linalg.vector_norm(x - xref) / torch.linalg.vector_norm(xref))


def test_diffusion_256cubed_mixed_error_against_fp64(diffusion):
    """256^3 GRF diffusion to a true residual of 1e-10: FP32 PCG with
    reliable FP64 updates (Jacobi) and FP32-inner refinement, each solution
    against a FP64 solve converged to a true residual of 1e-13."""
    t = tnl()
    g = _gen()
    A = diffusion
    M = t.SparseMatrix(t.CSR, torch.float64).assign(A.rowptr, A.cols, A.vals)
    b = torch.tensor(g.uniform_vector(A.n, 1), device="cuda")
    xref, _ = _fp64_to_true_residual(M, b, 1e-13)
    x64, _ = _fp64_to_true_residual(M, b, 1e-10)
    e64 = _rel_err(x64, xref)
    x = torch.zeros(A.n, dtype=torch.float64, device="cuda")
    r = t.solve_mixed_reliable(M, b, x, tol=1e-10, inner="jacobi")
    assert r["converged"] and t.true_residual(M, b, x) < 1e-10
    assert _rel_err(x, xref) <= 4.0 * e64 + 1e-14, (_rel_err(x, xref), e64)
    x = torch.zeros(A.n, dtype=torch.float64, device="cuda")
    r = t.solve_mixed(M, b, x, tol=1e-10, inner="jacobi")
    assert r["converged"] and t.true_residual(M, b, x) < 1e-10
    assert _rel_err(x, xref) <= 4.0 * e64 + 1e-14, (_rel_err(x, xref), e64)


def test_learned_evaluation_problem_mixed_error_against_fp64():
    """2048^2 GRF diffusion (the learned preconditioner's evaluation size)
    to a true residual of 1e-8: FP32 PCG with reliable FP64 updates and the
    classical or the learned FSAI, against a FP64 solve converged to 1e-12.
    The reference point is FP64 PCG with the classical FSAI stopped at the
    same true residual (the error left at a given residual depends on the
    preconditioner, so the FP32 solves are compared with a FP64 solve of
    the same family): FP32 arithmetic may cost at most an order of magnitude
    of solution error at the same true residual (measured: 8x for the
    classical FSAI, 6.7x for the learned one)."""
    t = tnl()
    g = _gen()
    from tnl_b200.lfsai import LearnedFSAI

    A = g.diffusion_2d_problem(2048, 1234)
    M = t.SparseMatrix(t.CSR, torch.float64).assign(A.rowptr, A.cols, A.vals)
    b = torch.tensor(g.uniform_vector(A.n, 1), device="cuda")
    xref, _ = _fp64_to_true_residual(M, b, 1e-12)
    x64, _ = _fp64_to_true_residual(M, b, 1e-8, precond="fsai")
    e64 = _rel_err(x64, xref)
    A32 = t.SparseMatrix(t.CSR, torch.float32).assign(A.rowptr, A.cols, A.vals.astype(np.float32))
    net = LearnedFSAI(seed=0)
    net.load(Path(t.__file__).resolve().parent / "weights" / "lfsai_diffusion.npy")
    errs = {}
    for name, P, bound in (("classical", "fsai", 12.0), ("learned", net.preconditioner(A32), 12.0)):
        x = torch.zeros(A.n, dtype=torch.float64, device="cuda")
        r = t.solve_mixed_reliable(M, b, x, tol=1e-8, inner=P)
        assert r["converged"] and t.true_residual(M, b, x) < 1e-8, name
        errs[name] = _rel_err(x, xref)
        assert errs[name] <= bound * e64 + 1e-14, (name, errs[name], e64)
    print({"fp64_fsai": e64, **errs})
