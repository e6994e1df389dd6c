"""The oracle (oracle/tnl_oracle.c) pinned against the reference.

CPU only.  Checks the C restatement against
  * the known-answer vectors of the reference's unit tests,
  * the golden fixtures produced by the reference itself (always), and
  * the reference compiled here from its headers (oracle/_ref), when built.
"""
import hashlib

import numpy as np
import pytest

from helpers import FORMATS
from known_answers import cases as known_cases
from tnl_b200 import generators as g

KINDS = ["CSR", "Ellpack", "SlicedEllpack", "ChunkedEllpack", "BiEllpack"]


@pytest.mark.parametrize("fmt", list(FORMATS))
@pytest.mark.parametrize("colmajor", [True, False])
def test_known_answers(oracle, fmt, colmajor):
    for name, rp, c, v, nc, x, y0, expected in known_cases():
        seg = oracle.build(FORMATS[fmt], np.diff(rp), colmajor=colmajor)
        oc, ov = oracle.fill(seg, rp, c, v)
        y = oracle.spmv(seg, oc, ov, x, y0)
        assert np.array_equal(y, expected), (name, fmt)


@pytest.mark.parametrize("kname", KINDS)
def test_builders_match_golden(oracle, golden, kname):
    for case in golden.size_cases():
        sizes = golden.get(f"sizes/{case}")
        key = f"{case}/{kname}"
        if key not in golden.meta["builders"]:
            continue
        if golden.meta["builders"][key] == "overflow":
            with pytest.raises(OverflowError):
                oracle.build(FORMATS[kname], sizes)
            continue
        seg = oracle.build(FORMATS[kname], sizes)
        for k, v in golden.meta["builders"][key].items():
            if k == "storage":
                assert seg.storage == v, (case, kname)
            else:
                assert seg.meta[k] == v, (case, kname, k)
        prefix = f"build/{case}/{kname}/"
        for name in golden.arrays.files:
            if name.startswith(prefix):
                assert np.array_equal(np.asarray(seg.meta[name[len(prefix):]]), golden.get(name)), (case, kname, name)


def test_acsr_blocks_match_golden(oracle, golden):
    checked = 0
    for case in golden.size_cases():
        sizes = golden.get(f"sizes/{case}")
        off = np.zeros(len(sizes) + 1, np.int32)
        off[1:] = np.cumsum(sizes)
        for sl in range(6):
            if golden.meta["acsr"].get(f"{case}/{sl}") in (None, "unavailable"):
                continue
            b = oracle.acsr_blocks(off, sl)
            for k in b:
                assert np.array_equal(b[k], golden.get(f"acsr/{case}/{sl}/{k}")), (case, sl, k)
            checked += 1
    assert checked > 20


def _digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("mname", ["powerlaw2000", "laplacian32"])
def test_fill_and_spmv_match_golden(oracle, golden, mname):
    rp = golden.get(f"mat/{mname}/rowptr")
    cols = golden.get(f"mat/{mname}/cols")
    vals = golden.get(f"mat/{mname}/vals")
    x = golden.get(f"mat/{mname}/x")
    for kname, kind in FORMATS.items():
        for cm in (True, False):
            for real in (np.float64, np.float32):
                tag = f"{mname}/{kname}/{'col' if cm else 'row'}/{np.dtype(real).name}"
                seg = oracle.build(kind, np.diff(rp), colmajor=cm)
                oc, ov = oracle.fill(seg, rp, cols, vals.astype(real))
                ref = golden.meta["fill"][tag]
                assert seg.storage == ref["storage"], tag
                assert _digest(oc) == ref["cols"] and _digest(ov) == ref["vals"], tag
        seg = oracle.build(kind, np.diff(rp), colmajor=False)
        oc, ov = oracle.fill(seg, rp, cols, vals)
        y = oracle.spmv(seg, oc, ov, x)
        # same per-row summation order as the Host reference -> bit-identical
        assert np.array_equal(y, golden.get(f"spmv/{mname}/{kname}")), (mname, kname)


def test_builders_match_reference_random(oracle, reference):
    rng = np.random.default_rng(7)
    for trial in range(25):
        n = int(rng.integers(1, 3000))
        mode = trial % 3
        if mode == 0:
            sizes = rng.integers(0, 64, n)
        elif mode == 1:
            sizes = g.zipf_lengths(n, float(rng.uniform(1.2, 2.5)), 4096, int(rng.integers(1 << 30)))
        else:
            sizes = np.where(rng.random(n) < 0.5, 0, rng.integers(0, 600, n))
        sizes = sizes.astype(np.int32)
        for kname in KINDS:
            r = reference.build(FORMATS[kname], sizes)
            o = oracle.build(FORMATS[kname], sizes)
            for k, v in r.items():
                if k == "storage":
                    assert o.storage == v
                else:
                    assert np.array_equal(np.asarray(o.meta[k]), np.asarray(v)), (trial, kname, k)


def test_ellpack_overflow_like_reference(oracle, reference):
    sizes = np.full(40000, 60000, np.int32)  # 40000*60000 > 2^31
    with pytest.raises(OverflowError):
        reference.build(FORMATS["Ellpack"], sizes)
    with pytest.raises(OverflowError):
        oracle.build(FORMATS["Ellpack"], sizes)


@pytest.mark.parametrize("pname", ["laplacian32", "diffusion32"])
def test_solvers_match_golden(oracle, golden, pname):
    class A:
        pass

    A.rowptr = golden.get(f"prob/{pname}/rowptr")
    A.cols = golden.get(f"prob/{pname}/cols")
    A.vals = golden.get(f"prob/{pname}/vals")
    A.n = len(A.rowptr) - 1
    b = golden.get(f"prob/{pname}/b")
    for key, ref in golden.meta["solvers"].items():
        p, solver, pre = key.split("/")
        if p != pname:
            continue
        pre = int(pre)
        r = oracle.solve(solver, A, b, precond=pre, tol=1e-8, maxit=20000, gmres_m=30, gmres_reorth=2)
        assert r["converged"] == ref["converged"], key
        if solver in ("bicgstab", "bicgstabl"):
            # BiCGStab amplifies the reference's non-reproducible OpenMP
            # reductions: the reference itself moves by up to ~10% of its
            # iteration count between thread counts (1..8 threads).
            assert abs(r["iterations"] - ref["iterations"]) <= max(5, ref["iterations"] // 10), key
            assert r["residue"] < 1e-8
        else:
            assert r["iterations"] == ref["iterations"], key
            assert r["residue"] == pytest.approx(ref["residue"], rel=1e-6), key
            xr = golden.get(f"solve/{key}/x")
            if solver in ("tfqmr", "idrs"):
                # their recurrences amplify the reference's blocked dot-product
                # order more than CG / GMRES do
                assert np.allclose(r["x"], xr, rtol=1e-6, atol=1e-9 * np.abs(xr).max()), key
            else:
                assert np.allclose(r["x"], xr, rtol=1e-9, atol=1e-12), key


def test_preconditioners_match_reference(oracle, reference):
    A = g.diffusion_2d(24, 0.1, 1.5, 4)
    b = g.uniform_vector(A.n, 3)
    for kind in (1, 2):
        assert np.array_equal(oracle.prec_apply(A, kind, b), reference.prec_apply(A, kind, b)), kind


def test_bicgstab_within_reference_spread(oracle, reference):
    """The reference's own BiCGStab changes with its OpenMP thread count; the
    oracle must stay inside that spread."""
    A = g.diffusion_2d(40, 0.1, 1.0, 3)
    b = g.uniform_vector(A.n, 1)
    o = oracle.solve("bicgstab", A, b, precond=1, tol=1e-8, maxit=20000)
    its = []
    try:
        for t in (1, 2, 3, 4, 8):
            reference.set_threads(t)
            r = reference.solve("bicgstab", A, b, precond=1, tol=1e-8, maxit=20000)
            assert r["converged"]
            its.append(r["iterations"])
    finally:
        reference.set_threads(reference.threads())
    assert o["converged"]
    spread = max(its) - min(its)
    assert min(its) - max(2, spread) <= o["iterations"] <= max(its) + max(2, spread), (o["iterations"], its)
    assert oracle.true_residual(A, b, o["x"]) < 1e-7


@pytest.mark.parametrize("level", [0, 1])
def test_lfsai_reference_fd(level):
    """The FP64 backpropagation of the learned-FSAI reference against central
    finite differences (BF16 rounding off), for the probe loss and the
    Kaporin loss, on G's level-0 and level-1 patterns."""
    from oracle import lfsai_ref as R
    from tnl_b200 import generators as g

    A = g.diffusion_2d(10, 0.2, 1.0, 3)
    theta = R.init_params(7)
    rng = np.random.default_rng(0)
    Z = rng.choice([-1.0, 1.0], size=(A.n, 3))
    old = R.ROUND
    R.ROUND = False
    try:
        for loss in (lambda th: R.loss_and_grad(th, A, Z, level), lambda th: R.kaporin_and_grad(th, A, level)):
            _, grad = loss(theta)
            idx = np.nonzero(np.abs(grad) > 1e-4 * np.abs(grad).max())[0]
            for i in rng.choice(idx, 10, replace=False):
                e = np.zeros_like(theta)
                e[i] = 1e-6
                fd = (loss(theta + e)[0] - loss(theta - e)[0]) / 2e-6
                assert fd == pytest.approx(grad[i], rel=1e-5, abs=1e-10)
    finally:
        R.ROUND = old


def test_lfsai_two_factor_reference_fd():
    """The two-factor (nonsymmetric) probe-loss backpropagation of the
    learned-FSAI reference against central finite differences (BF16
    rounding off), on an upwind convection-diffusion operator."""
    from oracle import lfsai_ref as R
    from tnl_b200 import generators as g

    A = g.convection_diffusion_3d(5)
    theta = R.init_params(3)
    rng = np.random.default_rng(0)
    Z = rng.choice([-1.0, 1.0], size=(A.n, 3))
    old = R.ROUND
    R.ROUND = False
    try:
        _, grad = R.loss_and_grad2(theta, A, Z)
        idx = np.nonzero(np.abs(grad) > 1e-4 * np.abs(grad).max())[0]
        for i in rng.choice(idx, 10, replace=False):
            e = np.zeros_like(theta)
            e[i] = 1e-6
            fd = (R.loss_and_grad2(theta + e, A, Z)[0] - R.loss_and_grad2(theta - e, A, Z)[0]) / 2e-6
            assert fd == pytest.approx(grad[i], rel=1e-5, abs=1e-10)
    finally:
        R.ROUND = old


def test_lfsai_reference_patterns_and_classical_fsai():
    """Level-1 pattern of a 5-point operator: the 7 lower entries of its
    13-point square; classical FSAI on it is the Kaporin minimiser, so it
    has a smaller Kaporin number than FSAI on A's own pattern, and the
    warm-start target is the level-0 FSAI padded with zeros."""
    import scipy.sparse as sp

    from oracle import lfsai_ref as R
    from tnl_b200 import generators as g

    N = 9
    A = g.diffusion_2d(N, 0.2, 1.5, 4)
    p1 = R.pattern(A, 1)
    i = 4 * N + 4  # an interior cell
    assert p1[i] == sorted([i, i - 1, i - 2, i - N, i - 2 * N, i - N + 1, i - N - 1])
    As = sp.csr_matrix((A.vals, A.cols, A.rowptr), shape=(A.n, A.n)).toarray()

    def kaporin(level, vals):
        pat = R.pattern(A, level)
        G = R.g_matrix(vals, pat, A.n).toarray()
        M = G @ As @ G.T
        ev = np.linalg.eigvalsh(M)
        return np.mean(ev) / np.exp(np.mean(np.log(ev)))

    k0 = kaporin(0, R.fsai_classical(A, 0))
    k1 = kaporin(1, R.fsai_classical(A, 1))
    assert k1 < k0
    assert np.isclose(kaporin(1, R.fit_target(A, 1)), k0)


@pytest.mark.parametrize("solver,kw", [("tfqmr", {}), ("bicgstabl", {"ell": 1}), ("bicgstabl", {"ell": 3}),
                                       ("bicgstabl", {"ell": 2, "bicgstab_exact": True}), ("idrs", {"idr_s": 4}),
                                       ("idrs", {"idr_s": 2, "idr_smoothing": True})])
def test_more_krylov_match_reference(oracle, reference, solver, kw):
    """TFQMR, BiCGStab(ell) and IDR(s) restated in the oracle against the
    reference's own solvers.  The reference sums dot products in a blocked
    order (and in OpenMP threads, so its own counts move between runs), the
    oracle sequentially: IDR(s) stays within 2 % of the reference's
    iterations; BiCGStab(ell) and TFQMR, whose short recurrences amplify the
    rounding (TFQMR moves 150-158 between runs of the reference on the
    convection-diffusion matrix), within 10 %.  The reference runs on one
    thread, so that its counts do not move between runs."""
    probs = [g.laplacian_2d(32), g.diffusion_2d(33, 0.1, 2.0, 6), g.convection_diffusion_3d(10)]
    threads = reference.threads()
    reference.set_threads(1)
    try:
        for A in probs:
            b = g.uniform_vector(A.n, 1)
            for pre in (1, 2):
                r = reference.solve(solver, A, b, precond=pre, tol=1e-8, maxit=20000, **kw)
                o = oracle.solve(solver, A, b, precond=pre, tol=1e-8, maxit=20000, **kw)
                assert r["converged"] and o["converged"], (solver, kw, pre)
                slack = (max(5, r["iterations"] // 10) if solver in ("bicgstabl", "tfqmr")
                         else max(2, r["iterations"] // 50))
                assert abs(r["iterations"] - o["iterations"]) <= slack, (solver, kw, pre, r["iterations"],
                                                                         o["iterations"])
                assert np.allclose(o["x"], r["x"], rtol=1e-5, atol=1e-6 * np.abs(r["x"]).max()), (solver, kw, pre)
    finally:
        reference.set_threads(threads)


def test_idrs_shadow_space_matches_reference_draws(oracle, reference):
    """The IDR(s) shadow space is drawn from std::mt19937 / std::normal_distribution
    as the reference does: with a preconditioner that makes the solve short, the
    oracle reproduces the reference's iterates to rounding."""
    A = g.laplacian_2d(32)
    b = g.uniform_vector(A.n, 1)
    r = reference.solve("idrs", A, b, precond=2, tol=1e-8, maxit=100, idr_s=4)
    o = oracle.solve("idrs", A, b, precond=2, tol=1e-8, maxit=100, idr_s=4)
    assert r["iterations"] == o["iterations"]
    assert np.allclose(o["x"], r["x"], rtol=1e-10, atol=1e-12)


def _lower_triangle(A):
    keep = np.asarray(A.cols) <= np.repeat(np.arange(A.n), np.diff(A.rowptr))
    lens = np.add.reduceat(keep.astype(np.int64), A.rowptr[:-1]) if A.nnz else np.zeros(A.n, np.int64)
    lens[np.diff(A.rowptr) == 0] = 0
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    return g.CSRMatrix(rp, A.cols[keep], A.vals[keep], A.ncols)


def test_symmetric_and_transposed_products_match_reference(oracle, reference):
    """vectorProduct of a SymmetricMatrix and transposedVectorProduct restated
    in the oracle against the reference's Host code run on one thread (its
    atomic additions then come in row order): bit-exact; and both against
    the full / transposed product."""
    import scipy.sparse as sp

    threads = reference.threads()
    reference.set_threads(1)
    try:
        A = g.diffusion_2d(40, 0.1, 1.0, 3)
        L = _lower_triangle(A)
        seg = oracle.build(FORMATS["CSR"], L.row_lengths())
        x, y0 = g.uniform_vector(A.n, 2), g.uniform_vector(A.n, 3)
        for al, be, b, e in ((1.0, 0.0, 0, 0), (2.5, -0.5, 0, 0), (1.0, 1.0, 100, 900)):
            yr = reference.spmv_symmetric(L, x, y0, al, be, b, e)
            yo = oracle.spmv_symmetric(seg, L.cols, L.vals, x, y0, al, be, b, e)
            assert np.array_equal(yr, yo), (al, be, b, e)
        S = sp.csr_matrix((A.vals, A.cols, A.rowptr), shape=(A.n, A.n))
        assert np.allclose(oracle.spmv_symmetric(seg, L.cols, L.vals, x), S @ x, rtol=1e-13, atol=1e-13)
        P = g.power_law(3000, 1.73, 500, 4)
        segP = oracle.build(FORMATS["CSR"], P.row_lengths())
        xP, yP = g.uniform_vector(P.n, 5), g.uniform_vector(P.ncols, 6)
        for al, be, b, e in ((1.0, 0.0, 0, 0), (2.5, -0.5, 0, 0), (1.0, 1.0, 100, 2000)):
            yr = reference.spmv_transposed(P, xP, yP, al, be, b, e)
            yo = oracle.spmv_transposed(segP, P.cols, P.vals, P.ncols, xP, yP, al, be, b, e)
            assert np.array_equal(yr, yo), (al, be, b, e)
        SP = sp.csr_matrix((P.vals, P.cols, P.rowptr), shape=(P.n, P.ncols))
        assert np.allclose(oracle.spmv_transposed(segP, P.cols, P.vals, P.ncols, xP), SP.T @ xP, rtol=1e-12,
                           atol=1e-12)
    finally:
        reference.set_threads(threads)


def test_reliable_update_pcg_restatement(oracle):
    """The restatement of the library's reliable-update mixed PCG (no
    reference counterpart) reaches the FP64 tolerance on the true residual
    with close to the FP64 Jacobi-CG iteration count, folding its FP32
    correction into x about once per factor-10 drop of the residual."""
    A = g.diffusion_2d(96, 0.1, 2.0, 7)
    b = g.uniform_vector(A.n, 1)
    f = oracle.solve("cg", A, b, precond=1, tol=1e-9)
    r = oracle.pcg_reliable(A, b, precond=1, tol=1e-8, delta=0.1)
    assert r["converged"] and oracle.true_residual(A, b, r["x"]) < 1e-8
    assert abs(r["residue"] - oracle.true_residual(A, b, r["x"])) < 1e-15
    assert r["iterations"] <= 1.3 * f["iterations"], (r["iterations"], f["iterations"])
    assert 6 <= r["updates"] <= 10
    # max_iterations bounds the FP32 iterations
    s = oracle.pcg_reliable(A, b, precond=1, tol=1e-8, delta=0.1, maxit=50)
    assert not s["converged"] and s["iterations"] == 50
    # FP64 vectors with the FP32 values
    v = oracle.pcg_reliable(A, b, precond=1, tol=1e-8, delta=0.1, vec64=True)
    assert v["converged"] and oracle.true_residual(A, b, v["x"]) < 1e-8
    assert v["iterations"] <= 1.3 * f["iterations"], (v["iterations"], f["iterations"])


def test_reliable_update_pcg_restatement_stalls(oracle):
    """On a matrix whose FP32 values are singular (a Neumann Laplacian plus
    1e-7 I) the restatement's FP32 iteration cannot reach the tolerance: it
    reports a stall within the window (16384 iterations past the last
    halving of the true residual, updates forced every 4096 iterations)
    and returns the x of its lowest true residual.  FP64 Jacobi CG, the
    library's fallback, solves the same system."""
    from helpers import fp32_singular_laplacian, nonzero_mean_rhs

    A = fp32_singular_laplacian(32)
    assert np.unique(A.vals.astype(np.float32)).tolist() == [-1.0, 2.0, 3.0, 4.0]
    b = nonzero_mean_rhs(A.n)
    for vec64 in (False, True):
        r = oracle.pcg_reliable(A, b, precond=1, tol=1e-10, delta=0.3, maxit=200000, vec64=vec64, excess=False)
        assert r["stalled"] and not r["converged"]
        assert 16384 < r["iterations"] < 2 * 16384 + 4096, r["iterations"]
        assert r["updates"] >= 4  # forced ones among them
        assert abs(oracle.true_residual(A, b, r["x"]) - r["residue"]) < 1e-12
        assert r["residue"] < 1e-2
    f = oracle.solve("cg", A, b, precond=1, tol=1e-10)
    assert f["converged"] and oracle.true_residual(A, b, f["x"]) < 1e-9


def test_reliable_update_pcg_restatement_row_excess(oracle):
    """The row-excess form of the FP32 product keeps what FP32 rounding
    of the diagonal loses: on the matrix that is singular in FP32 (plain
    form: a stall) it converges with FP64 vectors in the iterations of FP64
    Jacobi CG, and on a high-contrast diffusion matrix (sigma = 3) it takes
    a fifth fewer FP32 iterations than the plain form."""
    from helpers import fp32_singular_laplacian, nonzero_mean_rhs

    A = fp32_singular_laplacian(32)
    b = nonzero_mean_rhs(A.n)
    f = oracle.solve("cg", A, b, precond=1, tol=1e-10)
    r64 = oracle.pcg_reliable(A, b, precond=1, tol=1e-10, delta=0.3, maxit=200000, vec64=True, excess=True)
    assert r64["converged"] and abs(r64["iterations"] - f["iterations"]) <= 0.05 * f["iterations"], (r64, f)
    D = g.diffusion_2d(128, 0.05, 3.0, 11)
    bd = g.uniform_vector(D.n, 1)
    plain = oracle.pcg_reliable(D, bd, precond=1, tol=1e-8, delta=0.3, maxit=200000, excess=False)
    exc = oracle.pcg_reliable(D, bd, precond=1, tol=1e-8, delta=0.3, maxit=200000, excess=True)
    assert plain["converged"] and exc["converged"]
    assert exc["iterations"] < 0.9 * plain["iterations"], (exc["iterations"], plain["iterations"])


def test_reliable_update_pcg_restatement_fsai(oracle):
    """The FSAI form of the restatement (z = G^T G r, (r, z) = |G r|^2):
    with G = I it takes the unpreconditioned steps bit for bit; with the
    diagonal factor G = D^-1/2 it converges like Jacobi."""
    A = g.diffusion_2d(64, 0.1, 2.0, 3)
    b = g.uniform_vector(A.n, 1)
    n = A.n
    eye = (np.arange(n + 1, dtype=np.int32), np.arange(n, dtype=np.int32), np.ones(n, np.float32))
    r0 = oracle.pcg_reliable(A, b, precond=0, tol=1e-8, delta=0.1)
    ri = oracle.pcg_reliable_fsai(A, b, eye, eye, tol=1e-8, delta=0.1)
    assert ri["converged"] and (ri["iterations"], ri["updates"]) == (r0["iterations"], r0["updates"])
    assert np.array_equal(ri["x"], r0["x"])
    d = np.array([A.vals[A.rowptr[i]:A.rowptr[i + 1]][A.cols[A.rowptr[i]:A.rowptr[i + 1]] == i][0]
                  for i in range(n)])
    gd = (eye[0], eye[1], (1.0 / np.sqrt(d)).astype(np.float32))
    rj = oracle.pcg_reliable(A, b, precond=1, tol=1e-8, delta=0.1)
    rd = oracle.pcg_reliable_fsai(A, b, gd, gd, tol=1e-8, delta=0.1)
    assert rd["converged"] and oracle.true_residual(A, b, rd["x"]) < 1e-8
    assert abs(rd["iterations"] - rj["iterations"]) <= max(3, 0.03 * rj["iterations"]), (rd, rj["iterations"])


def test_transposition_matches_reference(oracle, reference):
    """getTransposition: the restatement (stable sort by column) equals the
    reference's single-threaded Host result bit for bit -- row pointer,
    columns in order and values times the multiplicator -- on square,
    rectangular and empty-row matrices."""
    from tnl_b200.generators import CSRMatrix

    t0 = reference.threads()
    reference.set_threads(1)
    try:
        P = g.power_law(3000, 1.73, 300, 5)
        rng = np.random.default_rng(3)
        # rectangular: 500 rows, 1700 columns, some empty rows
        lens = rng.integers(0, 9, 500)
        lens[::7] = 0
        rp = np.zeros(501, np.int32)
        rp[1:] = np.cumsum(lens)
        cols = np.concatenate([np.sort(rng.choice(1700, k, replace=False)) for k in lens]).astype(np.int32)
        R = CSRMatrix(rp, cols, rng.uniform(-1, 1, rp[-1]), ncols=1700)
        for A in (g.laplacian_2d(20), P, R):
            for mult in (1.0, -2.5):
                trp, tc, tv = oracle.transpose(A, mult)
                rrp, rc, rv = reference.transpose(A, mult)
                assert np.array_equal(trp, rrp) and np.array_equal(tc, rc)
                assert np.array_equal(tv, rv)
    finally:
        reference.set_threads(t0)


def _ilut_reference_as_combined(L, U, n):
    """The reference's separate L and (row-reversed) U, padding dropped, as
    one CSR with row i = L_i then U_i (the restatement's layout)."""
    (lrp, lc, lv), (urp, uc, uv) = L, U
    rp, cols, vals = [0], [], []
    for i in range(n):
        for q in range(lrp[i], lrp[i + 1]):
            if lc[q] >= 0:
                cols.append(lc[q])
                vals.append(lv[q])
        r = n - 1 - i
        for q in range(urp[r], urp[r + 1]):
            if uc[q] >= 0:
                cols.append(uc[q])
                vals.append(uv[q])
        rp.append(len(cols))
    return np.array(rp, np.int32), np.array(cols, np.int32), np.array(vals)


@pytest.mark.parametrize("p,tau", [(0, 1e-4), (2, 1e-3), (5, 1e-2), (1, 0.0)])
def test_ilut_restatement_matches_reference(oracle, reference, p, tau):
    """ILUT factors of the restatement equal the reference's ILUT::update bit
    for bit (pattern, order, values), and one application equals its solve,
    on a Laplacian (many equal magnitudes: heap tie order), a
    diffusion matrix and a nonsymmetric convection-diffusion matrix."""
    for A in (g.laplacian_2d(12), g.diffusion_2d(14, 0.1, 2.0, 5), g.convection_diffusion_3d(6)):
        frp, fc, fv = oracle.ilut_factor(A, p, tau)
        rrp, rc, rv = _ilut_reference_as_combined(*reference.ilut_factor(A, p, tau), A.n)
        assert np.array_equal(frp, rrp) and np.array_equal(fc, rc)
        assert np.array_equal(fv, rv)
        b = g.uniform_vector(A.n, 3)
        assert np.array_equal(oracle.lu_apply(frp, fc, fv, b), reference.ilut_apply(A, b, p, tau))
