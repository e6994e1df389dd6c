"""SpMV and linear-solver benchmarks: the counterparts of the reference's
tnl-benchmark-spmv (Benchmarks/SpMV/spmv.h) and
tnl-benchmark-linear-solvers (Benchmarks/LinearSolvers/tnl-benchmark-linear-solvers.h),
on seeded synthetic matrices.  One JSON object per line on stdout.

    python -m tnl_b200.benchmarks spmv    [--configs laplacian,power_law] [--reals f64,f32] [--steps K]
    python -m tnl_b200.benchmarks solvers [--problem laplacian|diffusion] [--N 1024]
    python -m tnl_b200.benchmarks sweep   [--problem laplacian|diffusion|convection_diffusion] [--N 1024]
    python -m tnl_b200.benchmarks profile-solvers [--problem diffusion] [--N 2048] [--iterations 40]
    python -m tnl_b200.benchmarks configs --which c3|c5
    python -m tnl_b200.benchmarks learned-eval [--count 64] [--N 2048]
    python -m tnl_b200.benchmarks c1-solves
    python -m tnl_b200.benchmarks assembly [--max-grid 8192]

spmv: every segment format and kernel on the 1024^2 5-point Laplacian
(n = 1,048,576), the power-law matrix (n = 4,194,304, Zipf 1.73 row
lengths, cap 4096, seed 2) and, with --configs diffusion3d, the 256^3
7-point diffusion matrix (n = 16,777,216, GRF coefficients).  GB/s counts algorithmic bytes, the same for
every format: nnz*(R+4) + (n+1)*4 + n*R (x) + n*R (y); padding therefore
lowers the figure.  Device time per product from CUDA events over K
back-to-back products; a matrix smaller than L2 (the Laplacian's 84 MB) is
timed in copies cycled so that the ring exceeds three times the 126 MB L2.

solvers: time to an FP64 true residual ||b - A x|| / ||b|| <= 1e-8 (CUDA
events around the solve call; preconditioner set-up timed separately) for
FP64 Jacobi-PCG, FP64 FSAI-PCG, FP32-inner refinement with FSAI, and the
learned FSAI with FP32-inner refinement (weights from a training run on
smaller seeded diffusion problems, or trained on the spot).
"""
from __future__ import annotations

import argparse
import json
import sys
from pathlib import Path

import numpy as np
import torch

ROOT = Path(__file__).resolve().parents[1]


def spmv_bytes(n: int, ncols: int, nnz: int, real_bytes: int) -> int:
    return nnz * (real_bytes + 4) + (n + 1) * 4 + ncols * real_bytes + n * real_bytes


def hbm_peak() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _matrix(config: str):
    from . import generators as g

    if config == "laplacian":
        return g.laplacian_2d(1024)
    if config == "power_law":
        return g.power_law(4_194_304, 1.73, 4096, 2)
    if config == "power_law_15":  # the literal Zipf 1.5 of the power-law config: mean ~49, ~2.06e8 nonzeros
        return g.power_law(4_194_304, 1.5, 4096, 2)
    if config == "diffusion3d":
        return g.diffusion_3d(256)
    raise ValueError(config)


# (label, segments class name, launch mapping, threads per segment)
SPMV_VARIANTS = [
    ("CSR default", "CSR", "Default", 0),
    ("CSR tile", "CSR", "Tile", 0),
    ("CSR Light", "CSR", "Light", 0),
    ("CSR Scalar", "CSR", "Scalar", 0),
    ("CSR Vector", "CSR", "Vector", 32),
    ("AdaptiveCSR", "AdaptiveCSR", "Adaptive", 0),
    ("Ellpack", "Ellpack", "Default", 0),
    ("SlicedEllpack", "SlicedEllpack", "Default", 0),
    ("ChunkedEllpack", "ChunkedEllpack", "Default", 0),
    ("BiEllpack", "BiEllpack", "Default", 0),
]


def time_spmv(Ms, xs, ys, lc, steps: int) -> float:
    """Mean device milliseconds per product over `steps` back-to-back calls
    (replayed from a CUDA graph), cycling through the copies Ms[k] (with
    their own xs[k], ys[k]).  A
    matrix larger than L2 is timed alone; a smaller one (the 84 MB
    Laplacian) in enough copies that the ring exceeds three times the
    126 MB L2, so every product reads its matrix from HBM -- without a
    scrub kernel between products, whose dirty lines the product would
    otherwise write back, and with the launch latency (about 5 us on its own
    for an isolated launch) hidden behind the previous product."""
    for k in range(len(Ms)):
        Ms[k].vectorProduct(xs[k], ys[k], launchConfig=lc, synchronize=False)
    torch.cuda.synchronize()

    def launch_all():
        for i in range(steps):
            k = i % len(Ms)
            Ms[k].vectorProduct(xs[k], ys[k], launchConfig=lc, synchronize=False)

    # The products are captured in a CUDA graph and replayed, so that the
    # time is the GPU's: a Python-level call costs more than a small
    # product takes.  A capture that fails falls back to direct calls.
    graph = None
    try:
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            launch_all()
        graph = g
    except Exception:
        torch.cuda.synchronize()
    run = graph.replay if graph is not None else launch_all
    run()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    run()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def bench_spmv(configs, reals, steps: int, formats=None, out=sys.stdout):
    import tnl_b200 as t
    from . import generators as g

    peak, peak_kind = hbm_peak()
    for config in configs:
        A = _matrix(config)
        xh = g.uniform_vector(A.ncols, 0)
        for real in reals:
            dt = torch.float64 if real == "f64" else torch.float32
            R = 8 if real == "f64" else 4
            nbytes = spmv_bytes(A.n, A.ncols, A.nnz, R)
            x = torch.tensor(xh, dtype=dt, device="cuda")
            y = torch.empty(A.n, dtype=dt, device="cuda")
            for label, seg, mapping, tps in SPMV_VARIANTS:
                if formats and label not in formats:
                    continue
                rec = {"bench": "spmv", "config": config, "rows": A.n, "nnz": A.nnz, "real": real, "format": label}
                try:
                    M = t.SparseMatrix(getattr(t, seg), dt).assign(A.rowptr, A.cols, A.vals)
                except OverflowError as e:  # Ellpack of the power-law matrix: 4096 x 4.19M > 2^31
                    rec["error"] = f"overflow_error: {e}"
                    print(json.dumps(rec), file=out, flush=True)
                    continue
                copies = 1 if nbytes > 512e6 else int(np.ceil(3 * 126e6 / nbytes))
                Ms, xs, ys = [M], [x], [y]
                for _ in range(copies - 1):
                    Ms.append(t.SparseMatrix(getattr(t, seg), dt).assign(A.rowptr, A.cols, A.vals))
                    xs.append(x.clone())
                    ys.append(torch.empty_like(y))
                ms = time_spmv(Ms, xs, ys, t.LaunchConfiguration(mapping, tps), max(steps, 4 * copies))
                gbs = nbytes / (ms / 1e3) / 1e9
                rec.update({"ms": ms, "GB/s": gbs, "frac_of_hbm": gbs / peak, "hbm_peak": f"{peak} ({peak_kind})",
                            "storage": M.segments.getStorageSize(), "padding": M.segments.getStorageSize() / A.nnz,
                            "l2": (f"{copies} copies cycled (ring > 3x L2)" if copies > 1
                                   else "inputs larger than L2")})
                print(json.dumps(rec), file=out, flush=True)
                del M, Ms, xs, ys
                torch.cuda.empty_cache()


def _timed(fn):
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    r = fn()
    e1.record()
    torch.cuda.synchronize()
    return r, e0.elapsed_time(e1)


def _median_timed(run, reps: int = 5):
    """run(x) on a fresh zero x, `reps` times: (result of the last run, its x,
    the fastest of the device times, all times).  The machine is shared with
    other jobs, whose host load stalls a single solve's host loop now and
    then by hundreds of ms; the fastest run is each method's own time."""
    times, res, x = [], None, None
    for _ in range(reps):
        x = run.new_x()
        res, ms = _timed(lambda: run(x))
        times.append(ms)
    return res, x, min(times), times


class _Run:
    def __init__(self, fn, n):
        self.fn, self.n = fn, n

    def new_x(self):
        return torch.zeros(self.n, dtype=torch.float64, device="cuda")

    def __call__(self, x):
        return self.fn(x)


def bench_solvers(problem: str, N: int, weights: str | None, out=sys.stdout):
    import tnl_b200 as t
    from . import generators as g
    from .lfsai import LearnedFSAI, diffusion_problem

    if problem == "laplacian":
        A = g.laplacian_2d(N)
        M = t.SparseMatrix.from_csr(A)
    else:
        M = diffusion_problem(N, 1234)
    n = M.getRows()
    b = torch.tensor(g.uniform_vector(n, 1), device="cuda")
    base = {"bench": "solver", "problem": problem, "N": N, "rows": n, "nnz": int(M.getValues().numel()),
            "tol": 1e-8}

    # every method is run once for 20 iterations before it is timed (module
    # loading and first-touch allocations stay out of the timed solve)
    def pcg(P, name, setup_ms):
        S = t.CG()
        S.setMatrix(M)
        S.setPreconditioner(P)
        S.setConvergenceResidue(1e-8)
        S.setMaxIterations(20)
        S.solve(b, torch.zeros(n, dtype=torch.float64, device="cuda"))
        S.setMaxIterations(200000)
        ok, x, ms, times = _median_timed(_Run(lambda x: S.solve(b, x), n))
        rec = dict(base, method=name, converged=bool(ok), iterations=S.getIterations(), solve_ms=ms,
                   solve_ms_runs=times, setup_ms=setup_ms, true_residual=t.true_residual(M, b, x))
        print(json.dumps(rec), file=out, flush=True)
        return rec

    P = t.Diagonal()
    _, s = _timed(lambda: P.update(M))
    jac = pcg(P, "FP64 Jacobi-PCG", s)
    P = t.FSAI()
    _, s = _timed(lambda: P.update(M))
    pcg(P, "FP64 FSAI-PCG", s)

    A32 = t.SparseMatrix(t.CSR, torch.float32)
    A32.assign(M.segments.getOffsets(), M.getColumnIndexes().cpu().numpy(), M.getValues().cpu().numpy())

    def mixed(name, inner, setup_ms):
        t.solve_mixed(M, b, torch.zeros(n, dtype=torch.float64, device="cuda"), tol=1e-8, inner_tol=1e-4,
                      inner=inner, max_outer=1, max_iterations=20)
        r, x, ms, times = _median_timed(_Run(lambda x: t.solve_mixed(M, b, x, tol=1e-8, inner_tol=1e-4,
                                                                     inner=inner), n))
        rec = dict(base, method=name, converged=r["converged"], iterations=r["inner_iterations"],
                   outer_iterations=r["outer_iterations"], solve_ms=ms, solve_ms_runs=times, setup_ms=setup_ms,
                   true_residual=t.true_residual(M, b, x), speedup_vs_fp64_jacobi=jac["solve_ms"] / ms)
        print(json.dumps(rec), file=out, flush=True)

    def reliable(name, inner, setup_ms, vectors=torch.float32, layout="auto"):
        # speed-up on set-up + solve against the FP64 Jacobi-PCG's set-up +
        # solve, both to a true residual below 1e-8
        t.solve_mixed_reliable(M, b, torch.zeros(n, dtype=torch.float64, device="cuda"), tol=1e-8, inner=inner,
                               max_iterations=20, vectors=vectors, layout=layout)
        r, x, ms, times = _median_timed(_Run(lambda x: t.solve_mixed_reliable(M, b, x, tol=1e-8, delta=0.3,
                                                                              inner=inner, vectors=vectors,
                                                                              layout=layout), n))
        rec = dict(base, method=name, converged=r["converged"], iterations=r["iterations"],
                   reliable_updates=r["reliable_updates"], solve_ms=ms, solve_ms_runs=times, setup_ms=setup_ms,
                   true_residual=t.true_residual(M, b, x),
                   speedup_vs_fp64_jacobi=(jac_true["solve_ms"] + jac_true["setup_ms"]) / (ms + setup_ms))
        print(json.dumps(rec), file=out, flush=True)

    # FP64 Jacobi-PCG run until its TRUE residual is below 1e-8 (the
    # reference's stopping rule uses the preconditioned residue): the
    # convergence-residue is halved until it is
    P = t.Diagonal()
    P.update(M)
    tol_j = 1e-8
    while True:
        S = t.CG()
        S.setMatrix(M)
        S.setPreconditioner(P)
        S.setConvergenceResidue(tol_j)
        S.setMaxIterations(200000)
        x = torch.zeros(n, dtype=torch.float64, device="cuda")
        S.solve(b, x)
        tr = t.true_residual(M, b, x)
        if tr < 1e-8 or tol_j < 1e-12:
            break
        tol_j *= 0.5
    ok, x, ms, times = _median_timed(_Run(lambda x: S.solve(b, x), n))
    jac_true = dict(base, method="FP64 Jacobi-PCG to true residual 1e-8", converged=bool(ok),
                    iterations=S.getIterations(), solve_ms=ms, solve_ms_runs=times, setup_ms=jac["setup_ms"],
                    true_residual=t.true_residual(M, b, x), convergence_residue=tol_j)
    print(json.dumps(jac_true), file=out, flush=True)

    mixed("FP32-inner IR, FSAI", "fsai", 0.0)
    reliable("FP32 reliable-update PCG, Jacobi", "jacobi", 0.0)
    reliable("FP32 reliable-update PCG, FSAI", "fsai", 0.0)
    reliable("FP32 reliable-update PCG, FSAI, 16-bit-offset copies", "fsai", 0.0, layout="offsets")
    reliable("FP32-matrix FP64-vector reliable-update PCG, FSAI", "fsai", 0.0, torch.float64)
    net = LearnedFSAI(seed=2)
    if weights and Path(weights).exists():
        net.load(weights)
    else:
        train = [diffusion_problem(128, s) for s in range(8)]
        net.fit_classical(train, steps=400, lr=3e-3)
        net.train(train, steps=400, nprobes=8, lr=5e-4)
    # set-up timed warm (the first call loads the network's kernels), fastest of 3
    net.preconditioner(A32)
    P32, s = _timed(lambda: net.preconditioner(A32))
    for _ in range(2):
        P32, s2 = _timed(lambda: net.preconditioner(A32))
        s = min(s, s2)
    mixed("FP32-inner IR, learned FSAI", P32, s)
    reliable("FP32 reliable-update PCG, learned FSAI", P32, s)
    reliable("FP32-matrix FP64-vector reliable-update PCG, learned FSAI", P32, s, torch.float64)


SOLVER_SWEEP = [
    ("CG", "cg", "jacobi", {}), ("BICGStab", "bicgstab", "jacobi", {}), ("TFQMR", "tfqmr", "jacobi", {}),
    ("BICGStab(2)", "bicgstabl", "jacobi", {"bicgstab-ell": 2}), ("IDR(4)", "idrs", "jacobi", {"idr-s": 4}),
    ("GMRES(30) MGSR", "gmres", "jacobi", {"gmres-variant": "MGSR"}),
    ("GMRES(30) CWY", "gmres", "jacobi", {"gmres-variant": "CWY"}),
    ("GMRES(30) MGSR", "gmres", "ilu0", {"gmres-variant": "MGSR"}),
    ("GMRES(30) MGSR", "gmres", "ilut", {"gmres-variant": "MGSR"}),
]


def bench_solver_sweep(problem: str, N: int, tol: float = 1e-8, max_iterations: int = 100000, out=sys.stdout):
    """Every Krylov solver with Jacobi (and GMRES with ILU(0) and ILUT) on one problem,
    as the reference's linear-solver benchmark does: iterations, device time of
    the solve call, set-up time of the preconditioner, true FP64 residual."""
    import tnl_b200 as t
    from . import generators as g
    from .lfsai import diffusion_problem

    if problem == "laplacian":
        M = t.SparseMatrix.from_csr(g.laplacian_2d(N))
    elif problem == "convection_diffusion":
        M = t.SparseMatrix.from_csr(g.convection_diffusion_3d(N))
    else:
        M = diffusion_problem(N, 1234)
    n = M.getRows()
    b = torch.tensor(g.uniform_vector(n, 1), device="cuda")
    classes = {"cg": t.CG, "bicgstab": t.BICGStab, "tfqmr": t.TFQMR, "bicgstabl": t.BICGStabL, "idrs": t.IDRs,
               "gmres": t.GMRES}
    precs = {"jacobi": t.Diagonal, "ilu0": t.ILU0, "ilut": t.ILUT}
    for label, kind, pname, keys in SOLVER_SWEEP:
        if kind == "cg" and problem == "convection_diffusion":
            continue  # nonsymmetric
        P = precs[pname]()
        _, setup_ms = _timed(lambda: P.update(M))
        S = classes[kind]()
        S.setMatrix(M)
        S.setPreconditioner(P)
        S.setup({"convergence-residue": tol, "max-iterations": max_iterations, "gmres-restarting-min": 30,
                 "gmres-restarting-max": 30, **keys})
        x = torch.zeros(n, dtype=torch.float64, device="cuda")
        ok, ms = _timed(lambda: S.solve(b, x))
        rec = {"bench": "solver_sweep", "problem": problem, "N": N, "rows": n, "solver": label, "precond": pname,
               "converged": bool(ok), "iterations": S.getIterations(), "solve_ms": ms, "setup_ms": setup_ms,
               "ms_per_iteration": ms / max(1, S.getIterations()), "residue": S.getResidue(),
               "true_residual": t.true_residual(M, b, x), "tol": tol}
        print(json.dumps(rec), file=out, flush=True)


def bench_configs(which: str, out=sys.stdout):
    """The mixed-precision and nonsymmetric configurations:
    c3 -- 256^3 GRF diffusion (n = 16.8M): FP32-inner Jacobi-PCG inside FP64
          refinement, and FP32 Jacobi-PCG with reliable FP64 updates, vs
          plain FP64 Jacobi-PCG, to FP64 relative residual 1e-10;
    c5 -- 192^3 upwind convection-diffusion (n = 7.1M): FGMRES(30) with the
          two-factor FSAI (FP64, and as the FP32 inner solver of FP64
          refinement) and with the learned two-factor FSAI vs plain FP64
          GMRES(30) + ILU(0), to 1e-8."""
    import tnl_b200 as t
    from . import generators as g

    if which == "c3":
        A = g.diffusion_3d(256)
        tol = 1e-10
    else:
        A = g.convection_diffusion_3d(192)
        tol = 1e-8
    M = t.SparseMatrix.from_csr(A)
    n = M.getRows()
    b = torch.tensor(g.uniform_vector(n, 1), device="cuda")
    base = {"bench": "config", "config": which, "rows": n, "nnz": A.nnz, "tol": tol}

    def report(name, conv, its, ms, setup_ms, x, **extra):
        rec = dict(base, method=name, converged=bool(conv), iterations=its, solve_ms=ms, setup_ms=setup_ms,
                   true_residual=t.true_residual(M, b, x), **extra)
        print(json.dumps(rec), file=out, flush=True)
        return rec

    def krylov(name, cls, P, keys, setup_ms=0.0, **extra):
        S = cls()
        S.setMatrix(M)
        S.setPreconditioner(P)
        S.setup({"convergence-residue": tol, "max-iterations": 20000, "gmres-restarting-min": 30,
                 "gmres-restarting-max": 30, **keys})
        x = torch.zeros(n, dtype=torch.float64, device="cuda")
        ok, ms = _timed(lambda: S.solve(b, x))
        return report(name, ok, S.getIterations(), ms, setup_ms, x, **extra)

    if which == "c3":
        # each method warmed up by a short solve, then the fastest of 3 (the
        # first call of a process loads its kernels and builds its copies)
        P = t.Diagonal()
        P.update(M)
        S = t.CG()
        S.setMatrix(M)
        S.setPreconditioner(P)
        S.setup({"convergence-residue": tol, "max-iterations": 20})
        S.solve(b, torch.zeros(n, dtype=torch.float64, device="cuda"))
        S.setup({"convergence-residue": tol, "max-iterations": 20000})
        ok, x, ms, times = _median_timed(_Run(lambda x: S.solve(b, x), n), reps=3)
        report("FP64 Jacobi-PCG", ok, S.getIterations(), ms, 0.0, x, solve_ms_runs=times)
        t.solve_mixed(M, b, torch.zeros(n, dtype=torch.float64, device="cuda"), tol=tol, inner_tol=1e-4,
                      inner="jacobi", max_outer=1, max_iterations=20)
        r, x, ms, times = _median_timed(_Run(lambda x: t.solve_mixed(M, b, x, tol=tol, inner_tol=1e-4,
                                                                     inner="jacobi", max_outer=20), n), reps=3)
        report("FP32-inner Jacobi-PCG in FP64 refinement", r["converged"], r["inner_iterations"], ms, 0.0, x,
               outer_iterations=r["outer_iterations"], solve_ms_runs=times)
        t.solve_mixed_reliable(M, b, torch.zeros(n, dtype=torch.float64, device="cuda"), tol=tol, inner="jacobi",
                               max_iterations=20)
        r, x, ms, times = _median_timed(_Run(lambda x: t.solve_mixed_reliable(M, b, x, tol=tol, delta=0.3,
                                                                              inner="jacobi"), n), reps=3)
        report("FP32 Jacobi-PCG with reliable FP64 updates", r["converged"], r["iterations"], ms, 0.0, x,
               reliable_updates=r["reliable_updates"], solve_ms_runs=times)
        # the same with the 7-diagonal copy of A read by ordinary loads
        # instead of the bulk-copy-staged product
        t.solve_mixed_reliable(M, b, torch.zeros(n, dtype=torch.float64, device="cuda"), tol=tol, inner="jacobi",
                               max_iterations=20, layout="diagonal")
        r, x, ms, times = _median_timed(_Run(lambda x: t.solve_mixed_reliable(M, b, x, tol=tol, delta=0.3,
                                                                              inner="jacobi", layout="diagonal"), n),
                                        reps=3)
        report("FP32 Jacobi-PCG with reliable FP64 updates, diagonal copy read by ordinary loads", r["converged"],
               r["iterations"], ms, 0.0, x, reliable_updates=r["reliable_updates"], solve_ms_runs=times)
        # beyond the config: the same solver with the classical FSAI of A's
        # pattern (4-diagonal factors), set-up timed apart
        A32 = t.SparseMatrix(t.CSR, torch.float32).assign(A.rowptr, A.cols, A.vals.astype(np.float32))
        Pf = t.FSAI()
        Pf.update(A32)
        Pf = t.FSAI()
        _, s_f = _timed(lambda: Pf.update(A32))
        t.solve_mixed_reliable(M, b, torch.zeros(n, dtype=torch.float64, device="cuda"), tol=tol, inner=Pf,
                               max_iterations=20)
        r, x, ms, times = _median_timed(_Run(lambda x: t.solve_mixed_reliable(M, b, x, tol=tol, delta=0.3,
                                                                              inner=Pf), n), reps=3)
        report("FP32 FSAI-PCG with reliable FP64 updates", r["converged"], r["iterations"], ms, s_f, x,
               reliable_updates=r["reliable_updates"], solve_ms_runs=times)
        return
    P = t.ILU0()
    _, s_ilu = _timed(lambda: P.update(M))
    krylov("FP64 GMRES(30) + ILU(0)", t.GMRES, P, {"gmres-variant": "MGSR"}, s_ilu)
    P = t.FSAI2()
    _, s_f2 = _timed(lambda: P.update(M))
    krylov("FP64 FGMRES(30) + two-factor FSAI", t.FGMRES, P, {"gmres-variant": "MGSR"}, s_f2)
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    r, ms = _timed(lambda: t.solve_mixed(M, b, x, tol=tol, inner_tol=1e-4, inner="fsai2", solver="fgmres",
                                         max_outer=20))
    report("FP32-inner FGMRES(30) + two-factor FSAI in FP64 refinement", r["converged"], r["inner_iterations"], ms,
           s_f2, x, outer_iterations=r["outer_iterations"])
    # the learned two-factor FSAI: trained on the spot on small problems of
    # the same family (24^3, seeds 0..7: warm start, then the probe loss on
    # Rademacher vectors and BiCGStab residuals), applied to this matrix
    from .lfsai import LearnedFSAI

    train = [t.SparseMatrix.from_csr(g.convection_diffusion_3d(24, seed=s_)) for s_ in range(8)]
    net = LearnedFSAI(seed=1, two_factor=True)
    _, train_ms = _timed(lambda: (net.fit_classical(train, steps=400, lr=3e-3),
                                  net.train(train, steps=200, nprobes=8, lr=2e-4)))
    net.preconditioner(M)
    P, s_l = _timed(lambda: net.preconditioner(M))
    krylov("FP64 FGMRES(30) + learned two-factor FSAI", t.FGMRES, P, {"gmres-variant": "MGSR"}, s_l,
           training_ms=train_ms)


def bench_c1_solves(out=sys.stdout):
    """The library's GPU solves of the reference's linear-solver benchmark
    on the 1024 x 1024 Laplacian (b ~ U[-1,1) seed 1, tolerance 1e-8 on the
    reference's residue): CG and BiCGStab with Jacobi, GMRES(30) with ILU(0)
    in the MGSR and CWY variants; CUDA-event time of one solve after a
    warm-up solve (set-up excluded, as the reference times only solve())."""
    import tnl_b200 as t
    from . import generators as g

    A = g.laplacian_2d(1024)
    M = t.SparseMatrix.from_csr(A)
    b = torch.tensor(g.uniform_vector(A.n, 1), device="cuda")
    for name, cls, pre, variant in (("CG + Jacobi", t.CG, "jacobi", "MGSR"), ("BiCGStab + Jacobi", t.BICGStab, "jacobi", "MGSR"),
                                    ("GMRES(30) MGSR + ILU(0)", t.GMRES, "ilu0", "MGSR"),
                                    ("GMRES(30) CWY + ILU(0)", t.GMRES, "ilu0", "CWY")):
        P = t.Diagonal() if pre == "jacobi" else t.ILU0()
        P.update(M)
        S = cls()
        S.setMatrix(M)
        S.setPreconditioner(P)
        S.setup({"convergence-residue": 1e-8, "max-iterations": 20000, "gmres-variant": variant,
                 "gmres-restarting-min": 30, "gmres-restarting-max": 30})
        S.solve(b, torch.zeros(A.n, dtype=torch.float64, device="cuda"))
        x = torch.zeros(A.n, dtype=torch.float64, device="cuda")
        ok, ms = _timed(lambda: S.solve(b, x))
        print(json.dumps({"bench": "c1_solve", "method": name, "converged": bool(ok), "iterations": S.getIterations(),
                          "seconds": ms / 1e3, "residue": S.getResidue(), "true_residual": t.true_residual(M, b, x)}),
              file=out, flush=True)


def profile_solvers(problem: str, N: int, iterations: int, fsai_level: int = 0, out=sys.stdout):
    """A fixed number of iterations of the FP32 reliable-update FSAI-PCG and
    of FP64 FSAI-PCG, for a kernel launch list (ncu) of both iterations;
    ``fsai_level`` 1 runs the reliable-update PCG with the classical FSAI of
    the level-1 pattern (the pattern of the learned preconditioner)."""
    import tnl_b200 as t
    from . import generators as g
    from .lfsai import diffusion_problem

    M = t.SparseMatrix.from_csr(g.laplacian_2d(N)) if problem == "laplacian" else diffusion_problem(N, 1234)
    n = M.getRows()
    b = torch.tensor(g.uniform_vector(n, 1), device="cuda")
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    inner = "fsai"
    if fsai_level:
        h = M.toHostCSR()
        A32 = t.SparseMatrix(t.CSR, torch.float32).assign(h.rowptr, h.cols, h.vals.astype(np.float32))
        inner = t.FSAI(fsai_level)
        inner.update(A32)
    r = t.solve_mixed_reliable(M, b, x, tol=1e-8, inner=inner, max_iterations=iterations)
    print(json.dumps({"method": f"FP32 reliable-update PCG, FSAI level {fsai_level}", "iterations": r["iterations"]}),
          file=out)
    P = t.FSAI()
    P.update(M)
    S = t.CG()
    S.setMatrix(M)
    S.setPreconditioner(P)
    S.setup({"convergence-residue": 1e-8, "max-iterations": iterations})
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    S.solve(b, x)
    print(json.dumps({"method": "FP64 FSAI-PCG", "iterations": S.getIterations()}), file=out)


def bench_assembly(max_grid: int = 8192, reps: int = 10, out=sys.stdout):
    """Device-side assembly of the 2D Laplace operator (the reference's
    sparse set-up benchmark, Documentation/UsersGuide/Matrices/
    SparseMatrixSetup_Benchmark.cpp: FP32, CSR, row capacities 5, then the
    stencil written on the GPU), for grid sides 16, 32, ..., max_grid: mean
    time of `reps` set-ups (setRowCapacities, storage allocation and the
    assembly kernel), CUDA events around each, after one warm-up."""
    import tnl_b200 as t

    N = 16
    while N <= max_grid:
        t.assemble_laplace_2d(N, real=torch.float32)
        torch.cuda.synchronize()
        times = []
        for _ in range(reps):
            M, ms = _timed(lambda: t.assemble_laplace_2d(N, real=torch.float32))
            times.append(ms)
            del M
        print(json.dumps({"bench": "assembly_laplace_2d", "grid": N, "rows": N * N, "real": "f32", "format": "CSR",
                          "seconds_mean": float(np.mean(times)) / 1e3, "seconds_min": float(np.min(times)) / 1e3}),
              file=out, flush=True)
        torch.cuda.empty_cache()
        N *= 2


def bench_learned_eval(count: int, N: int, weights: str, ilu_count: int = 4, first_seed: int = 10000,
                       out=sys.stdout):
    """The learned preconditioner's evaluation: `count` unseen 2D diffusion
    problems (seeds first_seed.., GRF correlation length ~ U[0.02, 0.2],
    sigma ~ U[1, 3]) on N x N grids, each solved to an FP64 true residual of
    1e-8 by
      * FP64 Jacobi-PCG (convergence residue lowered until the true
        residual is below 1e-8) -- the baseline,
      * FP32 PCG with reliable FP64 updates and the learned FSAI (network
        inference = set-up time), the classical FSAI of A's pattern, and the
        classical FSAI of the level-1 pattern,
      * FP64 ILU(0)-PCG on the first `ilu_count` problems (its level-
        scheduled triangular solves make it slow at this size);
    one JSON line per problem and method, then a summary line with the
    distribution (min / median / max) of iterations and speed-ups."""
    import tnl_b200 as t
    from . import generators as g
    from .lfsai import LearnedFSAI

    net = LearnedFSAI(seed=0)
    net.load(weights)
    rows = []
    for q in range(count):
        seed = first_seed + q
        A = g.diffusion_2d_problem(N, seed)
        M = t.SparseMatrix.from_csr(A)
        A32 = t.SparseMatrix(t.CSR, torch.float32).assign(A.rowptr, A.cols, A.vals.astype(np.float32))
        n = A.n
        b = torch.tensor(g.uniform_vector(n, 1), device="cuda")

        def zeros():
            return torch.zeros(n, dtype=torch.float64, device="cuda")

        rec = {"bench": "learned_eval", "problem": seed, "N": N}
        # FP64 Jacobi-PCG to a true residual of 1e-8
        P = t.Diagonal()
        P.update(M)
        tol = 1e-8
        while True:
            S = t.CG()
            S.setMatrix(M)
            S.setPreconditioner(P)
            S.setConvergenceResidue(tol)
            S.setMaxIterations(200000)
            x = zeros()
            ok, ms = _timed(lambda: S.solve(b, x))
            tr = t.true_residual(M, b, x)
            if tr < 1e-8 or tol < 1e-13:
                break
            tol *= 0.5 * 1e-8 / tr  # the next run's stopping residue scaled by the gap seen
        rec["fp64_jacobi"] = {"iterations": S.getIterations(), "solve_ms": ms, "converged": bool(ok),
                              "true_residual": t.true_residual(M, b, x)}

        def reliable(key, make):
            Pm, setup = make()
            t.solve_mixed_reliable(M, b, zeros(), tol=1e-8, inner=Pm, max_iterations=20)
            x = zeros()
            r, ms = _timed(lambda: t.solve_mixed_reliable(M, b, x, tol=1e-8, delta=0.3, inner=Pm))
            rec[key] = {"iterations": r["iterations"], "fallback_iterations": r["fallback_iterations"],
                        "solve_ms": ms, "setup_ms": setup,
                        "converged": bool(r["converged"]), "true_residual": t.true_residual(M, b, x),
                        "speedup_vs_fp64_jacobi": rec["fp64_jacobi"]["solve_ms"] / ms,
                        "speedup_with_setup": rec["fp64_jacobi"]["solve_ms"] / (ms + setup)}

        def learned():
            net.preconditioner(A32)
            return _timed(lambda: net.preconditioner(A32))

        def classical(level):
            def make():
                Pc = t.FSAI(level)
                _, s = _timed(lambda: Pc.update(A32))
                return Pc, s
            return make

        reliable("fp32_learned_fsai", learned)
        reliable("fp32_fsai_level0", classical(0))
        reliable("fp32_fsai_level1", classical(1))
        if q < ilu_count:
            P = t.ILU0()
            _, setup = _timed(lambda: P.update(M))
            S = t.CG()
            S.setMatrix(M)
            S.setPreconditioner(P)
            S.setConvergenceResidue(1e-8)
            S.setMaxIterations(200000)
            x = zeros()
            ok, ms = _timed(lambda: S.solve(b, x))
            rec["fp64_ilu0"] = {"iterations": S.getIterations(), "solve_ms": ms, "setup_ms": setup,
                                "converged": bool(ok), "true_residual": t.true_residual(M, b, x)}
        print(json.dumps(rec), file=out, flush=True)
        rows.append(rec)
        del M, A32
        torch.cuda.empty_cache()
    summary = {"bench": "learned_eval_summary", "problems": len(rows), "N": N}
    for key in ("fp64_jacobi", "fp32_learned_fsai", "fp32_fsai_level0", "fp32_fsai_level1", "fp64_ilu0"):
        its = [r[key]["iterations"] for r in rows if key in r]
        if not its:
            continue
        ent = {"iterations": [int(np.min(its)), float(np.median(its)), int(np.max(its))],
               "all_converged": all(r[key]["converged"] for r in rows if key in r)}
        ms = [r[key]["solve_ms"] for r in rows if key in r]
        ent["solve_ms"] = [float(np.min(ms)), float(np.median(ms)), float(np.max(ms))]
        if key.startswith("fp32"):
            sp = [r[key]["speedup_with_setup"] for r in rows]
            ent["speedup_with_setup_vs_fp64_jacobi"] = [float(np.min(sp)), float(np.median(sp)), float(np.max(sp))]
            ent["share_at_least_2x_with_setup"] = float(np.mean([v >= 2.0 for v in sp]))
            ent["fallbacks"] = int(sum(r[key]["fallback_iterations"] > 0 for r in rows))
            ent["setup_ms_median"] = float(np.median([r[key]["setup_ms"] for r in rows]))
        summary[key] = ent
    summary["learned_vs_fsai_level0_iterations_median"] = float(np.median(
        [r["fp32_learned_fsai"]["iterations"] / r["fp32_fsai_level0"]["iterations"] for r in rows]))
    print(json.dumps(summary), file=out, flush=True)
    return summary


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m tnl_b200.benchmarks")
    sub = ap.add_subparsers(dest="cmd", required=True)
    a = sub.add_parser("spmv")
    a.add_argument("--configs", default="laplacian,power_law")
    a.add_argument("--reals", default="f64,f32")
    a.add_argument("--steps", type=int, default=50)
    a.add_argument("--formats", default="", help="comma-separated labels, e.g. 'CSR default,SlicedEllpack'")
    cf = sub.add_parser("configs")
    cf.add_argument("--which", default="c3", choices=["c3", "c5"])
    sw = sub.add_parser("sweep")
    sw.add_argument("--problem", default="laplacian", choices=["laplacian", "diffusion", "convection_diffusion"])
    sw.add_argument("--N", type=int, default=1024)
    sw.add_argument("--max-iterations", type=int, default=100000)
    b = sub.add_parser("solvers")
    b.add_argument("--problem", default="laplacian", choices=["laplacian", "diffusion"])
    b.add_argument("--N", type=int, default=1024)
    b.add_argument("--weights", default=str(Path(__file__).resolve().parent / "weights" / "lfsai_diffusion.npy"))
    asm = sub.add_parser("assembly")
    asm.add_argument("--max-grid", type=int, default=8192)
    sub.add_parser("c1-solves")
    le = sub.add_parser("learned-eval")
    le.add_argument("--count", type=int, default=64)
    le.add_argument("--N", type=int, default=2048)
    le.add_argument("--ilu-count", type=int, default=4)
    le.add_argument("--weights", default=str(Path(__file__).resolve().parent / "weights" / "lfsai_diffusion.npy"))
    pr = sub.add_parser("profile-solvers")
    pr.add_argument("--problem", default="diffusion", choices=["laplacian", "diffusion"])
    pr.add_argument("--N", type=int, default=2048)
    pr.add_argument("--iterations", type=int, default=40)
    pr.add_argument("--fsai-level", type=int, default=0, choices=[0, 1])
    args = ap.parse_args(argv)
    if args.cmd == "assembly":
        bench_assembly(args.max_grid)
        return 0
    if args.cmd == "learned-eval":
        bench_learned_eval(args.count, args.N, args.weights, args.ilu_count)
        return 0
    if args.cmd == "c1-solves":
        bench_c1_solves()
        return 0
    if args.cmd == "profile-solvers":
        profile_solvers(args.problem, args.N, args.iterations, args.fsai_level)
        return 0
    if args.cmd == "configs":
        bench_configs(args.which)
        return 0
    if args.cmd == "sweep":
        bench_solver_sweep(args.problem, args.N, max_iterations=args.max_iterations)
        return 0
    if args.cmd == "spmv":
        bench_spmv(args.configs.split(","), args.reals.split(","), args.steps,
                   [f for f in args.formats.split(",") if f])
    else:
        bench_solvers(args.problem, args.N, args.weights)
    return 0


if __name__ == "__main__":
    sys.exit(main())
