"""Learned FSAI preconditioner: the network handle, its training loop and
the preconditioner it produces (no counterpart in the reference library).

The network and every kernel it runs live in libtnlb200.so (lfsai.cu):
features, forward and backward passes, the probe loss built from the
library's SpMVs, and Adam.  This module only orchestrates them:

* ``LearnedFSAI.fit_classical`` -- warm start: regress the network onto the
  classical Kolotilina-Yeremin FSAI values of the training matrices (on the
  lower triangle of A; zero on the fill entries of the default, wider
  pattern -- the lower triangle of the pattern of A^2);
* ``LearnedFSAI.train_kaporin`` -- minimise the Kaporin loss
  log(trace(G A G^T)/n) - (2/n) sum_i log G_ii (exact, no probes), the
  log of Kaporin's condition number, which bounds CG's iteration count;
* ``LearnedFSAI.train`` -- minimise (1/(n P)) sum_p ||z_p - G A G^T z_p||^2
  over probe vectors z_p: Rademacher vectors and residuals left by a few
  Jacobi-PCG iterations on the same matrix (the error modes a cheap
  preconditioner leaves behind);
* ``LearnedFSAI.preconditioner(M)`` -- M^-1 = G^T G for a matrix, usable by
  the solvers and by the mixed-precision refinement (FP32 matrices give an
  FP32 preconditioner).
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np
import torch

from . import BICGStab, CG, Diagonal, SparseMatrix, _real_code, _stream, check
from . import _capi as capi
from ._capi import lib  # noqa: F401  (fails loudly without the library)


class LearnedPreconditioner:
    """M^-1 = G^T G with G from the network (a tnlb_precond handle)."""

    KIND = capi.PRECOND_FSAI

    def __init__(self, handle, matrix):
        self._h = handle
        self.matrix = matrix

    @property
    def handle(self):
        return self._h

    def solve(self, b: torch.Tensor, x: torch.Tensor) -> None:
        check(capi.tnlb_precond_solve(self._h, b.data_ptr(), x.data_ptr(), _stream()))

    def __del__(self):
        try:
            if self._h:
                capi.tnlb_precond_destroy(self._h)
        except Exception:
            pass


class LearnedFSAI:
    """The network handle.  ``level`` picks G's pattern: 1 (default) the
    lower triangle of the pattern of A^2, 0 the lower triangle of A (at most
    8 entries per row either way).  ``two_factor=True`` is the form for a
    nonsymmetric A: G_L and G_U on A's own pattern, M^-1 = G_U G_L (used
    by FGMRES).  The dense layers run on tcgen05 tensor cores unless
    ``tensor_cores=False`` (CUDA cores)."""

    NPARAMS = 10952
    FEATURES, OUTPUTS = 32, 8

    def __init__(self, seed: int = 0, tensor_cores: bool = True, level: int = 1, two_factor: bool = False):
        h = C.c_void_p()
        check(capi.tnlb_lfsai_create(seed, _stream(), C.byref(h)))
        self._h = h
        self.set_tensor_cores(tensor_cores)
        self.set_level(level)
        check(capi.tnlb_lfsai_set_two_factor(self._h, int(bool(two_factor))))
        self.two_factor = bool(two_factor)

    def __del__(self):
        try:
            if self._h:
                capi.tnlb_lfsai_destroy(self._h)
        except Exception:
            pass

    def set_tensor_cores(self, enable: bool) -> None:
        check(capi.tnlb_lfsai_set_tensor_cores(self._h, int(bool(enable))))

    def set_level(self, level: int) -> None:
        check(capi.tnlb_lfsai_set_level(self._h, int(level)))
        self.level = int(level)

    # -- parameters ---------------------------------------------------------
    def params(self) -> np.ndarray:
        out = np.zeros(self.NPARAMS, np.float32)
        check(capi.tnlb_lfsai_get_params(self._h, out.ctypes.data, out.size))
        return out

    def set_params(self, theta) -> None:
        t = np.ascontiguousarray(theta, np.float32)
        check(capi.tnlb_lfsai_set_params(self._h, t.ctypes.data, t.size))

    def grad(self) -> np.ndarray:
        out = np.zeros(self.NPARAMS, np.float32)
        check(capi.tnlb_lfsai_get_grad(self._h, out.ctypes.data, out.size))
        return out

    def save(self, path) -> None:
        np.save(Path(path), self.params())

    def load(self, path) -> None:
        self.set_params(np.load(Path(path)))

    # -- evaluation -------------------------------------------------------------
    def evaluate(self, M: SparseMatrix):
        """(features n x 32, outputs n x 8) of a matrix."""
        n = M.getRows()
        f = np.zeros((n, self.FEATURES), np.float32)
        o = np.zeros((n, self.OUTPUTS), np.float32)
        check(capi.tnlb_lfsai_eval(self._h, M.segments.handle, _real_code(M.real), M.columnIndexes.data_ptr(),
                                   M.values.data_ptr(), _stream(), f.ctypes.data, o.ctypes.data))
        return f, o

    def preconditioner(self, M: SparseMatrix) -> LearnedPreconditioner:
        h = C.c_void_p()
        check(capi.tnlb_lfsai_precond_create(self._h, M.segments.handle, _real_code(M.real),
                                             M.columnIndexes.data_ptr(), M.values.data_ptr(), _stream(), C.byref(h)))
        return LearnedPreconditioner(h, M)

    # -- training ---------------------------------------------------------------
    def gradient(self, M: SparseMatrix, probes: torch.Tensor | None = None, mode: int = 0) -> float:
        """Loss of one matrix; the gradient stays in the handle (see grad()).
        mode 0: probe loss (probes required), 1: warm start, 2: Kaporin."""
        loss = C.c_double()
        nprobes = 0 if probes is None else probes.shape[0]
        check(capi.tnlb_lfsai_gradient(self._h, mode, M.segments.handle, _real_code(M.real),
                                       M.columnIndexes.data_ptr(), M.values.data_ptr(),
                                       probes.data_ptr() if probes is not None else None, nprobes, _stream(),
                                       C.byref(loss)))
        return loss.value

    def adam_step(self, lr: float) -> None:
        check(capi.tnlb_lfsai_adam_step(self._h, lr, _stream()))

    def fit_classical(self, matrices, steps: int = 300, lr: float = 3e-3) -> list[float]:
        hist = []
        for k in range(steps):
            M = matrices[k % len(matrices)]
            hist.append(self.gradient(M, None, mode=1))
            self.adam_step(lr)
        return hist

    def train_kaporin(self, matrices, steps: int = 300, lr: float = 1e-3) -> list[float]:
        """Adam on the Kaporin loss, cycling over the training matrices."""
        hist = []
        for k in range(steps):
            M = matrices[k % len(matrices)]
            hist.append(self.gradient(M, None, mode=2))
            self.adam_step(lr)
        return hist

    @staticmethod
    def probes(M: SparseMatrix, count: int, seed: int, residual_share: float = 0.5, pcg_iterations: int = 20,
               symmetric: bool = True):
        """Probe vectors (count x n): Rademacher, and unit-RMS residuals left by a
        few Jacobi-PCG iterations (Jacobi-BiCGStab for a nonsymmetric matrix)
        from x = 0 on Rademacher right-hand sides."""
        n = M.getRows()
        g = torch.Generator(device="cuda")
        g.manual_seed(seed)
        Z = (torch.randint(0, 2, (count, n), generator=g, device="cuda", dtype=torch.int8).to(M.real) * 2 - 1)
        nres = int(round(count * residual_share))
        if nres:
            S = CG() if symmetric else BICGStab()
            S.setMatrix(M)
            P = Diagonal()
            P.update(M)
            S.setPreconditioner(P)
            S.setMaxIterations(pcg_iterations)
            S.setConvergenceResidue(0.0)
            for p in range(nres):
                b = Z[p].clone()
                x = torch.zeros(n, dtype=M.real, device="cuda")
                S.solve(b, x)
                r = b.clone()
                M.vectorProduct(x, r, -1.0, 1.0)
                Z[p] = r * (n ** 0.5 / torch.linalg.vector_norm(r))
        return Z.contiguous()

    def train(self, matrices, steps: int = 500, nprobes: int = 8, lr: float = 1e-3, seed: int = 0,
              probe_cache: int = 8) -> list[float]:
        """Adam on the probe loss, cycling over the training matrices; each
        matrix keeps a few probe sets that are reused before new ones are drawn."""
        hist = []
        cache: dict[int, torch.Tensor] = {}
        for k in range(steps):
            idx = k % len(matrices)
            M = matrices[idx]
            if idx not in cache or (k // len(matrices)) % probe_cache == 0:
                cache[idx] = self.probes(M, nprobes, seed + 7919 * k + idx, symmetric=not self.two_factor)
            hist.append(self.gradient(M, cache[idx], mode=0))
            self.adam_step(lr)
        return hist


def diffusion_problem(N: int, seed: int, corr_range=(0.02, 0.2), sigma_range=(1.0, 3.0)) -> SparseMatrix:
    """One seeded 2D diffusion matrix of the learned-preconditioner workload:
    correlation length ~ U[corr_range], sigma ~ U[sigma_range]."""
    from .generators import diffusion_2d_problem

    return SparseMatrix.from_csr(diffusion_2d_problem(N, seed, corr_range, sigma_range), real=torch.float64)


def main(argv=None):
    """Train the learned FSAI on seeded 2D diffusion problems and save the
    weights (float32, 10952 values, level-1 pattern):

        python -m tnl_b200.lfsai --out tnl_b200/weights/lfsai_diffusion.npy

    The default training set is the learned-preconditioner workload: 512
    problems on 256 x 256 grids, k = exp(g) with g a Gaussian random field of
    correlation length ~ U[0.02, 0.2] and sigma ~ U[1, 3] (seeds 0..511).
    Phases: warm start on classical FSAI of A's own pattern, the Kaporin
    loss on the level-1 pattern, then (``--probe-steps``) the probe loss on
    Rademacher vectors and residuals left by the solver.  A held-out problem
    (seed 100000) is solved by FP64 PCG after each phase; its iteration
    counts go to the JSON summary printed at the end.
    """
    import argparse
    import json
    import sys
    import time

    from . import FSAI
    from .generators import uniform_vector

    ap = argparse.ArgumentParser(prog="python -m tnl_b200.lfsai")
    ap.add_argument("--out", required=True)
    ap.add_argument("--N", type=int, default=256, help="grid side of the training problems")
    ap.add_argument("--problems", type=int, default=512)
    ap.add_argument("--fit-steps", type=int, default=1024)
    ap.add_argument("--kaporin-steps", type=int, default=2048)
    ap.add_argument("--probe-steps", type=int, default=0)
    ap.add_argument("--seed", type=int, default=2)
    ap.add_argument("--validate-N", type=int, default=512)
    args = ap.parse_args(argv)
    t0 = time.perf_counter()
    train = [diffusion_problem(args.N, s) for s in range(args.problems)]
    t_gen = time.perf_counter() - t0
    val = diffusion_problem(args.validate_N, 100000)
    b = torch.tensor(uniform_vector(val.getRows(), 1), device="cuda")

    def iterations(P):
        S = CG()
        S.setMatrix(val)
        S.setPreconditioner(P)
        S.setConvergenceResidue(1e-8)
        S.setMaxIterations(100000)
        x = torch.zeros(val.getRows(), dtype=torch.float64, device="cuda")
        S.solve(b, x)
        return S.getIterations()

    record = {"problems": args.problems, "N": args.N, "generation_s": t_gen}
    for level in (0, 1):
        P = FSAI(level)
        P.update(val)
        record[f"validation_classical_fsai_level{level}"] = iterations(P)
    net = LearnedFSAI(seed=args.seed)
    t1 = time.perf_counter()
    fit = net.fit_classical(train, steps=args.fit_steps, lr=3e-3)
    record["fit_loss"] = [fit[0], float(np.mean(fit[-16:]))]
    record["validation_warm_start"] = iterations(net.preconditioner(val))
    kap = net.train_kaporin(train, steps=args.kaporin_steps, lr=1e-3)
    record["kaporin_loss"] = [float(np.mean(kap[:16])), float(np.mean(kap[-16:]))]
    record["validation_after_kaporin"] = iterations(net.preconditioner(val))
    if args.probe_steps:
        hist = net.train(train, steps=args.probe_steps, nprobes=8, lr=2e-4)
        record["probe_loss"] = [float(np.mean(hist[:16])), float(np.mean(hist[-16:]))]
        record["validation_after_probe"] = iterations(net.preconditioner(val))
    torch.cuda.synchronize()
    record["training_s"] = time.perf_counter() - t1
    Path(args.out).parent.mkdir(parents=True, exist_ok=True)
    net.save(args.out)
    record["out"] = str(args.out)
    print(json.dumps(record), file=sys.stdout)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
