"""Generate golden fixtures from the REFERENCE itself (oracle/_ref/libtnlref.so,
TNL's own Host/OpenMP code compiled from its headers).

    python tests/golden/make_golden.py

Writes tests/golden/reference_golden.npz and reference_golden.json.  Needs
the reference sources (to build oracle/_ref); the fixtures are committed so
that tests run where the reference is absent (e.g. on GPU machines).

Contents:
* builder metadata of CSR, Ellpack, SlicedEllpack, ChunkedEllpack, BiEllpack
  (column-major) and the AdaptiveCSR descriptors, for a set of seeded
  segment-size vectors (edge cases included);
* SHA-256 digests of the column/value arrays produced by the reference's
  cross-format operator= (both organizations) and the SpMV output y = A x,
  for a seeded power-law matrix and a 2D Laplacian;
* CG / BiCGStab / GMRES(30, MGSR) results (iterations, stopping residue,
  solution) with Jacobi and ILU(0) on a Laplacian and a diffusion problem.
"""
from __future__ import annotations

import hashlib
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle.oracle import (ADAPTIVE_CSR, BIELLPACK, CHUNKED_ELLPACK, CSR, ELLPACK, SLICED_ELLPACK,  # noqa: E402
                           Reference)
from tnl_b200 import generators as g  # noqa: E402

OUT = Path(__file__).resolve().parent


def size_cases() -> dict[str, np.ndarray]:
    rng = np.random.default_rng(12345)
    return {
        "empty": np.zeros(0, np.int32),
        "one": np.array([5], np.int32),
        "one_zero": np.array([0], np.int32),
        "zeros100": np.zeros(100, np.int32),
        "small37": rng.integers(0, 10, 37).astype(np.int32),
        "uniform1000": rng.integers(0, 50, 1000).astype(np.int32),
        "with_zero_rows": np.where(rng.random(3000) < 0.3, 0, g.zipf_lengths(3000, 1.73, 4096, 5)).astype(np.int32),
        "zipf173": g.zipf_lengths(5000, 1.73, 4096, 2),
        "zipf15": g.zipf_lengths(4000, 1.5, 4096, 9),
        "const33": np.full(33, 7, np.int32),
        "wide600": rng.integers(0, 3000, 600).astype(np.int32),
        "laplacian40": g.laplacian_2d(40).row_lengths(),
    }


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main() -> None:
    R = Reference()
    arrays: dict[str, np.ndarray] = {}
    meta: dict = {"builders": {}, "acsr": {}, "fill": {}, "spmv": {}, "solvers": {}}
    for name, sizes in size_cases().items():
        arrays[f"sizes/{name}"] = sizes
        for kind, kname in ((CSR, "CSR"), (ELLPACK, "Ellpack"), (SLICED_ELLPACK, "SlicedEllpack"),
                            (CHUNKED_ELLPACK, "ChunkedEllpack"), (BIELLPACK, "BiEllpack")):
            if kind == CHUNKED_ELLPACK and len(sizes) == 0:
                continue
            try:
                m = R.build(kind, sizes)
            except OverflowError:
                meta["builders"][f"{name}/{kname}"] = "overflow"
                continue
            scal = {}
            for k, v in m.items():
                if isinstance(v, np.ndarray):
                    arrays[f"build/{name}/{kname}/{k}"] = v
                else:
                    scal[k] = int(v)
            meta["builders"][f"{name}/{kname}"] = scal
        for sl in range(6):
            b = R.acsr_blocks(sizes, sl)
            if b is None:
                meta["acsr"][f"{name}/{sl}"] = "unavailable"
                continue
            for k, v in b.items():
                arrays[f"acsr/{name}/{sl}/{k}"] = v
            meta["acsr"][f"{name}/{sl}"] = int(len(b["type"]))

    mats = {"powerlaw2000": g.power_law(2000, 1.73, 300, 11), "laplacian32": g.laplacian_2d(32)}
    for mname, A in mats.items():
        arrays[f"mat/{mname}/rowptr"] = A.rowptr
        arrays[f"mat/{mname}/cols"] = A.cols
        arrays[f"mat/{mname}/vals"] = A.vals
        x = g.uniform_vector(A.ncols, 0)
        arrays[f"mat/{mname}/x"] = x
        for kind, kname in ((CSR, "CSR"), (ELLPACK, "Ellpack"), (SLICED_ELLPACK, "SlicedEllpack"),
                            (CHUNKED_ELLPACK, "ChunkedEllpack"), (BIELLPACK, "BiEllpack"), (ADAPTIVE_CSR, "AdaptiveCSR")):
            for cm in (True, False):
                for real in (np.float64, np.float32):
                    tag = f"{mname}/{kname}/{'col' if cm else 'row'}/{np.dtype(real).name}"
                    oc, ov = R.fill(kind, A, real=real, colmajor=cm)
                    meta["fill"][tag] = {"storage": int(len(oc)), "cols": digest(oc), "vals": digest(ov)}
            y, _ = R.spmv(kind, A, x, colmajor=False)
            arrays[f"spmv/{mname}/{kname}"] = y

    probs = {"laplacian32": g.laplacian_2d(32), "diffusion32": g.diffusion_2d(32, 0.1, 1.0, 3)}
    for pname, A in probs.items():
        b = g.uniform_vector(A.n, 1)
        arrays[f"prob/{pname}/rowptr"] = A.rowptr
        arrays[f"prob/{pname}/cols"] = A.cols
        arrays[f"prob/{pname}/vals"] = A.vals
        arrays[f"prob/{pname}/b"] = b
        for solver, pre in (("cg", 1), ("cg", 2), ("bicgstab", 1), ("gmres", 1), ("gmres", 2), ("gmres_cwy", 1),
                            ("gmres_cwy", 2), ("tfqmr", 1), ("tfqmr", 2), ("bicgstabl", 1), ("idrs", 1), ("idrs", 2)):
            # "gmres" is the MGSR variant, "gmres_cwy" the Householder (CWY) one;
            # BiCGStab(ell) and IDR(s) with their defaults ell = 1, s = 4
            variant = 4 if solver == "gmres_cwy" else 3
            r = R.solve(solver.split("_")[0], A, b, precond=pre, tol=1e-8, maxit=20000, gmres_m=30,
                        gmres_variant=variant)
            key = f"{pname}/{solver}/{pre}"
            meta["solvers"][key] = {"iterations": r["iterations"], "residue": r["residue"],
                                    "converged": bool(r["converged"])}
            arrays[f"solve/{key}/x"] = r["x"]
    meta["reference_threads"] = R.threads()
    np.savez_compressed(OUT / "reference_golden.npz", **arrays)
    (OUT / "reference_golden.json").write_text(json.dumps(meta, indent=1, sort_keys=True))
    print("wrote", OUT / "reference_golden.npz", sum(a.nbytes for a in arrays.values()) // 1024, "KiB raw")


if __name__ == "__main__":
    main()
