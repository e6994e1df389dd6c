"""Golden results of the REFERENCE (oracle/_ref/libtnlref.so, TNL's own
Host/OpenMP code) at the full sizes of the benchmark configurations.

    python tests/golden/make_config_golden.py

Writes tests/golden/config_golden.json (committed: GPU machines have no
reference sources).  Contents:

* builder metadata of the power-law matrices (n = 4,194,304; Zipf 1.73 and
  1.5 row lengths, cap 4096, seed 2), the 1024^2 Laplacian and the 256^3
  7-point operator, as SHA-256 digests of the reference's arrays (CSR
  offsets, SlicedEllpack slice offsets and sizes, BiEllpack permutation and
  group pointers) plus storage sizes; the reference's ChunkedEllpack storage
  count where it wraps around int32;
* Jacobi-CG on the 1024^2 Laplacian with b ~ U[-1, 1) (seed 1) to the
  reference's default stopping rule at 1e-8: iterations and residue with
  the default OpenMP thread count and with one thread, and the true
  residual ||b - A x|| / ||b|| of the reference's solution.
"""
from __future__ import annotations

import hashlib
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle.oracle import BIELLPACK, CHUNKED_ELLPACK, CSR, SLICED_ELLPACK, Reference  # noqa: E402
from tnl_b200 import generators as g  # noqa: E402

OUT = Path(__file__).resolve().parent / "config_golden.json"


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def size_vectors() -> dict[str, np.ndarray]:
    return {
        "powerlaw_zipf173": g.zipf_lengths(4_194_304, 1.73, 4096, 2),
        "powerlaw_zipf15": g.zipf_lengths(4_194_304, 1.5, 4096, 2),
        "laplacian1024": g.laplacian_2d(1024).row_lengths(),
        "diffusion256": np.full(256 ** 3, 7, np.int32) - _boundary_deficit(256),
    }


def _boundary_deficit(N: int) -> np.ndarray:
    """Missing neighbours of each cell of an N^3 grid (the 7-point rows are
    7 minus this); equal to diffusion_3d(N).row_lengths() without building
    the operator."""
    i = np.arange(N)
    edge = (i == 0).astype(np.int32) + (i == N - 1).astype(np.int32)
    return (edge[:, None, None] + edge[None, :, None] + edge[None, None, :]).reshape(-1)


def main() -> None:
    R = Reference()
    out: dict = {"builders": {}, "solves": {}, "reference_threads": R.threads()}
    for name, sizes in size_vectors().items():
        out["builders"][name] = {"segments": int(len(sizes)), "elements": int(np.sum(sizes, dtype=np.int64)),
                                 "sizes_digest": digest(sizes)}
        for kind, kname in ((CSR, "CSR"), (SLICED_ELLPACK, "SlicedEllpack"), (BIELLPACK, "BiEllpack"),
                            (CHUNKED_ELLPACK, "ChunkedEllpack")):
            m = R.build(kind, sizes)
            rec = {}
            for k, v in m.items():
                if isinstance(v, np.ndarray):
                    if kind == CHUNKED_ELLPACK:
                        continue  # only its storage count is kept
                    rec[k] = digest(v)
                else:
                    rec[k] = int(v)
            out["builders"][name][kname] = rec
        print(name, {k: v.get("storage") for k, v in out["builders"][name].items() if isinstance(v, dict)},
              flush=True)

    A = g.laplacian_2d(1024)
    b = g.uniform_vector(A.n, 1)
    for threads in (R.threads(), 1):
        R.set_threads(threads)
        r = R.solve("cg", A, b, precond=1, tol=1e-8, maxit=100000)
        x = r["x"]
        ax = np.zeros(A.n)
        rows = np.repeat(np.arange(A.n), np.diff(A.rowptr))
        np.add.at(ax, rows, A.vals * x[A.cols])
        tr = float(np.linalg.norm(b - ax) / np.linalg.norm(b))
        out["solves"][f"laplacian1024/cg/jacobi/threads{threads}"] = {
            "iterations": r["iterations"], "residue": r["residue"], "converged": bool(r["converged"]),
            "true_residual": tr, "seconds": r["seconds"], "threads": threads}
        print(threads, out["solves"][f"laplacian1024/cg/jacobi/threads{threads}"], flush=True)
    OUT.write_text(json.dumps(out, indent=1, sort_keys=True))
    print("wrote", OUT)


if __name__ == "__main__":
    main()
