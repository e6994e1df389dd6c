"""Shared test helpers: golden fixtures and the SpMV tolerance rule."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np

GOLDEN_DIR = Path(__file__).resolve().parent / "golden"

# Format ids shared by the oracle, the reference driver and the C ABI.
FORMATS = {"CSR": 0, "Ellpack": 1, "SlicedEllpack": 2, "ChunkedEllpack": 3, "BiEllpack": 4, "AdaptiveCSR": 5}


class Golden:
    """Fixtures produced by the reference itself (tests/golden/make_golden.py)."""

    def __init__(self):
        self.arrays = np.load(GOLDEN_DIR / "reference_golden.npz")
        self.meta = json.loads((GOLDEN_DIR / "reference_golden.json").read_text())

    def get(self, key):
        return self.arrays[key]

    def has(self, key):
        return key in self.arrays.files

    def size_cases(self):
        return sorted(k.split("/", 1)[1] for k in self.arrays.files if k.startswith("sizes/"))


def row_abs_sums(rowptr, cols, vals, x):
    """sum_j |a_ij x_j| per row (padding -1 ignored), in float64."""
    c = np.asarray(cols)
    keep = c >= 0
    prod = np.zeros(len(c))
    prod[keep] = np.abs(np.asarray(vals, np.float64)[keep] * np.asarray(x, np.float64)[c[keep]])
    out = np.zeros(len(rowptr) - 1)
    rows = np.repeat(np.arange(len(rowptr) - 1), np.diff(rowptr))
    np.add.at(out, rows, prod)
    return out


def assert_spmv_close(y, y_ref, scale, rtol):
    """|y - y_ref| <= rtol * max(|y_ref|, scale) per row.

    ``scale`` is sum_j |alpha a_ij x_j| + |beta y0_i| for the row: the bound
    on reordering a sum of those terms.  The tolerance is 1e-13 for FP64
    (only the reduction order differs from the Host path) and 2e-5 for FP32.
    """
    y = np.asarray(y, np.float64)
    y_ref = np.asarray(y_ref, np.float64)
    bound = rtol * np.maximum(np.abs(y_ref), scale) + 1e-300
    err = np.abs(y - y_ref)
    bad = np.nonzero(err > bound)[0]
    assert bad.size == 0, (f"{bad.size} rows outside tolerance; first {bad[:5]}: got {y[bad[:5]]}, "
                           f"expected {y_ref[bad[:5]]}, bound {bound[bad[:5]]}")


def fp32_singular_laplacian(N, eps=1e-7):
    """The graph Laplacian of an N x N grid (Neumann rows: diagonal = degree
    2, 3 or 4) plus eps I: SPD in FP64, but eps vanishes when the values are
    rounded to FP32, which leaves the singular Laplacian.  With a right-hand
    side whose mean is not zero, CG on the FP32 values cannot reduce the
    constant component of the residual."""
    import scipy.sparse as sp
    from tnl_b200 import generators as g

    T = sp.diags([-np.ones(N - 1), np.r_[1.0, 2.0 * np.ones(N - 2), 1.0], -np.ones(N - 1)], [-1, 0, 1])
    E = sp.identity(N)
    A = (sp.kron(T, E) + sp.kron(E, T) + eps * sp.identity(N * N)).tocsr()
    A.sort_indices()
    return g.CSRMatrix(A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data.astype(np.float64))


def nonzero_mean_rhs(n, seed=1, mean=1e-3):
    """Standard normal entries shifted to the given mean."""
    b = np.random.default_rng(seed).standard_normal(n)
    return b - b.mean() + mean
