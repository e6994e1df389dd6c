"""Known-answer SpMV cases of the reference's unit tests, restated as data.

Source: src/UnitTests/Matrices/SparseMatrixVectorProductTest.hpp (TNL 0.4.0).
Each case gives a CSR matrix, the input vector, the expected output and the
initial output vector (beta = 0, so it is overwritten).
"""
from __future__ import annotations

import numpy as np


def _from_triplets(rows, cols_n, triplets, capacities=None):
    """CSR arrays from (row, col, value) triplets; extra capacity is padding (-1, 0)."""
    per_row = [[] for _ in range(rows)]
    for r, c, v in triplets:
        per_row[r].append((c, v))
    caps = capacities or [len(p) for p in per_row]
    rowptr = np.zeros(rows + 1, np.int32)
    rowptr[1:] = np.cumsum(caps)
    cols = np.full(rowptr[-1], -1, np.int32)
    vals = np.zeros(rowptr[-1], np.float64)
    for r, p in enumerate(per_row):
        for k, (c, v) in enumerate(sorted(p)):
            cols[rowptr[r] + k] = c
            vals[rowptr[r] + k] = v
    return rowptr, cols, vals, cols_n


def cases():
    out = []
    # zeroMatrix (:16-74): capacities [1,2,1,1], all padding, x = 1, y0 = -1 -> 0
    rp, c, v, nc = _from_triplets(4, 4, [], capacities=[1, 2, 1, 1])
    out.append(("zeroMatrix", rp, c, v, nc, np.ones(4), np.full(4, -1.0), np.zeros(4)))
    # smallMatrix1 (:78-137)
    rp, c, v, nc = _from_triplets(4, 4, [(0, 0, 1), (1, 1, 2), (1, 3, 3), (2, 1, 4), (3, 2, 5)])
    out.append(("smallMatrix1", rp, c, v, nc, np.full(4, 2.0), np.zeros(4), np.array([2, 10, 8, 10.0])))
    # smallMatrix2 (:141-199)
    rp, c, v, nc = _from_triplets(4, 4, [(0, 0, 1), (0, 1, 2), (0, 2, 3), (1, 3, 4), (2, 0, 5), (2, 1, 6), (2, 2, 7),
                                         (3, 1, 8)])
    out.append(("smallMatrix2", rp, c, v, nc, np.full(4, 2.0), np.zeros(4), np.array([12, 8, 36, 16.0])))
    # smallMatrix3 (:203-267)
    rp, c, v, nc = _from_triplets(4, 4, [(0, 0, 1), (0, 1, 2), (0, 2, 3), (1, 1, 4), (1, 2, 5), (1, 3, 6), (2, 0, 7),
                                         (2, 1, 8), (2, 2, 9), (3, 1, 10), (3, 2, 11), (3, 3, 12)])
    out.append(("smallMatrix3", rp, c, v, nc, np.full(4, 2.0), np.zeros(4), np.array([12, 30, 48, 66.0])))
    # largeMatrix (:422-497): diagonal y_i = i+1, lower-triangular y_i = (i+1)(i+2)/2
    n = 1051
    rp, c, v, nc = _from_triplets(n, n, [(i, i, i + 1.0) for i in range(n)])
    out.append(("largeMatrix_diag", rp, c, v, nc, np.ones(n), np.zeros(n), np.arange(1, n + 1, dtype=np.float64)))
    tri = [(r, k, k + 1.0) for r in range(n) for k in range(r + 1)]
    rp, c, v, nc = _from_triplets(n, n, tri)
    out.append(("largeMatrix_lower", rp, c, v, nc, np.ones(n), np.zeros(n),
                np.array([(i + 1) * (i + 2) / 2 for i in range(n)], np.float64)))
    # longRowsMatrix (:499-533): 33 rows, values localIdx+row at column localIdx
    for columns in (64, 65, 128, 129, 256, 257, 512, 513, 1024, 1025, 2048, 2049, 3000):
        rows = 33
        trip = [(r, k, float(k + r)) for r in range(rows) for k in range(columns)]
        rp, c, v, nc = _from_triplets(rows, columns, trip)
        exp = np.array([columns * (columns - 1) / 2.0 + columns * r for r in range(rows)])
        out.append((f"longRows_{columns}", rp, c, v, nc, np.ones(columns), np.zeros(rows), exp))
    return out
