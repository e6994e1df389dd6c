"""The seeded matrix generators produce the same workloads on every machine.

Every measured number of this library (the SpMV bench, the solver configs,
the learned-preconditioner evaluation) is taken on matrices made by
tnl_b200/generators.py from fixed seeds, so a change to a generator would
change the workload under the same name.  These digests pin them: the
index arrays and the hash-based values exactly (SHA-256 prefixes), the
values that go through numpy's FFT (the Gaussian random fields of the
diffusion and convection-diffusion operators) by their sums to 1e-12.
"""
import hashlib

import numpy as np
import pytest

from tnl_b200 import generators as g


def _d(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()[:16]


def test_power_law_and_vectors_are_pinned():
    A = g.power_law(20000, 1.73, 4096, 2)
    assert (A.n, A.nnz) == (20000, 319011)
    assert (_d(A.rowptr), _d(A.cols), _d(A.vals)) == ("abfa53f89577e300", "a37ba7405d52f148", "7eb6f96952023603")
    assert _d(g.uniform_vector(20000, 0)) == "a216e9f09cec1242"


def test_stencil_operators_are_pinned():
    L = g.laplacian_2d(64)
    assert (L.n, L.nnz, _d(L.rowptr), _d(L.cols), _d(L.vals)) == (
        4096, 20224, "0b827ef1db7cc068", "b676d0fc27b5eca5", "71d80f0e60471d81")
    for A, n, nnz, rp, cols, s, sa in (
            (g.diffusion_2d_problem(64, 1234), 4096, 20224, "0b827ef1db7cc068", "b676d0fc27b5eca5",
             840.8027543411092, 55503.90529946925),
            (g.convection_diffusion_3d(12), 1728, 11232, "f1662c165b8b648c", "1f36f34f5b7f67c2",
             3469993.2142186146, 79318581.11212125),
            (g.diffusion_3d(16), 4096, 27136, "15e75219f2a5fc44", "313e204f814fc0dc",
             22947.686977049434, 185289.07477259176)):
        assert (A.n, A.nnz, _d(A.rowptr), _d(A.cols)) == (n, nnz, rp, cols)
        assert float(A.vals.sum()) == pytest.approx(s, rel=1e-12)
        assert float(np.abs(A.vals).sum()) == pytest.approx(sa, rel=1e-12)


def test_bench_matrix_is_pinned():
    """The SpMV bench's matrix: 4,194,304 rows, Zipf 1.73 row lengths capped
    at 4096, seed 2."""
    B = g.power_law(4_194_304, 1.73, 4096, 2)
    assert (B.n, B.nnz) == (4_194_304, 67_106_293)
    assert _d(B.rowptr) == "2cf68d8d787835d1"
    assert _d(B.cols[:1_000_000]) == "e8b08815de848d05"
