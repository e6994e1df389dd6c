"""tnlb_spmv_csr_noalloc (CSR SpMV with its scratch in a static device array)
against tnlb_spmv with the tile kernel on CSR segments: the same kernels and tile plan, so
the results must be bit-identical, on two calls in a row that reuse the
scratch without any reset.  Collected last so that it also runs after every
other GPU test in the same process."""
import numpy as np
import pytest
import scipy.sparse
import torch

pytestmark = pytest.mark.gpu

LIMIT = 262144 * 256  # rows + nonzeros the static scratch holds


def _noalloc(M, x, y, alpha, beta):
    import tnl_b200
    from tnl_b200 import _capi as capi

    rowptr = torch.as_tensor(M.segments.getOffsets(), dtype=torch.int32, device="cuda")
    cols, vals = M.getColumnIndexes(), M.getValues()
    real = capi.F64 if vals.dtype == torch.float64 else capi.F32
    st = torch.cuda.current_stream().cuda_stream
    tnl_b200.check(capi.tnlb_spmv_csr_noalloc(real, M.getRows(), M.getColumns(), cols.numel(), rowptr.data_ptr(),
                                              cols.data_ptr(), vals.data_ptr(), x.data_ptr(), y.data_ptr(),
                                              float(alpha), float(beta), st))
    torch.cuda.current_stream().synchronize()


def _matrices():
    from tnl_b200 import generators as g

    yield "power_law", g.power_law(300_000)  # rows up to 4096 nonzeros: rows split across tiles
    A = g.power_law(50_000, seed=7)
    keep = np.repeat(np.arange(A.n) % 3 != 0, np.diff(A.rowptr))  # every third row empty
    lens = np.where(np.arange(A.n) % 3 != 0, np.diff(A.rowptr), 0)
    rowptr = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    yield "power_law_empty_rows", g.CSRMatrix(rowptr, A.cols[keep], A.vals[keep], A.ncols)
    yield "laplacian_2d", g.laplacian_2d(300)


@pytest.mark.parametrize("real", [torch.float64, torch.float32])
@pytest.mark.parametrize("alpha,beta", [(1.0, 0.0), (2.5, -0.5)])
def test_noalloc_matches_tnlb_spmv_twice(real, alpha, beta):
    import tnl_b200
    from tnl_b200 import generators as g

    for name, A in _matrices():
        M = tnl_b200.SparseMatrix.from_csr(A, tnl_b200.CSR, real)
        x = torch.tensor(g.uniform_vector(M.getColumns(), 11), dtype=real, device="cuda")
        y0 = torch.tensor(g.uniform_vector(M.getRows(), 12), dtype=real, device="cuda")
        y_ref = y0.clone()
        M.vectorProduct(x, y_ref, alpha, beta, launchConfig=tnl_b200.LaunchConfiguration("Tile"))
        for call in range(2):
            y = y0.clone()
            _noalloc(M, x, y, alpha, beta)
            assert torch.equal(y, y_ref), (name, call, (y - y_ref).abs().max().item())
        # and the product itself is right (FP64 host product, loose bound)
        S = scipy.sparse.csr_matrix((A.vals.astype(np.float64), A.cols, A.rowptr), shape=(M.getRows(), M.getColumns()))
        xh, y0h = x.double().cpu().numpy(), y0.double().cpu().numpy()
        ref = alpha * (S @ xh) + beta * y0h
        scale = abs(S) @ np.abs(xh)
        tol = (1e-12 if real == torch.float64 else 1e-4) * (abs(alpha) * scale + abs(beta) * np.abs(y0h))
        assert np.all(np.abs(y.double().cpu().numpy() - ref) <= tol), name


def test_noalloc_rejects_sizes_above_the_scratch():
    import tnl_b200
    from tnl_b200 import _capi as capi

    # rejected on the host before any pointer is used or any kernel launched
    with pytest.raises(ValueError, match="static scratch limit"):
        tnl_b200.check(capi.tnlb_spmv_csr_noalloc(capi.F64, 1, 1, LIMIT, None, None, None, None, None, 1.0, 0.0,
                                                  None))
    with pytest.raises(ValueError, match="negative size"):
        tnl_b200.check(capi.tnlb_spmv_csr_noalloc(capi.F64, -1, 1, 0, None, None, None, None, None, 1.0, 0.0, None))
    # zero rows: nothing to do
    tnl_b200.check(capi.tnlb_spmv_csr_noalloc(capi.F32, 0, 0, 0, None, None, None, None, None, 1.0, 0.0, None))
