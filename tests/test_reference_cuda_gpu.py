"""The reference's own CUDA SpMV on the same GPU (the secondary GPU comparison).

oracle/_ref/libtnlref_cuda.so is TNL's Devices::Cuda vectorProduct compiled
from the reference's headers for sm_100a (oracle/Makefile, oracle/ref_cuda.cu).
On the benchmark matrices at full size this test
* checks the reference's CUDA product against the oracle (1e-13 per row in
  FP64), which pins the comparison, and the library's product likewise;
* times both the same way -- mean ms per synchronous vectorProduct call
  (the reference's call ends with a stream synchronisation), CUDA events
  around back-to-back calls -- the reference under its default launch
  configuration and under every entry of its reductionLaunchConfigurations
  list, the library under its default kernel;
* prints one JSON line per matrix and format (pytest -s shows them; with
  TNLB_REPORT=<file> they are appended to that file).
Speed is reported, not asserted: the GPU is shared.
"""
import json
import os

import numpy as np
import pytest
import torch

from helpers import FORMATS, assert_spmv_close

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def refcuda():
    from oracle.oracle import REF_CUDA_SO, ReferenceCuda

    if not REF_CUDA_SO.exists():
        pytest.skip("the reference's CUDA driver oracle/_ref/libtnlref_cuda.so is not built")
    return ReferenceCuda()


def _matrix(name):
    from tnl_b200 import generators as g

    if name == "laplacian1024":
        return g.laplacian_2d(1024)
    if name == "powerlaw_zipf173":
        return g.power_law(4_194_304, 1.73, 4096, 2)
    return g.diffusion_3d(256)


def _time_sync_calls(M, x, y, reps):
    M.vectorProduct(x, y)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        M.vectorProduct(x, y)  # synchronous, as the reference's call
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


@pytest.mark.parametrize("name", ["laplacian1024", "powerlaw_zipf173", "diffusion256"])
def test_reference_cuda_spmv_against_oracle_and_timed(oracle, refcuda, name):
    import tnl_b200 as t
    from tnl_b200 import generators as g

    A = _matrix(name)
    x = g.uniform_vector(A.ncols, 0)
    seg = oracle.build(FORMATS["CSR"], A.row_lengths())
    yref = oracle.spmv(seg, A.cols, A.vals, x)
    scale = oracle.spmv(seg, A.cols, np.abs(A.vals), np.abs(x))
    nbytes = A.nnz * 12 + (A.n + 1) * 4 + A.ncols * 8 + A.n * 8
    # SlicedEllpack of the power-law matrix pads to 20.7x its nonzeros
    fmts = ("CSR",) if name == "powerlaw_zipf173" else ("CSR", "SlicedEllpack")
    for fmt in fmts:
        r = refcuda.spmv(FORMATS[fmt], A, x, reps=20)
        assert_spmv_close(r["y"], yref, scale, 1e-13)
        M = t.SparseMatrix(t.FORMATS[fmt], torch.float64).assign(A.rowptr, A.cols, A.vals)
        xs = torch.tensor(x, device="cuda")
        ys = torch.empty(A.n, dtype=torch.float64, device="cuda")
        ours = _time_sync_calls(M, xs, ys, 20)
        assert_spmv_close(ys.cpu().numpy(), yref, scale, 1e-13)
        rec = {"matrix": name, "format": fmt, "rows": A.n, "nnz": A.nnz, "algorithmic_bytes": nbytes,
               "reference_cuda_default_ms": r["ms_default"], "reference_cuda_best_ms": r["ms_best"],
               "reference_cuda_best_config": r["best"], "reference_cuda_all_ms": r["ms_all"],
               "library_default_ms": ours, "speedup_vs_reference_default": r["ms_default"] / ours,
               "speedup_vs_reference_best": r["ms_best"] / ours,
               "timing": "mean ms per synchronous call, CUDA events around 20 back-to-back calls"}
        line = json.dumps(rec)
        print(line)
        if os.environ.get("TNLB_REPORT"):
            with open(os.environ["TNLB_REPORT"], "a") as f:
                f.write(line + "\n")
        del M
        torch.cuda.empty_cache()
