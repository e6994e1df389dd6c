"""Row-block distribution of a sparse matrix (TNL::Matrices::DistributedMatrix).

CPU (gloo, world size 2, run here): the row split of splitRange, the ghost
columns and their remapping, the exchange of the request lists and of the
ghost values among real ranks; the local products are checked with scipy
on each rank's remapped columns.

GPU (one device): the two ranks' local matrices built from the same plans
and multiplied by the library's SpMV after an emulated exchange (the values
one rank sends are the other's ghosts), against the global product; the
DistributedMatrix / DistributedCG classes themselves on a world of one rank
(NCCL), against the single-GPU solver's iteration count.
"""
import os
import socket

import numpy as np
import pytest
import torch


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_split_range_matches_the_reference_rule():
    from tnl_b200.distributed import split_range

    # the first size % parts ranks take one row more (BlockPartitioning.h:27-40)
    assert [split_range(10, r, 3) for r in range(3)] == [(0, 4), (4, 7), (7, 10)]
    assert [split_range(7, r, 7) for r in range(7)] == [(r, r + 1) for r in range(7)]
    assert [split_range(2, r, 3) for r in range(3)] == [(0, 1), (1, 2), (2, 2)]


def _laplacian(N):
    from tnl_b200 import generators as g

    return g.laplacian_2d(N)


def _local_rows(A, b, e):
    rp = A.rowptr[b:e + 1] - A.rowptr[b]
    return rp.astype(np.int32), A.cols[A.rowptr[b]:A.rowptr[e]], A.vals[A.rowptr[b]:A.rowptr[e]]


def test_halo_plan_ghosts_and_remap():
    """On a 2D Laplacian split in two, rank 0's ghosts are the first grid
    row of rank 1 and vice versa; remapped columns index [x_local, x_ghost]."""
    from tnl_b200.distributed import HaloPlan, split_range

    N = 8
    A = _laplacian(N)
    ranges = [split_range(A.n, r, 2) for r in range(2)]
    plans = []
    for r, (b, e) in enumerate(ranges):
        _, cols, _ = _local_rows(A, b, e)
        plans.append(HaloPlan(cols, r, ranges))
    assert np.array_equal(plans[0].ghosts, np.arange(32, 40))
    assert np.array_equal(plans[1].ghosts, np.arange(24, 32))
    assert list(plans[0].recv_counts) == [0, 8] and list(plans[1].recv_counts) == [8, 0]
    for r, P in enumerate(plans):
        b, e = ranges[r]
        _, cols, _ = _local_rows(A, b, e)
        own = P.local_cols < P.n_local
        back = np.empty_like(P.local_cols, dtype=np.int64)
        back[own] = P.local_cols[own] + b
        back[~own] = P.ghosts[P.local_cols[~own] - P.n_local]
        assert np.array_equal(back, cols)
    # the send lists are what the other rank requests
    plans[0].set_send_lists([np.zeros(0, np.int64), plans[1].requests()[0]])
    assert np.array_equal(plans[0].send_idx, np.arange(24, 32))
    with pytest.raises(ValueError):
        plans[0].set_send_lists([np.zeros(0, np.int64), np.array([40])])


def _gloo_worker(rank, world, port, N, q):
    import torch.distributed as dist
    import scipy.sparse as sp

    from tnl_b200.distributed import build_plan, split_range

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from tnl_b200 import generators as g

        A = g.laplacian_2d(N)
        b, e = split_range(A.n, rank, world)
        rp, cols, vals = _local_rows(A, b, e)
        plan = build_plan(cols, None, "cpu", A.n)
        x = g.uniform_vector(A.n, 0)
        xl = torch.tensor(x[b:e])
        send = xl.index_select(0, torch.tensor(plan.send_idx))
        recv = torch.empty(plan.n_ghost, dtype=torch.float64)
        dist.all_to_all_single(recv, send, [int(c) for c in plan.recv_counts], [int(c) for c in plan.send_counts])
        xe = np.concatenate([x[b:e], recv.numpy()])
        ok_ghosts = np.array_equal(recv.numpy(), x[plan.ghosts])
        L = sp.csr_matrix((vals, plan.local_cols, rp), shape=(e - b, plan.n_local + plan.n_ghost))
        G = sp.csr_matrix((A.vals, A.cols, A.rowptr), shape=(A.n, A.n))
        ok_product = np.allclose(L @ xe, (G @ x)[b:e], rtol=1e-14, atol=1e-14)
        q.put((rank, ok_ghosts, ok_product, plan.n_ghost))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_halo_exchange_with_gloo_ranks(world):
    """world_size 2 and 3 gloo ranks on the CPU: the plan's request lists
    and the ghost values go through all-to-all collectives; every rank's
    ghosts equal x at its ghost columns and its local product the global
    product's rows."""
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gloo_worker, args=(r, world, port, 12, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ok_ghosts, ok_product, n_ghost in res:
        assert ok_ghosts and ok_product, rank
        assert n_ghost > 0


@pytest.mark.gpu
def test_two_rank_local_products_on_one_gpu(oracle):
    """Both ranks' local matrices (remapped ghost columns) multiplied by the
    library's SpMV after an emulated exchange equal the global product."""
    import tnl_b200 as t
    from tnl_b200 import generators as g
    from tnl_b200.distributed import HaloPlan, split_range

    from helpers import FORMATS, assert_spmv_close

    A = g.power_law(50_000, 1.73, 4096, 5)
    x = g.uniform_vector(A.n, 0)
    seg = oracle.build(FORMATS["CSR"], A.row_lengths())
    yref = oracle.spmv(seg, A.cols, A.vals, x)
    scale = oracle.spmv(seg, A.cols, np.abs(A.vals), np.abs(x))
    world = 2
    ranges = [split_range(A.n, r, world) for r in range(world)]
    plans = [HaloPlan(_local_rows(A, b, e)[1], r, ranges) for r, (b, e) in enumerate(ranges)]
    for r, P in enumerate(plans):
        P.set_send_lists([plans[p].requests()[r] for p in range(world)])
    xs = torch.tensor(x, device="cuda")
    y = np.zeros(A.n)
    for r, (b, e) in enumerate(ranges):
        P = plans[r]
        rp, _, vals = _local_rows(A, b, e)
        M = t.SparseMatrix(t.CSR, torch.float64).assign(rp, P.local_cols, vals, P.n_local + P.n_ghost)
        # the values rank r receives are what each owner sends it
        parts = []
        for p in range(world):
            bp, _ = ranges[p]
            req = plans[r].requests()[p]
            parts.append(xs[bp:][torch.tensor(req - bp, device="cuda")] if len(req) else xs[:0])
        xe = torch.cat([xs[b:e]] + parts)
        ys = torch.empty(e - b, dtype=torch.float64, device="cuda")
        M.vectorProduct(xe, ys)
        y[b:e] = ys.cpu().numpy()
    assert_spmv_close(y, yref, scale, 1e-13)


@pytest.mark.gpu
def test_distributed_cg_on_one_rank_matches_cg():
    """DistributedMatrix + DistributedCG with an NCCL group of one rank on
    the 256^2 Laplacian: the iteration count of the single-GPU CG with
    Jacobi (within 2) and the true residual."""
    import torch.distributed as dist

    import tnl_b200 as t
    from tnl_b200 import generators as g
    from tnl_b200.distributed import DistributedCG, DistributedMatrix

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(_free_port())
    dist.init_process_group("nccl", rank=0, world_size=1)
    try:
        A = g.laplacian_2d(256)
        D = DistributedMatrix(A.rowptr, A.cols, A.vals, A.n)
        b = torch.tensor(g.uniform_vector(A.n, 1), device="cuda")
        x = torch.zeros(A.n, dtype=torch.float64, device="cuda")
        S = DistributedCG(D, 1e-8)
        assert S.solve(b, x)
        M = t.SparseMatrix(t.CSR, torch.float64).assign(A.rowptr, A.cols, A.vals)
        C = t.CG()
        C.setMatrix(M)
        P = t.Diagonal()
        P.update(M)
        C.setPreconditioner(P)
        C.setup({"convergence-residue": 1e-8, "max-iterations": 100000})
        x2 = torch.zeros_like(x)
        assert C.solve(b, x2)
        assert abs(S.iterations - C.getIterations()) <= 2, (S.iterations, C.getIterations())
        assert t.true_residual(M, b, x) < 1e-7
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [1, 2, 3, 5])
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_halo_plans_exchange_and_products_on_random_matrices(world, seed):
    """Irregular matrices (random row lengths, columns anywhere, some rows
    empty, padding -1 entries), all ranks' plans built in one process and
    the all-to-all emulated: every rank's send lists are what the others
    request, its received values are x at its ghosts in plan order, and its
    local product over [x_local, x_ghost] equals the global product's rows;
    padding stays -1 after the remap."""
    import scipy.sparse as sp

    from tnl_b200.distributed import HaloPlan, split_range

    rng = np.random.default_rng(seed)
    n = int(rng.integers(world, 300))
    lens = rng.integers(0, 12, n)
    lens[rng.random(n) < 0.1] = 0
    rowptr = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    cols = np.concatenate([np.sort(rng.choice(n, size=int(k), replace=False)) if k <= n else np.arange(n)
                           for k in lens]).astype(np.int64) if rowptr[-1] else np.zeros(0, np.int64)
    vals = rng.uniform(-1, 1, cols.size)
    G = sp.csr_matrix((vals, cols, rowptr), shape=(n, n))
    x = rng.uniform(-1, 1, n)
    ranges = [split_range(n, r, world) for r in range(world)]
    plans = []
    for r, (b, e) in enumerate(ranges):
        c = cols[rowptr[b]:rowptr[e]].copy()
        pad = rng.random(c.size) < 0.05
        c[pad] = -1
        P = HaloPlan(c, r, ranges)
        assert np.array_equal(P.local_cols[pad], np.full(int(pad.sum()), -1))
        assert np.all(np.diff(P.ghosts) > 0)
        assert not np.any((P.ghosts >= b) & (P.ghosts < e))
        plans.append((P, c))
    for r, (P, _) in enumerate(plans):
        P.set_send_lists([plans[q][0].requests()[r] for q in range(world)])
    for r, (P, c) in enumerate(plans):
        b, e = ranges[r]
        # what rank r receives from p: p's send buffer segment for r
        recv = []
        for p, (Q, _) in enumerate(plans):
            o = int(Q.send_counts[:r].sum())
            seg = Q.send_idx[o:o + int(Q.send_counts[r])] + ranges[p][0]
            recv.append(x[seg])
        recv = np.concatenate(recv) if recv else np.zeros(0)
        assert np.array_equal(recv, x[P.ghosts])
        xe = np.concatenate([x[b:e], recv])
        keep = P.local_cols >= 0
        rl = np.diff(rowptr[b:e + 1])
        counts = np.array([keep[s:s + k].sum() for s, k in zip(rowptr[b:e] - rowptr[b], rl)], np.int64)
        rp = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
        L = sp.csr_matrix((vals[rowptr[b]:rowptr[e]][keep], P.local_cols[keep], rp),
                          shape=(e - b, P.n_local + P.n_ghost))
        Gk = sp.csr_matrix((vals[rowptr[b]:rowptr[e]][keep], c[keep], rp), shape=(e - b, n))
        assert np.allclose(L @ xe, Gk @ x, rtol=0, atol=1e-13)
    assert sum(int(P.send_counts.sum()) for P, _ in plans) == sum(P.n_ghost for P, _ in plans)
