"""Row-block distributed sparse matrix and CG: TNL::Matrices::DistributedMatrix
(Matrices/DistributedMatrix.h, DistributedMatrix_impl.h:217-249) over
torch.distributed, one process per GPU.

Layout (as the reference's): rank r owns the contiguous rows
[begin_r, end_r) given by splitRange (Containers/BlockPartitioning.h:27-40:
the first rows % ranks ranks take one row more).  Its local matrix has
those rows and n_local + n_ghost columns: the owned columns first (global
column - begin_r), then the ghost columns -- the off-rank columns its rows
touch, sorted by global index -- after them.  A product gathers the ghost
values of x from their owners (the halo exchange: one all-to-all of the
values each rank needs, ordered by owner rank and global index) into
x_ext = [x_local, x_ghost] and runs the library's SpMV on the local matrix
(the reference's localMatrix.vectorProduct on getConstLocalViewWithGhosts
after waitForSynchronization).  The exchange is the only collective of a
product; CG adds an all-reduce of its scalars.

``HaloPlan`` holds the index arithmetic (pure functions of the column
indices and the row ranges) separately from the exchange, so that it is
tested on the CPU with gloo ranks.  Values move through torch.distributed
(NCCL between GPUs); the arithmetic runs in the library's kernels.
"""
from __future__ import annotations

import numpy as np
import torch

from . import CSR, SparseMatrix, _real_code, _stream, check
from . import _capi as capi


def split_range(size: int, rank: int, parts: int) -> tuple[int, int]:
    """splitRange(0, size, rank, parts) (Containers/BlockPartitioning.h:27-40)."""
    part, rem = divmod(size, parts)
    if rank < rem:
        b = rank * (part + 1)
        return b, b + part + 1
    b = rem * (part + 1) + (rank - rem) * part
    return b, b + part


class HaloPlan:
    """Ghost columns and exchange lists of one rank.

    ``cols`` are the global column indices of the rank's local rows (padding
    -1 allowed), ``ranges`` the row range of every rank (equal to the column
    ranges: square matrices).  After construction:
      * ``local_cols``  -- cols remapped into [0, n_local + n_ghost);
      * ``ghosts``      -- the sorted global ghost columns;
      * ``recv_counts`` -- ghosts owned by each rank (their order in
        ``ghosts`` is by owner, then by global index);
    ``set_send_lists`` takes the ghost lists the other ranks request from
    this one and makes ``send_idx`` (local indices to gather) and
    ``send_counts``."""

    def __init__(self, cols, rank: int, ranges):
        cols = np.asarray(cols, np.int64)
        self.rank = rank
        self.ranges = [(int(b), int(e)) for b, e in ranges]
        b, e = self.ranges[rank]
        self.n_local = e - b
        valid = cols >= 0
        off = valid & ((cols < b) | (cols >= e))
        self.ghosts = np.unique(cols[off])
        ends = np.array([r[1] for r in self.ranges], np.int64)
        owners = np.searchsorted(ends, self.ghosts, side="right")
        self.recv_counts = np.bincount(owners, minlength=len(self.ranges)).astype(np.int64)
        local = np.where(valid, cols - b, -1)
        local[off] = self.n_local + np.searchsorted(self.ghosts, cols[off])
        self.local_cols = local.astype(np.int32)
        self.send_idx = np.zeros(0, np.int64)
        self.send_counts = np.zeros(len(self.ranges), np.int64)

    @property
    def n_ghost(self) -> int:
        return int(self.ghosts.size)

    def requests(self) -> list[np.ndarray]:
        """The ghost columns this rank needs from each rank (global indices)."""
        out, o = [], 0
        for c in self.recv_counts:
            out.append(self.ghosts[o:o + int(c)])
            o += int(c)
        return out

    def set_send_lists(self, requested: list[np.ndarray]) -> None:
        """requested[p]: the global columns rank p needs from this rank."""
        b, e = self.ranges[self.rank]
        for p, req in enumerate(requested):
            req = np.asarray(req, np.int64)
            if req.size and (req.min() < b or req.max() >= e):
                raise ValueError(f"rank {p} requested columns outside the range of rank {self.rank}")
        self.send_counts = np.array([len(r) for r in requested], np.int64)
        self.send_idx = (np.concatenate([np.asarray(r, np.int64) for r in requested]) - b if requested
                         else np.zeros(0, np.int64))


def _a2a(group, device, counts_out: np.ndarray, counts_in: np.ndarray, payload: torch.Tensor, dtype):
    import torch.distributed as dist

    out = torch.empty(int(counts_in.sum()), dtype=dtype, device=device)
    dist.all_to_all_single(out, payload, [int(c) for c in counts_in], [int(c) for c in counts_out], group=group)
    return out


def build_plan(cols, group=None, device="cpu", rows: int | None = None) -> HaloPlan:
    """HaloPlan of this rank, the request lists exchanged among all ranks of
    ``group`` (all-to-all of the counts, then of the requested indices).
    ``device`` is where the collective's tensors live ("cuda" under NCCL,
    "cpu" under gloo)."""
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    counts = torch.tensor([0], dtype=torch.int64)
    if rows is None:
        raise ValueError("build_plan needs the global row count")
    ranges = [split_range(rows, r, world) for r in range(world)]
    plan = HaloPlan(cols, rank, ranges)
    rc = torch.tensor(plan.recv_counts, dtype=torch.int64, device=device)
    sc = torch.empty(world, dtype=torch.int64, device=device)
    dist.all_to_all_single(sc, rc, group=group)
    send_counts = sc.cpu().numpy()
    req = torch.tensor(plan.ghosts, dtype=torch.int64, device=device)
    got = _a2a(group, device, plan.recv_counts, send_counts, req, torch.int64).cpu().numpy()
    lists, o = [], 0
    for c in send_counts:
        lists.append(got[o:o + int(c)])
        o += int(c)
    plan.set_send_lists(lists)
    del counts
    return plan


class DistributedMatrix:
    """TNL::Matrices::DistributedMatrix with CSR local matrices on the GPU.

    ``rowptr``, ``cols`` (global columns), ``vals`` are the CSR arrays of
    this rank's rows [begin, end) = splitRange(rows, rank, world)."""

    def __init__(self, rowptr, cols, vals, rows: int, columns: int | None = None, group=None,
                 real=torch.float64, exchange_device: str = "cuda"):
        import torch.distributed as dist

        if columns is not None and columns != rows:
            raise ValueError("DistributedMatrix: only square matrices are distributed by rows and columns alike")
        self.group = group
        self.rows = rows
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        self.local_range = split_range(rows, self.rank, self.world)
        n_local = self.local_range[1] - self.local_range[0]
        if len(rowptr) != n_local + 1:
            raise ValueError("DistributedMatrix: the local rows do not match splitRange of this rank")
        self.exchange_device = exchange_device
        self.plan = build_plan(cols, group, exchange_device, rows)
        self.real = real
        self.local = SparseMatrix(CSR, real).assign(np.asarray(rowptr, np.int32), self.plan.local_cols,
                                                    np.asarray(vals), n_local + self.plan.n_ghost)
        dev = torch.device("cuda")
        self._send_idx = torch.tensor(self.plan.send_idx, dtype=torch.int64, device=dev)
        self._x_ext = torch.zeros(n_local + self.plan.n_ghost, dtype=real, device=dev)

    def getLocalRowRange(self) -> tuple[int, int]:
        return self.local_range

    def getRows(self) -> int:
        return self.rows

    def getColumns(self) -> int:
        return self.rows

    def getLocalMatrix(self) -> SparseMatrix:
        return self.local

    def synchronize(self, x_local: torch.Tensor) -> torch.Tensor:
        """x_ext = [x_local, ghost values of x] (the halo exchange)."""
        import torch.distributed as dist

        n = self.plan.n_local
        self._x_ext[:n].copy_(x_local)
        send = x_local.index_select(0, self._send_idx).to(self.exchange_device)
        recv = torch.empty(self.plan.n_ghost, dtype=self.real, device=self.exchange_device)
        dist.all_to_all_single(recv, send, [int(c) for c in self.plan.recv_counts],
                               [int(c) for c in self.plan.send_counts], group=self.group)
        self._x_ext[n:].copy_(recv)
        return self._x_ext

    def vectorProduct(self, x_local: torch.Tensor, y_local: torch.Tensor) -> None:
        """y_local = (A x) restricted to this rank's rows."""
        if x_local.numel() != self.plan.n_local or y_local.numel() != self.plan.n_local:
            raise ValueError("vectorProduct: the local vectors do not match the local row range")
        self.local.vectorProduct(self.synchronize(x_local), y_local)


def _dot(a: torch.Tensor, b: torch.Tensor, group) -> float:
    import torch.distributed as dist

    d = torch.zeros(1, dtype=torch.float64, device=a.device)
    check(capi.tnlb_dot(_real_code(a.dtype), a.numel(), a.data_ptr(), b.data_ptr(), d.data_ptr(), _stream()))
    dist.all_reduce(d, group=group)
    return float(d.item())


def _axpby(alpha: float, x: torch.Tensor, beta: float, y: torch.Tensor) -> None:
    check(capi.tnlb_axpby(_real_code(x.dtype), x.numel(), alpha, x.data_ptr(), beta, y.data_ptr(), _stream()))


class DistributedCG:
    """CG with the Jacobi (Diagonal) preconditioner on a DistributedMatrix:
    the iteration of Solvers/Linear/CG.hpp:12-121 with distributed vectors
    (local dot products summed by an all-reduce), the reference's residue
    sqrt((r, z)) / ||M^-1 b|| and its stopping rule (iterate while the
    residue is not below the convergence residue and the iteration count is
    below the maximum).  The Jacobi step z = D^-1 r is a product with the
    diagonal matrix D^-1 through the library's SpMV."""

    def __init__(self, A: DistributedMatrix, convergence_residue: float = 1e-8, max_iterations: int = 100000):
        self.A = A
        self.tol = convergence_residue
        self.max_iterations = max_iterations
        self.iterations = 0
        self.residue = float("nan")
        h = A.getLocalMatrix().toHostCSR()
        rows = np.repeat(np.arange(h.n), np.diff(h.rowptr))
        diag = np.zeros(h.n)
        on = h.cols == rows  # the diagonal's local column is the local row
        diag[rows[on]] = h.vals[on]
        if np.any(diag == 0):
            raise ValueError("DistributedCG: a zero diagonal entry (the Jacobi preconditioner needs all of them)")
        n = h.n
        self.dinv = SparseMatrix(CSR, A.real).assign(np.arange(n + 1, dtype=np.int32), np.arange(n, dtype=np.int32),
                                                      1.0 / diag, n)

    def solve(self, b: torch.Tensor, x: torch.Tensor) -> bool:
        A, g = self.A, self.A.group
        r = torch.empty_like(b)
        z = torch.empty_like(b)
        p = torch.empty_like(b)
        q = torch.empty_like(b)
        self.dinv.vectorProduct(b, z)
        normb = np.sqrt(max(_dot(z, z, g), 0.0))
        if normb == 0.0:
            x.zero_()
            self.iterations, self.residue = 0, 0.0
            return True
        A.vectorProduct(x, r)
        _axpby(1.0, b, -1.0, r)  # r = b - A x
        self.dinv.vectorProduct(r, z)
        p.copy_(z)
        s1 = _dot(r, z, g)
        self.residue = np.sqrt(max(s1, 0.0)) / normb
        it = 0
        while not (self.residue < self.tol) and it < self.max_iterations:
            it += 1
            A.vectorProduct(p, q)
            s2 = _dot(q, p, g)
            if s2 == 0.0:
                self.residue = 0.0
                break
            alpha = s1 / s2
            _axpby(alpha, p, 1.0, x)
            _axpby(-alpha, q, 1.0, r)
            self.dinv.vectorProduct(r, z)
            s2, s1 = s1, _dot(r, z, g)
            beta = 0.0 if s2 == 0.0 else s1 / s2
            _axpby(1.0, z, beta, p)  # p = z + beta p
            self.residue = np.sqrt(max(s1, 0.0)) / normb
        self.iterations = it
        return bool(self.residue < self.tol)
