"""Seeded synthetic inputs with the shapes of the benchmark configurations.

All randomness comes from a counter-based SplitMix64 hash of
(seed, stream, element index), so every array is a pure function of its
arguments: the same on every machine and independent of how it is chunked.
Uniform doubles on [-1, 1) take the top 53 bits of the hash.

Matrices are returned in CSR form (int32 row pointers and columns, sorted
columns within each row, float64 values); the format builders of the
library turn them into the other TNL formats.

Workloads (no public matrix collection is used; these stand in for it):

* ``laplacian_2d(N)`` -- 2D 5-point Dirichlet Laplacian on an N x N grid in
  natural lexicographic order, values {4, -1}; nnz = 5 N^2 - 4 N.
* ``power_law(n, exponent, cap, seed)`` -- row lengths from a Zipf law
  truncated to [1, cap], column indices uniform on [0, n) without repeats
  inside a row (sorted), values U[-1, 1).
* ``diffusion_3d(N, ...)`` -- 7-point -div(k grad u) with harmonic-mean face
  coefficients and k = exp(g), g a Gaussian random field.
* ``diffusion_2d(N, ...)`` -- the 5-point analogue, for the learned
  preconditioner's training and evaluation problems.
* ``convection_diffusion_3d(N, ...)`` -- first-order upwind 7-point
  convection-diffusion with a divergence-free velocity.
"""
from __future__ import annotations

import numpy as np

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)
_G = np.uint64(0x9E3779B97F4A7C15)
_C1 = np.uint64(0xBF58476D1CE4E5B9)
_C2 = np.uint64(0x94D049BB133111EB)


def _mix(z: np.ndarray) -> np.ndarray:
    """SplitMix64 finaliser on a uint64 array (wrapping arithmetic)."""
    with np.errstate(over="ignore"):
        z = z + _G
        z = (z ^ (z >> np.uint64(30))) * _C1
        z = (z ^ (z >> np.uint64(27))) * _C2
        return z ^ (z >> np.uint64(31))


def hash64(seed: int, stream: int, index: np.ndarray) -> np.ndarray:
    """64-bit hash of (seed, stream, index) for every entry of ``index``."""
    base = _mix(np.array([(seed * 0x100000001B3 + stream * 0x9E37) & 0xFFFFFFFFFFFFFFFF], dtype=np.uint64))[0]
    with np.errstate(over="ignore"):
        return _mix(np.asarray(index, dtype=np.uint64) + base)


def uniform01(seed: int, stream: int, index: np.ndarray) -> np.ndarray:
    """U[0, 1) doubles from the top 53 bits of the hash."""
    return (hash64(seed, stream, index) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def uniform_vector(n: int, seed: int, lo: float = -1.0, hi: float = 1.0, stream: int = 0) -> np.ndarray:
    """x_i ~ U[lo, hi), i = 0..n-1."""
    u = uniform01(seed, stream, np.arange(n, dtype=np.uint64))
    return lo + (hi - lo) * u


def gaussian(seed: int, stream: int, index: np.ndarray) -> np.ndarray:
    """Standard normal samples by the Box-Muller transform of two hashes."""
    u1 = uniform01(seed, stream, index)
    u2 = uniform01(seed, stream + 1, index)
    u1 = np.maximum(u1, 1e-300)
    return np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)


class CSRMatrix:
    """Host CSR triple plus shape; columns sorted inside each row."""

    def __init__(self, rowptr, cols, vals, ncols=None):
        self.rowptr = np.ascontiguousarray(rowptr, dtype=np.int32)
        self.cols = np.ascontiguousarray(cols, dtype=np.int32)
        self.vals = np.ascontiguousarray(vals)
        self.n = len(self.rowptr) - 1
        self.ncols = self.n if ncols is None else int(ncols)

    @property
    def nnz(self) -> int:
        return int(self.rowptr[-1])

    def row_lengths(self) -> np.ndarray:
        return np.diff(self.rowptr).astype(np.int32)

    def astype(self, dtype) -> "CSRMatrix":
        return CSRMatrix(self.rowptr, self.cols, self.vals.astype(dtype), self.ncols)

    def matvec(self, x: np.ndarray) -> np.ndarray:
        """Plain numpy y = A x (pairwise summation order, for quick checks only)."""
        prod = self.vals.astype(np.float64) * x[self.cols]
        out = np.zeros(self.n, dtype=np.float64)
        rows = np.repeat(np.arange(self.n), np.diff(self.rowptr))
        np.add.at(out, rows, prod)
        return out


def laplacian_2d(N: int, dtype=np.float64) -> CSRMatrix:
    """5-point Dirichlet Laplacian, rows in natural order, columns ascending."""
    n = N * N
    iy, ix = np.divmod(np.arange(n, dtype=np.int64), N)
    offs = [(-N, iy > 0), (-1, ix > 0), (0, np.ones(n, bool)), (1, ix < N - 1), (N, iy < N - 1)]
    lens = sum(m.astype(np.int32) for _, m in offs)
    rowptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(lens, out=rowptr[1:])
    cols = np.empty(rowptr[-1], dtype=np.int32)
    vals = np.empty(rowptr[-1], dtype=dtype)
    pos = rowptr[:-1].copy()
    i = np.arange(n, dtype=np.int64)
    for d, m in offs:
        p = pos[m]
        cols[p] = (i[m] + d).astype(np.int32)
        vals[p] = 4.0 if d == 0 else -1.0
        pos[m] += 1
    return CSRMatrix(rowptr.astype(np.int32), cols, vals)


def zipf_lengths(n: int, exponent: float, cap: int, seed: int, lo: int = 1) -> np.ndarray:
    """Row lengths k in [lo, cap] with P(k) proportional to k^-exponent (inverse CDF)."""
    k = np.arange(lo, cap + 1, dtype=np.float64)
    p = k ** (-exponent)
    cdf = np.cumsum(p)
    cdf /= cdf[-1]
    cdf[-1] = 1.0
    u = uniform01(seed, 1, np.arange(n, dtype=np.uint64))
    return (np.searchsorted(cdf, u, side="right") + lo).astype(np.int32)


def distinct_sorted_columns(rowptr: np.ndarray, ncols: int, seed: int) -> np.ndarray:
    """Uniform column indices without repeats inside a row, ascending per row.

    Draws every slot from the hash, sorts (row, column) keys, and redraws the
    later copy of every repeated pair from a fresh hash stream until no row
    holds a repeat; only rows that had a repeat are re-sorted.
    """
    n = len(rowptr) - 1
    nnz = int(rowptr[-1])
    lens = np.diff(rowptr).astype(np.int64)
    if nnz and lens.max() > ncols:
        raise ValueError("a row is longer than the number of columns")
    row_of = np.repeat(np.arange(n, dtype=np.int64), lens)
    e = np.arange(nnz, dtype=np.uint64)
    cols = (hash64(seed, 100, e) % np.uint64(ncols)).astype(np.int64)
    keys = row_of * ncols + cols
    del cols
    keys.sort(kind="stable")
    t = 1
    while True:
        dup = np.nonzero(keys[1:] == keys[:-1])[0] + 1
        if dup.size == 0:
            break
        newc = (hash64(seed, 100 + t, dup.astype(np.uint64)) % np.uint64(ncols)).astype(np.int64)
        keys[dup] = row_of[dup] * ncols + newc
        rows = np.unique(row_of[dup])
        idx = np.nonzero(np.isin(row_of, rows))[0]
        keys[idx] = np.sort(keys[idx])
        t += 1
    return (keys - row_of * ncols).astype(np.int32)


def power_law(n: int, exponent: float = 1.73, cap: int = 4096, seed: int = 2, dtype=np.float64, lo: int = 1) -> CSRMatrix:
    """Power-law sparse matrix: Zipf row lengths, distinct uniform columns, U[-1,1) values."""
    lens = zipf_lengths(n, exponent, cap, seed, lo)
    rowptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(lens, out=rowptr[1:])
    if rowptr[-1] > np.iinfo(np.int32).max:
        raise OverflowError("nnz exceeds int32")
    cols = distinct_sorted_columns(rowptr, n, seed)
    vals = (-1.0 + 2.0 * uniform01(seed, 3, np.arange(rowptr[-1], dtype=np.uint64))).astype(dtype)
    return CSRMatrix(rowptr.astype(np.int32), cols, vals)


def gaussian_random_field(shape, corr_length: float, sigma: float, seed: int) -> np.ndarray:
    """Stationary Gaussian random field on the unit cube/square, cell-centred.

    Spectral synthesis: white noise from the hash is filtered in Fourier
    space by the square root of a Gaussian covariance spectrum
    exp(-|k|^2 l^2 / 4) (l = correlation length in units of the domain),
    then scaled to standard deviation ``sigma``.
    """
    shape = tuple(int(s) for s in shape)
    size = int(np.prod(shape))
    w = gaussian(seed, 7, np.arange(size, dtype=np.uint64)).reshape(shape)
    W = np.fft.rfftn(w)
    ks = [np.fft.fftfreq(s) * s * 2.0 * np.pi for s in shape[:-1]] + [np.fft.rfftfreq(shape[-1]) * shape[-1] * 2.0 * np.pi]
    grids = np.meshgrid(*ks, indexing="ij")
    k2 = sum(g * g for g in grids)
    W *= np.exp(-k2 * corr_length * corr_length / 8.0)
    g = np.fft.irfftn(W, s=shape, axes=tuple(range(len(shape))))
    g -= g.mean()
    std = g.std()
    if std > 0:
        g *= sigma / std
    return g


def _harmonic(a, b):
    return 2.0 * a * b / (a + b)


def diffusion_3d(N: int, corr_length: float = 0.1, sigma: float = 2.0, seed: int = 3) -> CSRMatrix:
    """-div(k grad u) on the unit cube, N^3 cells, Dirichlet boundary, k = exp(g).

    Face coefficients are harmonic means of the two cell values; a boundary
    face uses the cell's own k (distance h/2 to the wall, weight 2k).  The
    grid spacing factor 1/h^2 is dropped (it scales A uniformly).
    """
    k = np.exp(gaussian_random_field((N, N, N), corr_length, sigma, seed))
    return _stencil_from_coeffs(k)


def diffusion_2d(N: int, corr_length: float = 0.1, sigma: float = 2.0, seed: int = 3) -> CSRMatrix:
    """2D 5-point analogue of :func:`diffusion_3d` on an N x N grid."""
    k = np.exp(gaussian_random_field((N, N), corr_length, sigma, seed))
    return _stencil_from_coeffs(k)


def diffusion_2d_problem(N: int, seed: int, corr_range=(0.02, 0.2), sigma_range=(1.0, 3.0)) -> CSRMatrix:
    """One seeded problem of the learned-preconditioner workload: a 2D
    diffusion matrix whose GRF has correlation length ~ U[corr_range] and
    sigma ~ U[sigma_range], both drawn from the seed."""
    u = uniform01(seed, 99, np.arange(2, dtype=np.uint64))
    corr = corr_range[0] + (corr_range[1] - corr_range[0]) * u[0]
    sigma = sigma_range[0] + (sigma_range[1] - sigma_range[0]) * u[1]
    return diffusion_2d(N, corr, sigma, seed)


def _stencil_from_coeffs(k: np.ndarray, velocity=None) -> CSRMatrix:
    """Assemble the cell-centred finite-volume operator for coefficient field k.

    ``velocity`` (optional) is a tuple of face-normal velocities per axis,
    axis a holding the shape[a] + 1 faces along a (face i between cells i-1
    and i, faces 0 and shape[a] on the boundary); first-order upwinding adds
    the convective flux, inflow through a boundary face carrying the
    Dirichlet value 0.
    Rows are in natural lexicographic order (last axis fastest) and columns
    ascend inside each row.
    """
    shape = k.shape
    dim = k.ndim
    n = k.size
    strides = [int(np.prod(shape[a + 1:])) for a in range(dim)]
    diag = np.zeros(shape)
    offdiag = {}
    for a in range(dim):
        for side in (-1, 1):
            sl_self = [slice(None)] * dim
            sl_nb = [slice(None)] * dim
            if side == 1:
                sl_self[a] = slice(0, shape[a] - 1)
                sl_nb[a] = slice(1, shape[a])
            else:
                sl_self[a] = slice(1, shape[a])
                sl_nb[a] = slice(0, shape[a] - 1)
            coef = np.zeros(shape)
            coef[tuple(sl_self)] = _harmonic(k[tuple(sl_self)], k[tuple(sl_nb)])
            bnd = [slice(None)] * dim
            bnd[a] = shape[a] - 1 if side == 1 else 0
            wall = np.zeros(shape)
            wall[tuple(bnd)] = 2.0 * k[tuple(bnd)]
            off = -coef
            d = coef + wall
            if velocity is not None:
                v = velocity[a]  # shape[a] + 1 faces along axis a
                face = [slice(None)] * dim
                face[a] = slice(1, shape[a] + 1) if side == 1 else slice(0, shape[a])
                vf = v[tuple(face)] if side == 1 else -v[tuple(face)]  # outward normal
                out = np.maximum(vf, 0.0)
                inn = np.minimum(vf, 0.0)
                d = d + out
                interior = np.zeros(shape, bool)
                interior[tuple(sl_self)] = True
                off = off + np.where(interior, inn, 0.0)
            diag += d
            offdiag[(a, side)] = off
    idx = np.arange(n, dtype=np.int64).reshape(shape)
    entries = []
    for a in range(dim):
        for side in (-1, 1):
            entries.append((side * strides[a], offdiag[(a, side)]))
    entries.append((0, diag))
    entries.sort(key=lambda t: t[0])
    masks = []
    for d, vals in entries:
        if d == 0:
            m = np.ones(shape, bool)
        else:
            a = [s for s in range(dim) if strides[s] == abs(d)][0]
            m = np.zeros(shape, bool)
            sl = [slice(None)] * dim
            sl[a] = slice(0, shape[a] - 1) if d > 0 else slice(1, shape[a])
            m[tuple(sl)] = True
        masks.append(m.ravel())
    lens = np.sum([m.astype(np.int32) for m in masks], axis=0)
    rowptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(lens, out=rowptr[1:])
    cols = np.empty(rowptr[-1], dtype=np.int32)
    vals = np.empty(rowptr[-1], dtype=np.float64)
    pos = rowptr[:-1].copy()
    flat = idx.ravel()
    for (d, v), m in zip(entries, masks):
        p = pos[m]
        cols[p] = (flat[m] + d).astype(np.int32)
        vals[p] = v.ravel()[m]
        pos[m] += 1
    return CSRMatrix(rowptr.astype(np.int32), cols, vals)


def convection_diffusion_3d(N: int, peclet_range=(10.0, 1000.0), sigma: float = 1.0, seed: int = 5) -> CSRMatrix:
    """Steady 3D convection-diffusion, first-order upwind 7-point stencil.

    Velocity = curl of a random vector stream function (divergence free by
    construction on the discrete faces), scaled so cell Peclet numbers
    |v| h / k span ``peclet_range``; k is lognormal with the given sigma.
    """
    shape = (N, N, N)
    k = np.exp(gaussian_random_field(shape, 0.2, sigma, seed))
    psi = [gaussian_random_field((N + 1, N + 1, N + 1), 0.25, 1.0, seed + 10 + c) for c in range(3)]
    # face velocities from the discrete curl of psi defined on cell corners
    def d(f, axis):
        return np.diff(f, axis=axis)

    # u_x on x-faces: d psi_z / dy - d psi_y / dz, averaged to the face
    ux = d(psi[2], 1)[:, :, :-1] - d(psi[1], 2)[:, :-1, :]
    uy = d(psi[0], 2)[:-1, :, :] - d(psi[2], 0)[:, :, :-1]
    uz = d(psi[1], 0)[:, :-1, :] - d(psi[0], 1)[:-1, :, :]
    vel = [ux, uy, uz]
    # one uniform factor keeps the field divergence free; it puts the
    # geometric mean of the cell Peclet number |v| h / k (|v| from the
    # cell's + faces) at the geometric centre of peclet_range (h = 1/N)
    speed = np.sqrt(ux[1:, :, :] ** 2 + uy[:, 1:, :] ** 2 + uz[:, :, 1:] ** 2) + 1e-300
    pe = speed / (N * k)
    centre = 0.5 * (np.log(peclet_range[0]) + np.log(peclet_range[1]))
    scale = np.exp(centre - np.mean(np.log(pe)))
    vel = [v * scale * N for v in vel]
    return _stencil_from_coeffs(k, velocity=vel)
