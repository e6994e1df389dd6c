"""FP64 CPU reference of the learned FSAI preconditioner -- TEST INFRASTRUCTURE.

The learned factorised sparse approximate inverse has no counterpart in the
reference library; this module restates, in plain numpy FP64, exactly what
the GPU kernels of tnl_b200/csrc/lfsai.cu compute, so that the tests can
check the GPU features, network outputs, loss and gradients, and check this
backpropagation itself against finite differences.

Definitions (shared with lfsai.cu):

* Pattern of G: row i holds the stored columns j <= i of A (the lower
  triangle with the diagonal), at most 4 of them; they occupy the
  right-aligned slots 4-k .. 3 (slot 3 is the diagonal).
* Scaling s_j = 1/sqrt(a_jj); B = S A S has a unit diagonal.
* Features f (16, zero padded): f[0..5] = B(J_p, J_q) for the slot pairs
  (0,1) (0,2) (0,3) (1,2) (1,3) (2,3) (0 when a slot is empty); f[6..8] =
  B(i, j) for the first three stored columns j > i; f[9] = k/4;
  f[10] = (number of stored columns > i)/3.
* Network: h1 = relu(W1 f + b1), h2 = relu(W2 h1 + b2), h3 = relu(W3 h2 + b3),
  o = W4 h3 + b4 with W1 64x16, W2 W3 64x64, W4 4x64.  Every layer input
  and every weight is rounded to BF16 (round to nearest even) before the
  product; sums and biases are FP32 on the GPU, FP64 here.
* G'_i: slot 3 = exp(o_3), occupied slots t < 3 = o_t.  G_ij = G'_i,slot(j) s_j,
  so G A G^T = G' B G'^T.
* Loss over probes z_p: L = (1/(n P)) sum_p ||z_p - G A G^T z_p||^2 with
  gradient dL/dG = -(2/(n P)) sum_p (u_p w_p^T + z_p q_p^T) on the pattern,
  where w = A G^T z, u = z - G w, q = A G^T u.

Parameter vector layout (float32, 9668 entries): W1 (64x16 row-major), b1,
W2 (64x64), b2, W3, b3, W4 (4x64), b4.
"""
from __future__ import annotations

import numpy as np

F, H, K = 16, 64, 4
SHAPES = [("W1", (H, F)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (H, H)), ("b3", (H,)),
          ("W4", (K, H)), ("b4", (K,))]
NPARAMS = sum(int(np.prod(s)) for _, s in SHAPES)


def unpack(theta):
    out, o = {}, 0
    for name, shp in SHAPES:
        c = int(np.prod(shp))
        out[name] = np.asarray(theta[o:o + c], np.float64).reshape(shp)
        o += c
    return out


def pack(d):
    return np.concatenate([np.asarray(d[name], np.float64).ravel() for name, _ in SHAPES])


ROUND = True  # the finite-difference check turns the BF16 rounding off


def bf16(x):
    """Round FP64/FP32 values to BF16 (nearest even), returned as float64."""
    if not ROUND:
        return np.asarray(x, np.float64)
    a = np.asarray(x, np.float32).copy()
    u = a.view(np.uint32)
    rounding = ((u >> 16) & 1) + 0x7FFF
    u = ((u.astype(np.uint64) + rounding) & 0xFFFF0000).astype(np.uint32)
    return u.view(np.float32).astype(np.float64)


def pattern(A):
    """Per row: (slots, columns) of G's pattern; raises if a row has > 4."""
    rp, cols = A.rowptr, A.cols
    pat = []
    for i in range(A.n):
        c = cols[rp[i]:rp[i + 1]]
        low = sorted(int(x) for x in c if 0 <= x <= i)
        if len(low) > K:
            raise ValueError("learned FSAI: more than 4 stored entries in the lower triangle of a row")
        pat.append(low)
    return pat


def _row_dict(A):
    rp, cols, vals = A.rowptr, A.cols, A.vals
    return [dict(zip(cols[rp[i]:rp[i + 1]].tolist(), vals[rp[i]:rp[i + 1]].tolist())) for i in range(A.n)]


def features(A, pat=None):
    pat = pattern(A) if pat is None else pat
    rows = _row_dict(A)
    d = np.array([rows[i].get(i, 0.0) for i in range(A.n)], np.float64)
    s = 1.0 / np.sqrt(d)
    f = np.zeros((A.n, F))
    pairs = [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)]
    for i in range(A.n):
        J = pat[i]
        k = len(J)
        slot_col = [None] * K
        for t, j in enumerate(J):
            slot_col[K - k + t] = j
        for m, (p, q) in enumerate(pairs):
            jp, jq = slot_col[p], slot_col[q]
            if jp is not None and jq is not None:
                f[i, m] = rows[jp].get(jq, 0.0) * s[jp] * s[jq]
        upper = sorted(j for j in rows[i] if j > i)[:3]
        for m, j in enumerate(upper):
            f[i, 6 + m] = rows[i][j] * s[i] * s[j]
        f[i, 9] = k / 4.0
        f[i, 10] = sum(1 for j in rows[i] if j > i) / 3.0
    return f, s, pat


def forward(theta, f):
    """Returns o (n x 4) and the activations needed for backprop."""
    P = {k: bf16(v) if k.startswith("W") else v for k, v in unpack(theta).items()}
    x0 = bf16(f)
    z1 = x0 @ P["W1"].T + P["b1"]
    h1 = np.maximum(z1, 0)
    x1 = bf16(h1)
    z2 = x1 @ P["W2"].T + P["b2"]
    h2 = np.maximum(z2, 0)
    x2 = bf16(h2)
    z3 = x2 @ P["W3"].T + P["b3"]
    h3 = np.maximum(z3, 0)
    x3 = bf16(h3)
    o = x3 @ P["W4"].T + P["b4"]
    return o, (P, x0, z1, x1, z2, x2, z3, x3)


def g_values(o, s, pat):
    """Values of G on its pattern, row by row (CSR order = ascending columns)."""
    vals = []
    for i, J in enumerate(pat):
        k = len(J)
        for t, j in enumerate(J):
            slot = K - k + t
            gp = np.exp(o[i, 3]) if slot == 3 else o[i, slot]
            vals.append(gp * s[j])
    return np.array(vals, np.float64)


def g_matrix(vals, pat, n):
    import scipy.sparse as sp

    rows = np.repeat(np.arange(n), [len(J) for J in pat])
    cols = np.concatenate([np.array(J, np.int64) for J in pat]) if n else np.zeros(0, np.int64)
    return sp.csr_matrix((vals, (rows, cols)), shape=(n, n))


def loss_and_grad_G(A, Gm, probes):
    """L and dL/dG (dense over G's pattern via the sparse structure of Gm)."""
    import scipy.sparse as sp

    As = sp.csr_matrix((A.vals, A.cols, A.rowptr), shape=(A.n, A.n))
    n, P = probes.shape
    Z = probes
    W = As @ (Gm.T @ Z)
    U = Z - Gm @ W
    Q = As @ (Gm.T @ U)
    L = float(np.sum(U * U)) / (n * P)
    coo = Gm.tocoo()
    gi, gj = coo.row, coo.col
    dG = -(2.0 / (n * P)) * (np.sum(U[gi] * W[gj], axis=1) + np.sum(Z[gi] * Q[gj], axis=1))
    order = np.lexsort((gj, gi))
    return L, dG[order]


def backward(theta, cache, do):
    P, x0, z1, x1, z2, x2, z3, x3 = cache
    g = {}
    g["W4"] = do.T @ x3
    g["b4"] = do.sum(0)
    d3 = (do @ P["W4"]) * (z3 > 0)
    g["W3"] = d3.T @ x2
    g["b3"] = d3.sum(0)
    d2 = (d3 @ P["W3"]) * (z2 > 0)
    g["W2"] = d2.T @ x1
    g["b2"] = d2.sum(0)
    d1 = (d2 @ P["W2"]) * (z1 > 0)
    g["W1"] = d1.T @ x0
    g["b1"] = d1.sum(0)
    return pack(g)


def loss_and_grad(theta, A, probes):
    """L and dL/dtheta (straight-through for the BF16 rounding)."""
    f, s, pat = features(A)
    o, cache = forward(theta, f)
    vals = g_values(o, s, pat)
    Gm = g_matrix(vals, pat, A.n)
    L, dG = loss_and_grad_G(A, Gm, probes)
    do = np.zeros_like(o)
    q = 0
    for i, J in enumerate(pat):
        k = len(J)
        for t, j in enumerate(J):
            slot = K - k + t
            dgp = dG[q] * s[j]
            do[i, slot] += dgp * (np.exp(o[i, 3]) if slot == 3 else 1.0)
            q += 1
    return L, backward(theta, cache, do)


def init_params(seed: int) -> np.ndarray:
    """Deterministic initial parameters (same as lfsai.cu's initialiser):
    U(-a, a) with a = sqrt(6/(fan_in+fan_out)), biases 0; W4 and b4 scaled by
    0.1 so the initial G' is close to the identity (exp(0) = 1 on the
    diagonal).  Uniform numbers come from SplitMix64(seed, index)."""
    out = []
    idx = 0
    for name, shp in SHAPES:
        c = int(np.prod(shp))
        if name.startswith("W"):
            fan_out, fan_in = shp
            a = np.sqrt(6.0 / (fan_in + fan_out)) * (0.1 if name == "W4" else 1.0)
            u = _u01(seed, np.arange(idx, idx + c, dtype=np.uint64))
            out.append((2.0 * u - 1.0) * a)
        else:
            out.append(np.zeros(c))
        idx += c
    return np.concatenate(out).astype(np.float32).astype(np.float64)


def _u01(seed, index):
    M = np.uint64(0xFFFFFFFFFFFFFFFF)
    with np.errstate(over="ignore"):
        z = (np.uint64(seed) * np.uint64(0x9E3779B97F4A7C15) + index) & M
        z = z + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def fsai_classical(A):
    """Kolotilina-Yeremin FSAI values on the lower pattern (FP64, per row:
    A[J,J] g = e_last, G_i = g / sqrt(g_last)); CSR order of the pattern."""
    rows = _row_dict(A)
    out = []
    for i in range(A.n):
        J = sorted(j for j in rows[i] if 0 <= j <= i)
        B = np.array([[rows[p].get(q, 0.0) for q in J] for p in J])
        e = np.zeros(len(J))
        e[-1] = 1.0
        g = np.linalg.solve(B, e)
        out.extend(g / np.sqrt(g[-1]))
    return np.array(out)


def fsai2_classical(A):
    """Two-factor FSAI for nonsymmetric A: rows of G_L (B^-T e) and of
    H = G_U^T (B^-1 e) on the lower pattern, both / sqrt((B^-1)_last,last)."""
    rows = _row_dict(A)
    gl, h = [], []
    for i in range(A.n):
        J = sorted(j for j in rows[i] if 0 <= j <= i)
        B = np.array([[rows[p].get(q, 0.0) for q in J] for p in J])
        e = np.zeros(len(J))
        e[-1] = 1.0
        u = np.linalg.solve(B, e)
        w = np.linalg.solve(B.T, e)
        s = 1.0 / np.sqrt(u[-1])
        gl.extend(w * s)
        h.extend(u * s)
    return np.array(gl), np.array(h)
