"""FP64 CPU reference of the learned FSAI preconditioner -- TEST INFRASTRUCTURE.

The learned factorised sparse approximate inverse has no counterpart in the
reference library; this module restates, in plain numpy FP64, exactly what
the GPU kernels of tnl_b200/csrc/lfsai.cu compute, so that the tests can
check the GPU features, network outputs, losses and gradients, and check
this backpropagation itself against finite differences.

Definitions (shared with lfsai.cu):

* Pattern of G, row i: level 0 -- the stored columns j <= i of A (the
  lower triangle with the diagonal); level 1 -- the columns j <= i of the
  pattern of A^2 (i, its neighbours and their neighbours: one level of
  fill).  At most 8 columns per row; they occupy the right-aligned slots
  8-k .. 7 (slot 7 is the diagonal).
* Scaling s_j = 1/sqrt(a_jj); B = S A S has a unit diagonal.
* Features f (32): f[0..27] = B(J_p, J_q) for the slot pairs p < q in the
  order (0,1) (0,2) .. (0,7) (1,2) .. (6,7) (0 when a slot is empty or the
  entry is not stored); f[28..30] = B(i, j) for the first three stored
  columns j > i; f[31] = k/8.
* Network: h1 = relu(W1 f + b1), h2 = relu(W2 h1 + b2), h3 = relu(W3 h2 + b3),
  o = W4 h3 + b4 with W1 64x32, W2 W3 64x64, W4 8x64.  Every layer input
  and every weight is rounded to BF16 (round to nearest even) before the
  product; sums and biases are FP32 on the GPU, FP64 here.
* G'_i: slot 7 = exp(o_7), occupied slots t < 7 = o_t.  G_ij = G'_i,slot(j) s_j,
  so G A G^T = G' B G'^T.
* Probe loss over probes z_p: L = (1/(n P)) sum_p ||z_p - G A G^T z_p||^2 with
  gradient dL/dG = -(2/(n P)) sum_p (u_p w_p^T + z_p q_p^T) on the pattern,
  where w = A G^T z, u = z - G w, q = A G^T u.
* Kaporin loss (exact, no probes): K = log(T/n) - (2/n) sum_i log G'_ii with
  T = sum_i G'_i B[J,J] G'_i^T = trace(G A G^T); up to a constant it is the
  log of Kaporin's condition number of G A G^T, which classical FSAI
  minimises over a given pattern.  dK/dG'_i = (2/T) B[J,J] G'_i - (2/n)
  e_last / G'_ii.
* Warm start: L = (1/n) sum_i ||G'_i - target'_i||^2 over the occupied
  slots, the target being classical FSAI on the lower pattern of A (level
  0), zero on the fill slots of a level-1 pattern.

Parameter vector layout (float32, 10952 entries): W1 (64x32 row-major), b1,
W2 (64x64), b2, W3, b3, W4 (8x64), b4.
"""
from __future__ import annotations

import numpy as np

F, H, K = 32, 64, 8
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


def pattern(A, level: int = 0):
    """Per row: the sorted columns of G's pattern (level 0: lower triangle of
    A; level 1: lower triangle of the pattern of A^2); raises if a row has
    more than 8."""
    rp, cols = A.rowptr, A.cols
    adj = [set(int(x) for x in cols[rp[i]:rp[i + 1]] if x >= 0) | {i} for i in range(A.n)]
    pat = []
    for i in range(A.n):
        if level == 0:
            low = sorted(int(x) for x in cols[rp[i]:rp[i + 1]] if 0 <= x <= i)
        else:
            reach = set(adj[i])
            for l in adj[i]:
                reach |= adj[l]
            low = sorted(j for j in reach if j <= i)
        if len(low) > K:
            raise ValueError("learned FSAI: more than 8 entries in a row of the pattern")
        pat.append(low)
    return pat


PAIRS = [(p, q) for p in range(K) for q in range(p + 1, K)]


def _row_dict(A):
    rp, cols, vals = A.rowptr, A.cols, A.vals
    return [dict(zip(cols[rp[i]:rp[i + 1]].tolist(), vals[rp[i]:rp[i + 1]].tolist())) for i in range(A.n)]


def features(A, pat=None, level: int = 0):
    pat = pattern(A, level) if pat is None else pat
    rows = _row_dict(A)
    d = np.array([rows[i].get(i, 0.0) for i in range(A.n)], np.float64)
    s = 1.0 / np.sqrt(d)
    f = np.zeros((A.n, F))
    for i in range(A.n):
        J = pat[i]
        k = len(J)
        slot_col = [None] * K
        for t, j in enumerate(J):
            slot_col[K - k + t] = j
        for m, (p, q) in enumerate(PAIRS):
            jp, jq = slot_col[p], slot_col[q]
            if jp is not None and jq is not None:
                f[i, m] = rows[jp].get(jq, 0.0) * s[jp] * s[jq]
        upper = sorted(j for j in rows[i] if j > i)[:3]
        for m, j in enumerate(upper):
            f[i, 28 + m] = rows[i][j] * s[i] * s[j]
        f[i, 31] = k / 8.0
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
            gp = np.exp(o[i, K - 1]) if slot == K - 1 else o[i, slot]
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


def _do_from_dG(dG, o, s, pat):
    """dL/do from dL/dG on the pattern (CSR order)."""
    do = np.zeros_like(o)
    q = 0
    for i, J in enumerate(pat):
        k = len(J)
        for t, j in enumerate(J):
            slot = K - k + t
            do[i, slot] += dG[q] * s[j] * (np.exp(o[i, K - 1]) if slot == K - 1 else 1.0)
            q += 1
    return do


def loss_and_grad(theta, A, probes, level: int = 0):
    """Probe loss L and dL/dtheta (straight-through for the BF16 rounding)."""
    f, s, pat = features(A, level=level)
    o, cache = forward(theta, f)
    vals = g_values(o, s, pat)
    Gm = g_matrix(vals, pat, A.n)
    L, dG = loss_and_grad_G(A, Gm, probes)
    return L, backward(theta, cache, _do_from_dG(dG, o, s, pat))


def kaporin_and_grad(theta, A, level: int = 0):
    """Kaporin loss K and dK/dtheta (straight-through for the BF16 rounding)."""
    f, s, pat = features(A, level=level)
    o, cache = forward(theta, f)
    rows = _row_dict(A)
    n = A.n
    gps, Bs = [], []
    T = 0.0
    logdiag = 0.0
    for i, J in enumerate(pat):
        k = len(J)
        gp = np.array([np.exp(o[i, K - 1]) if K - k + t == K - 1 else o[i, K - k + t] for t in range(k)])
        B = np.array([[rows[p].get(q, 0.0) * s[p] * s[q] for q in J] for p in J])
        gps.append(gp)
        Bs.append(B)
        T += float(gp @ B @ gp)
        logdiag += np.log(gp[-1])
    L = np.log(T / n) - 2.0 * logdiag / n
    do = np.zeros_like(o)
    for i, J in enumerate(pat):
        k = len(J)
        dgp = (2.0 / T) * (Bs[i] @ gps[i])
        dgp[-1] -= 2.0 / (n * gps[i][-1])
        for t in range(k):
            slot = K - k + t
            do[i, slot] = dgp[t] * (gps[i][-1] if slot == K - 1 else 1.0)
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


def fsai_classical(A, level: int = 0):
    """Kolotilina-Yeremin FSAI values on the level-0 or level-1 lower pattern
    (FP64, per row: A[J,J] g = e_last, G_i = g / sqrt(g_last)); CSR order of
    the pattern."""
    rows = _row_dict(A)
    out = []
    for i, J in enumerate(pattern(A, level) if level else [sorted(j for j in rows[i] if 0 <= j <= i)
                                                              for i in range(A.n)]):
        B = np.array([[rows[p].get(q, 0.0) for q in J] for p in J])
        e = np.zeros(len(J))
        e[-1] = 1.0
        g = np.linalg.solve(B, e)
        out.extend(g / np.sqrt(g[-1]))
    return np.array(out)


def fit_target(A, level: int = 0):
    """Warm-start target on G's level-`level` pattern (CSR order): classical
    FSAI of the level-0 pattern, zero on the fill slots."""
    rows = _row_dict(A)
    narrow = fsai_classical(A, 0)
    out, q = [], 0
    for i, J in enumerate(pattern(A, level)):
        low = sorted(j for j in rows[i] if 0 <= j <= i)
        vals = dict(zip(low, narrow[q:q + len(low)]))
        q += len(low)
        out.extend(vals.get(j, 0.0) for j in J)
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


# ------------------------------------------------------------------------
# Two-factor learned FSAI for a nonsymmetric A (M^-1 = G_U G_L, G_L lower
# and G_U upper on the level-0 pattern, H = G_U^T stored on the lower one).
#
# * Features f (32, zero padded) of row i, with B = S A S: f[0..11] =
#   B(J_p, J_q), B(J_q, J_p) for the 6 pairs p < q of the last four slots
#   (slots 4..7: (4,5) (4,6) (4,7) (5,6) (5,7) (6,7)); f[12..14] = B(i, j)
#   for the first three stored columns j > i; f[15..17] = B(j, i) for the
#   same j; f[31] = k/8.  At most 4 entries per row.
# * Outputs: o[4..7] the row of G'_L, o[0..3] the row of H' (right-aligned
#   slots 4 - k .. 3 and 8 - k .. 7); the diagonals exp(o_3), exp(o_7).
#   G_L[i, j] = G'_L s_j, H[i, j] = H' s_j (G_L A G_U = G'_L B G'_U).
# * Probe loss L = (1/(n P)) sum_p ||z_p - G_L A G_U z_p||^2 with
#   dL/dG_L = -(2/(n P)) sum_p u w^T on the pattern, w = A G_U z,
#   u = z - G_L w, and dL/dH_ij = -(2/(n P)) sum_p z_i q_j, q = A^T G_L^T u.
# * Warm start: L = (1/n) sum_i (||G'_L,i - target_L||^2 + ||H'_i -
#   target_H||^2) towards classical two-factor FSAI (fsai2_classical).

PAIRS2 = [(4, 5), (4, 6), (4, 7), (5, 6), (5, 7), (6, 7)]


def features2(A):
    pat = pattern(A, 0)
    rows = _row_dict(A)
    d = np.array([rows[i].get(i, 0.0) for i in range(A.n)], np.float64)
    s = 1.0 / np.sqrt(d)
    f = np.zeros((A.n, F))
    for i in range(A.n):
        J = pat[i]
        k = len(J)
        if k > 4:
            raise ValueError("two-factor learned FSAI: more than 4 entries in a row of the lower pattern")
        slot_col = [None] * K
        for t, j in enumerate(J):
            slot_col[K - k + t] = j
        for m, (p, q) in enumerate(PAIRS2):
            jp, jq = slot_col[p], slot_col[q]
            if jp is not None and jq is not None:
                f[i, 2 * m] = rows[jp].get(jq, 0.0) * s[jp] * s[jq]
                f[i, 2 * m + 1] = rows[jq].get(jp, 0.0) * s[jp] * s[jq]
        upper = sorted(j for j in rows[i] if j > i)[:3]
        for m, j in enumerate(upper):
            f[i, 12 + m] = rows[i][j] * s[i] * s[j]
            f[i, 15 + m] = rows[j].get(i, 0.0) * s[i] * s[j]
        f[i, 31] = k / 8.0
    return f, s, pat


def g2_values(o, s, pat):
    """(G_L values, H values) on the lower pattern, CSR order."""
    gl, h = [], []
    for i, J in enumerate(pat):
        k = len(J)
        for t, j in enumerate(J):
            sl, sh = K - k + t, 4 - k + t
            gl.append((np.exp(o[i, K - 1]) if sl == K - 1 else o[i, sl]) * s[j])
            h.append((np.exp(o[i, 3]) if sh == 3 else o[i, sh]) * s[j])
    return np.array(gl), np.array(h)


def loss_and_grad2(theta, A, probes):
    """Two-factor probe loss and its gradient (straight-through BF16)."""
    import scipy.sparse as sp

    f, s, pat = features2(A)
    o, cache = forward(theta, f)
    gl, h = g2_values(o, s, pat)
    GL = g_matrix(gl, pat, A.n)
    H = g_matrix(h, pat, A.n)
    As = sp.csr_matrix((A.vals, A.cols, A.rowptr), shape=(A.n, A.n))
    n, P = probes.shape
    Z = probes
    W = As @ (H.T @ Z)
    U = Z - GL @ W
    Q = As.T @ (GL.T @ U)
    L = float(np.sum(U * U)) / (n * P)
    coo = GL.tocoo()
    gi, gj = coo.row, coo.col
    order = np.lexsort((gj, gi))
    c = -(2.0 / (n * P))
    dGL = (c * np.sum(U[gi] * W[gj], axis=1))[order]
    dH = (c * np.sum(Z[gi] * Q[gj], axis=1))[order]
    do = np.zeros_like(o)
    q = 0
    for i, J in enumerate(pat):
        k = len(J)
        for t, j in enumerate(J):
            sl, sh = K - k + t, 4 - k + t
            do[i, sl] += dGL[q] * s[j] * (np.exp(o[i, K - 1]) if sl == K - 1 else 1.0)
            do[i, sh] += dH[q] * s[j] * (np.exp(o[i, 3]) if sh == 3 else 1.0)
            q += 1
    return L, backward(theta, cache, do)
