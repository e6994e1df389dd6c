// lfsai.cu -- learned factorised sparse approximate inverse (no counterpart
// in the reference library).
//
// A per-row network maps local, scale-free coefficients of A to the values of
// G on a lower-triangular pattern with at most 8 entries per row: the lower
// triangle of A (level 0) or of the pattern of A^2 (level 1: one level of
// fill, 7 entries per row of a 5-point operator).  The preconditioner is
// M^-1 = G^T G, applied by two SpMVs (fsai.cu), so CG stays symmetric
// positive definite.  Three training objectives, each with its gradient
// dL/dG on the pattern:
//  * the probe estimate of ||I - G A G^T||_F^2 / n,
//       L = 1/(n P) sum_p ||z_p - G A G^T z_p||^2,
//       dL/dG = -2/(n P) sum_p (u_p w_p^T + z_p q_p^T),
//    with w = A G^T z, u = z - G w, q = A G^T u -- every product a library
//    SpMV; the probes are Rademacher vectors and residuals the solver leaves;
//  * the Kaporin loss K = log(trace(G A G^T)/n) - (2/n) sum_i log G_ii (+ a
//    constant): the log of Kaporin's condition number of G A G^T, exact,
//    from the local blocks A[J,J] (classical FSAI is its minimiser on a
//    given pattern);
//  * the warm start: regression onto classical FSAI of the level-0 pattern
//    (zero on the fill entries of a level-1 pattern).
//
// Definitions of the features, the network (32 -> 64 -> 64 -> 64 -> 8, ReLU,
// BF16 weights and layer inputs, FP32 accumulation), the output map
// (G'_diag = exp(o_7), G_ij = G'_ij / sqrt(a_jj)) and the parameter layout
// are written out in the CPU reference the tests use (oracle/lfsai_ref.py);
// this file implements exactly those.  Dense layers, forward and backward:
// the tensor-core path (lfsai_tc.cu, tcgen05 with accumulators in TMEM) by
// default, else the CUDA-core kernels below, which also serve as its
// on-GPU reference.
#include <cmath>
#include <vector>

#include "fsai.cuh"
#include "internal.cuh"
#include "lfsai.cuh"
#include "reduce.cuh"
#include "segview.cuh"

namespace tnlb {

namespace lf {

__device__ __forceinline__ float bf16r(float x)
{
   // round to nearest even BF16, kept in FP32
   uint32_t u = __float_as_uint(x);
   u = (u + 0x7FFFu + ((u >> 16) & 1u)) & 0xFFFF0000u;
   return __uint_as_float(u);
}

template <typename Real>
__device__ __forceinline__ Real lookup(const int32_t* rp, const int32_t* cols, const Real* vals, int32_t r, int32_t c)
{
   int32_t lo = rp[r], hi = rp[r + 1] - 1;
   while (lo <= hi) {
      const int32_t mid = (lo + hi) >> 1;
      const int32_t cm = cols[mid];
      if (cm == c) return vals[mid];
      if (cm < c)
         lo = mid + 1;
      else
         hi = mid - 1;
   }
   return Real(0);
}

// Features (n x 32, FP32) and scaling s = 1/sqrt(diag) from A (CSR, ascending
// columns) and G's pattern: the scaled entries B(J_p, J_q) of the 28 slot
// pairs p < q, the first three scaled entries right of the diagonal, k/8.
template <typename Real>
__global__ void k_features(const int32_t* __restrict__ arp, const int32_t* __restrict__ acols,
                           const Real* __restrict__ avals, const int32_t* __restrict__ grp,
                           const int32_t* __restrict__ gcols, int32_t n, float* __restrict__ f, Real* __restrict__ s,
                           int32_t* __restrict__ err)
{
   const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (i >= n) return;
   const int32_t b = grp[i], k = grp[i + 1] - b;
   if (k > kLfK || k < 1) {
      atomicExch(err, 1);
      for (int q = 0; q < kLfF; q++) f[i * kLfF + q] = 0.f;
      return;
   }
   int32_t slot_col[kLfK];
   double slot_s[kLfK];
#pragma unroll
   for (int t = 0; t < kLfK; t++) {
      slot_col[t] = -1;
      slot_s[t] = 0.0;
   }
   for (int t = 0; t < k; t++) {
      const int32_t j = gcols[b + t];
      slot_col[kLfK - k + t] = j;
      slot_s[kLfK - k + t] = 1.0 / sqrt((double)lookup(arp, acols, avals, j, j));
   }
   int m = 0;
   for (int p = 0; p < kLfK; p++)
      for (int q = p + 1; q < kLfK; q++, m++) {
         const int32_t jp = slot_col[p], jq = slot_col[q];
         float v = 0.f;
         if (jp >= 0 && jq >= 0) v = (float)((double)lookup(arp, acols, avals, jp, jq) * slot_s[p] * slot_s[q]);
         f[i * kLfF + m] = v;
      }
   const double si = slot_s[kLfK - 1];
   int up = 0;
   for (int32_t q = arp[i]; q < arp[i + 1] && up < 3; q++) {
      const int32_t j = acols[q];
      if (j > i) {
         const double sj = 1.0 / sqrt((double)lookup(arp, acols, avals, j, j));
         f[i * kLfF + kLfPairs + up++] = (float)((double)avals[q] * si * sj);
      }
   }
   for (; up < 3; up++) f[i * kLfF + kLfPairs + up] = 0.f;
   f[i * kLfF + kLfF - 1] = (float)k / (float)kLfK;
   s[i] = (Real)si;
}

// BF16-rounded copy of the weights (biases kept FP32) for the forward pass.
__global__ void k_round_weights(const float* __restrict__ theta, float* __restrict__ wr)
{
   for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < kLfParams; q += gridDim.x * blockDim.x) {
      const bool bias = (q >= kLfB1 && q < kLfW2) || (q >= kLfB2 && q < kLfW3) || (q >= kLfB3 && q < kLfW4) || q >= kLfB4;
      wr[q] = bias ? theta[q] : bf16r(theta[q]);
   }
}

// One layer of the network on CUDA cores, one thread per row:
// out = act(W bf16(in) + b); `in` has `fin` columns, `out` `fout`.
// Stores the pre-rounding output (the next layer rounds it again).
template <int FIN, int FOUT, bool RELU>
__global__ void __launch_bounds__(128) k_layer(const float* __restrict__ in, int64_t n, const float* __restrict__ W,
                                               const float* __restrict__ bias, float* __restrict__ out)
{
   __shared__ float sW[FOUT * FIN];
   __shared__ float sb[FOUT];
   for (int q = threadIdx.x; q < FOUT * FIN; q += blockDim.x) sW[q] = W[q];
   for (int q = threadIdx.x; q < FOUT; q += blockDim.x) sb[q] = bias[q];
   __syncthreads();
   const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (r >= n) return;
   float x[FIN];
#pragma unroll
   for (int q = 0; q < FIN; q++) x[q] = bf16r(in[r * FIN + q]);
   for (int o = 0; o < FOUT; o++) {
      float acc = sb[o];
#pragma unroll
      for (int q = 0; q < FIN; q++) acc = fmaf(sW[o * FIN + q], x[q], acc);
      out[r * FOUT + o] = RELU ? fmaxf(acc, 0.f) : acc;
   }
}

// G values on G's pattern from the network outputs o (n x 4).
template <typename Real>
__global__ void k_g_values(const float* __restrict__ o, const Real* __restrict__ s, const int32_t* __restrict__ grp,
                           const int32_t* __restrict__ gcols, int32_t n, Real* __restrict__ gvals)
{
   const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (i >= n) return;
   const int32_t b = grp[i], k = grp[i + 1] - b;
   for (int t = 0; t < k; t++) {
      const int slot = kLfK - k + t;
      const double gp = slot == kLfK - 1 ? exp((double)o[i * kLfK + slot]) : (double)o[i * kLfK + slot];
      gvals[b + t] = (Real)(gp * (double)s[gcols[b + t]]);
   }
}

// u = z - v and sum of u^2 (for the loss)
template <typename Real>
__global__ void __launch_bounds__(kRedThreads) k_resid(int64_t n, const Real* __restrict__ z, const Real* __restrict__ v,
                                                       Real* __restrict__ u, RedWork w, double* __restrict__ out)
{
   double acc = 0;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
      const Real ui = z[i] - v[i];
      u[i] = ui;
      acc += (double)ui * (double)ui;
   }
   double vv[1] = {acc};
   if (publish_and_arrive<1>(vv, w)) {
      double t[1];
      gather_totals<1>(t, w);
      if (threadIdx.x == 0) *out += t[0];
   }
}

// dG_ij += c (u_i w_j + z_i q_j) on G's pattern (thread per row)
template <typename Real>
__global__ void k_dg(const int32_t* __restrict__ grp, const int32_t* __restrict__ gcols, int32_t n,
                     const Real* __restrict__ u, const Real* __restrict__ w, const Real* __restrict__ z,
                     const Real* __restrict__ q, double c, double* __restrict__ dg)
{
   const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (i >= n) return;
   const double ui = u[i], zi = z[i];
   for (int32_t e = grp[i]; e < grp[i + 1]; e++) {
      const int32_t j = gcols[e];
      dg[e] += c * (ui * (double)w[j] + zi * (double)q[j]);
   }
}

// dL/do from dL/dG (FP32 per row, 4 slots)
template <typename Real>
__global__ void k_do(const double* __restrict__ dg, const float* __restrict__ o, const Real* __restrict__ s,
                     const int32_t* __restrict__ grp, const int32_t* __restrict__ gcols, int32_t n,
                     float* __restrict__ dout)
{
   const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (i >= n) return;
   float d[kLfK];
#pragma unroll
   for (int t = 0; t < kLfK; t++) d[t] = 0.f;
   const int32_t b = grp[i], k = grp[i + 1] - b;
   for (int t = 0; t < k; t++) {
      const int slot = kLfK - k + t;
      double v = dg[b + t] * (double)s[gcols[b + t]];
      if (slot == kLfK - 1) v *= exp((double)o[i * kLfK + slot]);
      d[slot] = (float)v;
   }
#pragma unroll
   for (int t = 0; t < kLfK; t++) dout[i * kLfK + t] = d[t];
}

// delta_in = (W^T delta_out) masked by (h_in > 0), thread per row.
template <int FIN, int FOUT>
__global__ void __launch_bounds__(128) k_back_layer(const float* __restrict__ dout, const float* __restrict__ h_in,
                                                    int64_t n, const float* __restrict__ W, float* __restrict__ din)
{
   __shared__ float sW[FOUT * FIN];
   for (int q = threadIdx.x; q < FOUT * FIN; q += blockDim.x) sW[q] = W[q];
   __syncthreads();
   const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (r >= n) return;
   float d[FOUT];
#pragma unroll
   for (int o = 0; o < FOUT; o++) d[o] = dout[r * FOUT + o];
   for (int q = 0; q < FIN; q++) {
      float acc = 0.f;
#pragma unroll
      for (int o = 0; o < FOUT; o++) acc = fmaf(sW[o * FIN + q], d[o], acc);
      din[r * FIN + q] = h_in[r * FIN + q] > 0.f ? acc : 0.f;
   }
}

// Weight gradient of one layer: dW (FOUT x FIN) = sum_r dout_r^T bf16(in_r),
// db = sum_r dout_r.  Per block a chunk of rows; partials then a reduction.
template <int FIN, int FOUT>
__global__ void __launch_bounds__(256) k_wgrad(const float* __restrict__ dout, const float* __restrict__ in, int64_t n,
                                               int64_t rows_per_block, float* __restrict__ partial)
{
   constexpr int NW = FOUT * FIN + FOUT;
   __shared__ float sd[32][FOUT];
   __shared__ float sx[32][FIN];
   float acc[(NW + 255) / 256];
#pragma unroll
   for (int q = 0; q < (NW + 255) / 256; q++) acc[q] = 0.f;
   const int64_t r0 = (int64_t)blockIdx.x * rows_per_block;
   const int64_t r1 = imin64(n, r0 + rows_per_block);
   for (int64_t rb = r0; rb < r1; rb += 32) {
      __syncthreads();
      for (int q = threadIdx.x; q < 32 * FOUT; q += 256) {
         const int64_t r = rb + q / FOUT;
         sd[q / FOUT][q % FOUT] = r < r1 ? dout[r * FOUT + q % FOUT] : 0.f;
      }
      for (int q = threadIdx.x; q < 32 * FIN; q += 256) {
         const int64_t r = rb + q / FIN;
         sx[q / FIN][q % FIN] = r < r1 ? bf16r(in[r * FIN + q % FIN]) : 0.f;
      }
      __syncthreads();
#pragma unroll
      for (int q = 0; q < (NW + 255) / 256; q++) {
         const int e = threadIdx.x + q * 256;
         if (e < FOUT * FIN) {
            const int o = e / FIN, c = e % FIN;
            float a = acc[q];
            for (int rr = 0; rr < 32; rr++) a = fmaf(sd[rr][o], sx[rr][c], a);
            acc[q] = a;
         }
         else if (e < NW) {
            const int o = e - FOUT * FIN;
            float a = acc[q];
            for (int rr = 0; rr < 32; rr++) a += sd[rr][o];
            acc[q] = a;
         }
      }
   }
#pragma unroll
   for (int q = 0; q < (NW + 255) / 256; q++) {
      const int e = threadIdx.x + q * 256;
      if (e < NW) partial[(int64_t)blockIdx.x * NW + e] = acc[q];
   }
}

// Sum block partials into the gradient slice [W | b] (FP64 sums, fixed order).
__global__ void k_sum_partials(const float* __restrict__ partial, int blocks, int nw, float* __restrict__ gW,
                               float* __restrict__ gb, int nwW)
{
   const int e = blockIdx.x * blockDim.x + threadIdx.x;
   if (e >= nw) return;
   double s = 0;
   for (int b = 0; b < blocks; b++) s += partial[(int64_t)b * nw + e];
   if (e < nwW)
      gW[e] = (float)s;
   else
      gb[e - nwW] = (float)s;
}

__global__ void k_adam(float* __restrict__ theta, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, int np, float lr, float b1, float b2, float eps, float c1, float c2)
{
   const int q = blockIdx.x * blockDim.x + threadIdx.x;
   if (q >= np) return;
   const float gq = g[q];
   const float mq = b1 * m[q] + (1.f - b1) * gq;
   const float vq = b2 * v[q] + (1.f - b2) * gq * gq;
   m[q] = mq;
   v[q] = vq;
   theta[q] -= lr * (mq / c1) / (sqrtf(vq / c2) + eps);
}

// Supervised warm start: dL/do for L = 1/n sum_rows ||G'_row - target'||^2
// over occupied slots (target' = classical FSAI values in the scaled frame).
template <typename Real>
__global__ void __launch_bounds__(kRedThreads) k_fit_do(const float* __restrict__ o, const Real* __restrict__ target,
                                                        const Real* __restrict__ s, const int32_t* __restrict__ grp,
                                                        const int32_t* __restrict__ gcols, int32_t n,
                                                        float* __restrict__ dout, RedWork w, double* __restrict__ loss)
{
   double acc = 0;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
      float d[kLfK];
#pragma unroll
      for (int t = 0; t < kLfK; t++) d[t] = 0.f;
      const int32_t b = grp[i], k = grp[i + 1] - b;
      for (int t = 0; t < k; t++) {
         const int slot = kLfK - k + t;
         const double tp = (double)target[b + t] / (double)s[gcols[b + t]];
         const double op = o[i * kLfK + slot];
         const double gp = slot == kLfK - 1 ? exp(op) : op;
         const double e = gp - tp;
         acc += e * e;
         d[slot] = (float)(2.0 * e * (slot == kLfK - 1 ? gp : 1.0) / n);
      }
      for (int t = 0; t < kLfK; t++) dout[i * kLfK + t] = d[t];
   }
   double vv[1] = {acc};
   if (publish_and_arrive<1>(vv, w)) {
      double t[1];
      gather_totals<1>(t, w);
      if (threadIdx.x == 0) *loss = t[0] / n;
   }
}

// Kaporin loss, pass 1: per row q_i = G'_i B[J,J] G'_i^T (B = S A S) and
// log G'_ii = o_7, summed over all rows in a fixed block order into
// tot[0] = T = trace(G A G^T) and tot[1] = sum_i log G'_ii.
template <typename Real>
__device__ __forceinline__ int kap_row(const int32_t* arp, const int32_t* acols, const Real* avals,
                                       const int32_t* grp, const int32_t* gcols, const float* o, int64_t i,
                                       int32_t (&col)[kLfK], double (&sc)[kLfK], double (&g)[kLfK])
{
   const int32_t b = grp[i], k = grp[i + 1] - b;
   for (int t = 0; t < k; t++) {
      col[t] = gcols[b + t];
      sc[t] = 1.0 / sqrt((double)lookup(arp, acols, avals, col[t], col[t]));
      const int slot = kLfK - k + t;
      g[t] = slot == kLfK - 1 ? exp((double)o[i * kLfK + slot]) : (double)o[i * kLfK + slot];
   }
   return k;
}

template <typename Real>
__global__ void __launch_bounds__(kRedThreads) k_kap_sums(const int32_t* __restrict__ arp,
                                                          const int32_t* __restrict__ acols,
                                                          const Real* __restrict__ avals,
                                                          const int32_t* __restrict__ grp,
                                                          const int32_t* __restrict__ gcols, int32_t n,
                                                          const float* __restrict__ o, RedWork w,
                                                          double* __restrict__ tot)
{
   double tr = 0, ld = 0;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
      int32_t col[kLfK];
      double sc[kLfK], g[kLfK];
      const int k = kap_row(arp, acols, avals, grp, gcols, o, i, col, sc, g);
      double q = 0;
      for (int p = 0; p < k; p++) {
         double r = 0;
         for (int c = 0; c < k; c++) r += (double)lookup(arp, acols, avals, col[p], col[c]) * sc[p] * sc[c] * g[c];
         q += g[p] * r;
      }
      tr += q;
      ld += (double)o[i * kLfK + kLfK - 1];
   }
   double vv[2] = {tr, ld};
   if (publish_and_arrive<2>(vv, w)) {
      double t[2];
      gather_totals<2>(t, w);
      if (threadIdx.x == 0) {
         tot[0] = t[0];
         tot[1] = t[1];
      }
   }
}

// Kaporin loss, pass 2: dK/do per row from dK/dG'_i = (2/T) B[J,J] G'_i -
// (2/n) e_last / G'_ii (the diagonal slot through G'_ii = exp(o_7)).
template <typename Real>
__global__ void k_kap_do(const int32_t* __restrict__ arp, const int32_t* __restrict__ acols,
                         const Real* __restrict__ avals, const int32_t* __restrict__ grp,
                         const int32_t* __restrict__ gcols, int32_t n, const float* __restrict__ o,
                         const double* __restrict__ tot, float* __restrict__ dout)
{
   const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (i >= n) return;
   const double T = tot[0];
   int32_t col[kLfK];
   double sc[kLfK], g[kLfK];
   const int k = kap_row(arp, acols, avals, grp, gcols, o, i, col, sc, g);
   float d[kLfK];
#pragma unroll
   for (int t = 0; t < kLfK; t++) d[t] = 0.f;
   for (int p = 0; p < k; p++) {
      double r = 0;
      for (int c = 0; c < k; c++) r += (double)lookup(arp, acols, avals, col[p], col[c]) * sc[p] * sc[c] * g[c];
      double dg = (2.0 / T) * r;
      if (p == k - 1) dg = (dg - 2.0 / ((double)n * g[k - 1])) * g[k - 1];
      d[kLfK - k + p] = (float)dg;
   }
#pragma unroll
   for (int t = 0; t < kLfK; t++) dout[i * kLfK + t] = d[t];
}

// Warm-start target on G's pattern: the values of `src` (classical FSAI of
// the level-0 pattern, rows sorted by column) where its pattern has the
// column, zero on the fill entries.
template <typename Real>
__global__ void k_map_target(const int32_t* __restrict__ grp, const int32_t* __restrict__ gcols,
                             const int32_t* __restrict__ srp, const int32_t* __restrict__ scols,
                             const Real* __restrict__ svals, int32_t n, Real* __restrict__ out)
{
   const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (i >= n) return;
   int32_t q = srp[i];
   const int32_t qe = srp[i + 1];
   for (int32_t e = grp[i]; e < grp[i + 1]; e++) {
      const int32_t j = gcols[e];
      while (q < qe && scols[q] < j) q++;
      out[e] = (q < qe && scols[q] == j) ? svals[q] : Real(0);
   }
}

// ---- two factors (nonsymmetric A): G_L and H = G_U^T on the lower pattern
// of A (at most 4 entries a row).  Features: B(J_p, J_q) and B(J_q, J_p) of
// the 6 pairs of slots 4..7, B(i, j) and B(j, i) of the first three stored
// columns j > i, k/8.  Outputs: o[4..7] the row of G'_L, o[0..3] that of
// H' (diagonals exp(o_7), exp(o_3)).
template <typename Real>
__global__ void k_features2(const int32_t* __restrict__ arp, const int32_t* __restrict__ acols,
                            const Real* __restrict__ avals, const int32_t* __restrict__ grp,
                            const int32_t* __restrict__ gcols, int32_t n, float* __restrict__ f,
                            Real* __restrict__ s, int32_t* __restrict__ err)
{
   const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (i >= n) return;
   const int32_t b = grp[i], k = grp[i + 1] - b;
   for (int q = 0; q < kLfF; q++) f[i * kLfF + q] = 0.f;
   if (k > 4 || k < 1) {
      atomicExch(err, 1);
      return;
   }
   int32_t slot_col[4];
   double slot_s[4];
   for (int t = 0; t < 4; t++) {
      slot_col[t] = -1;
      slot_s[t] = 0.0;
   }
   for (int t = 0; t < k; t++) {
      const int32_t j = gcols[b + t];
      slot_col[4 - k + t] = j;
      slot_s[4 - k + t] = 1.0 / sqrt((double)lookup(arp, acols, avals, j, j));
   }
   int m = 0;
   for (int p = 0; p < 4; p++)
      for (int q = p + 1; q < 4; q++, m++) {
         const int32_t jp = slot_col[p], jq = slot_col[q];
         if (jp >= 0 && jq >= 0) {
            const double sc = slot_s[p] * slot_s[q];
            f[i * kLfF + 2 * m] = (float)((double)lookup(arp, acols, avals, jp, jq) * sc);
            f[i * kLfF + 2 * m + 1] = (float)((double)lookup(arp, acols, avals, jq, jp) * sc);
         }
      }
   const double si = slot_s[3];
   int up = 0;
   for (int32_t q = arp[i]; q < arp[i + 1] && up < 3; q++) {
      const int32_t j = acols[q];
      if (j > i) {
         const double sj = 1.0 / sqrt((double)lookup(arp, acols, avals, j, j));
         f[i * kLfF + 12 + up] = (float)((double)avals[q] * si * sj);
         f[i * kLfF + 15 + up] = (float)((double)lookup(arp, acols, avals, j, (int32_t)i) * si * sj);
         up++;
      }
   }
   f[i * kLfF + kLfF - 1] = (float)k / (float)kLfK;
   s[i] = (Real)si;
}

// G_L and H values on the pattern from the outputs.
template <typename Real>
__global__ void k_g2_values(const float* __restrict__ o, const Real* __restrict__ s, const int32_t* __restrict__ grp,
                            const int32_t* __restrict__ gcols, int32_t n, Real* __restrict__ gl, Real* __restrict__ h)
{
   const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (i >= n) return;
   const int32_t b = grp[i], k = grp[i + 1] - b;
   for (int t = 0; t < k; t++) {
      const int sl = kLfK - k + t, sh = 4 - k + t;
      const double sj = (double)s[gcols[b + t]];
      const double vl = sl == kLfK - 1 ? exp((double)o[i * kLfK + sl]) : (double)o[i * kLfK + sl];
      const double vh = sh == 3 ? exp((double)o[i * kLfK + sh]) : (double)o[i * kLfK + sh];
      gl[b + t] = (Real)(vl * sj);
      h[b + t] = (Real)(vh * sj);
   }
}

// dG_L_ij += c u_i w_j and dH_ij += c z_i q_j on the pattern (thread per row)
template <typename Real>
__global__ void k_dg2(const int32_t* __restrict__ grp, const int32_t* __restrict__ gcols, int32_t n,
                      const Real* __restrict__ u, const Real* __restrict__ w, const Real* __restrict__ z,
                      const Real* __restrict__ q, double c, double* __restrict__ dgl, double* __restrict__ dh)
{
   const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (i >= n) return;
   const double ui = u[i], zi = z[i];
   for (int32_t e = grp[i]; e < grp[i + 1]; e++) {
      const int32_t j = gcols[e];
      dgl[e] += c * ui * (double)w[j];
      dh[e] += c * zi * (double)q[j];
   }
}

// dL/do from dL/dG_L (slots 4..7) and dL/dH (slots 0..3)
template <typename Real>
__global__ void k_do2(const double* __restrict__ dgl, const double* __restrict__ dh, const float* __restrict__ o,
                      const Real* __restrict__ s, const int32_t* __restrict__ grp, const int32_t* __restrict__ gcols,
                      int32_t n, float* __restrict__ dout)
{
   const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (i >= n) return;
   float d[kLfK];
#pragma unroll
   for (int t = 0; t < kLfK; t++) d[t] = 0.f;
   const int32_t b = grp[i], k = grp[i + 1] - b;
   for (int t = 0; t < k; t++) {
      const int sl = kLfK - k + t, sh = 4 - k + t;
      const double sj = (double)s[gcols[b + t]];
      double vl = dgl[b + t] * sj, vh = dh[b + t] * sj;
      if (sl == kLfK - 1) vl *= exp((double)o[i * kLfK + sl]);
      if (sh == 3) vh *= exp((double)o[i * kLfK + sh]);
      d[sl] = (float)vl;
      d[sh] = (float)vh;
   }
#pragma unroll
   for (int t = 0; t < kLfK; t++) dout[i * kLfK + t] = d[t];
}

// Warm start of the two factors: dL/do and L = 1/n sum over occupied slots
// of (G'_L - target_L)^2 + (H' - target_H)^2 in the scaled frame.
template <typename Real>
__global__ void __launch_bounds__(kRedThreads) k_fit2_do(const float* __restrict__ o, const Real* __restrict__ tgl,
                                                         const Real* __restrict__ th, const Real* __restrict__ s,
                                                         const int32_t* __restrict__ grp,
                                                         const int32_t* __restrict__ gcols, int32_t n,
                                                         float* __restrict__ dout, RedWork w, double* __restrict__ loss)
{
   double acc = 0;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
      float d[kLfK];
#pragma unroll
      for (int t = 0; t < kLfK; t++) d[t] = 0.f;
      const int32_t b = grp[i], k = grp[i + 1] - b;
      for (int t = 0; t < k; t++) {
         const double sj = (double)s[gcols[b + t]];
         for (int f2 = 0; f2 < 2; f2++) {
            const int slot = f2 == 0 ? kLfK - k + t : 4 - k + t;
            const bool diag = f2 == 0 ? slot == kLfK - 1 : slot == 3;
            const double tp = (double)(f2 == 0 ? tgl[b + t] : th[b + t]) / sj;
            const double op = o[i * kLfK + slot];
            const double gp = diag ? exp(op) : op;
            const double e = gp - tp;
            acc += e * e;
            d[slot] = (float)(2.0 * e * (diag ? gp : 1.0) / n);
         }
      }
      for (int t = 0; t < kLfK; t++) dout[i * kLfK + t] = d[t];
   }
   double vv[1] = {acc};
   if (publish_and_arrive<1>(vv, w)) {
      double t[1];
      gather_totals<1>(t, w);
      if (threadIdx.x == 0) *loss = t[0] / n;
   }
}

template <typename Real>
__global__ void k_scatter_src(const int32_t* __restrict__ src, int64_t nnz, const Real* __restrict__ from,
                              Real* __restrict__ to)
{
   for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < nnz; q += (int64_t)gridDim.x * blockDim.x)
      to[src[q]] = from[q];
}

__global__ void k_init_params(uint64_t seed, float* __restrict__ theta)
{
   const int q = blockIdx.x * blockDim.x + threadIdx.x;
   if (q >= kLfParams) return;
   // layer of parameter q: U(-a, a), a = sqrt(6/(fan_in+fan_out)), W4 x 0.1, biases 0
   // in FP64 (correctly rounded sqrt), as the host initialiser, then rounded once to FP32
   double a = 0.0;
   if (q < kLfB1)
      a = sqrt(6.0 / (kLfF + kLfH));
   else if (q >= kLfW2 && q < kLfB2)
      a = sqrt(6.0 / (kLfH + kLfH));
   else if (q >= kLfW3 && q < kLfB3)
      a = sqrt(6.0 / (kLfH + kLfH));
   else if (q >= kLfW4 && q < kLfB4)
      a = sqrt(6.0 / (kLfH + kLfK)) * 0.1;
   uint64_t z = seed * 0x9E3779B97F4A7C15ull + (uint64_t)q;
   z += 0x9E3779B97F4A7C15ull;
   z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
   z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
   z ^= z >> 31;
   const double u = (double)(z >> 11) * (1.0 / 9007199254740992.0);
   theta[q] = (float)((2.0 * u - 1.0) * a);
}

}  // namespace lf

// ------------------------------------------------------------------ host

struct LfsaiMatrix {
   Fsai* F = nullptr;      // pattern of G, transpose map, CSR of A
   DeviceBuffer feat, s;   // n x 16 features, scaling
   DeviceBuffer target;    // classical FSAI values (warm start)
   ~LfsaiMatrix() { fsai_destroy(F); }
};

namespace {

template <typename Real>
tnlb_status build_matrix_ctx(const tnlb_segments* seg, tnlb_real real, const int32_t* cols, const Real* vals,
                             int level, bool two_factor, cudaStream_t st, LfsaiMatrix* M)
{
   TNLB_TRY_STATUS(fsai_create(seg, real, cols, vals, false, st, &M->F, two_factor, two_factor ? 0 : level));
   const int32_t n = seg->n;
   TNLB_TRY_STATUS(M->feat.alloc(sizeof(float) * (size_t)n * kLfF));
   TNLB_TRY_STATUS(M->s.alloc(sizeof(Real) * n));
   DeviceBuffer err;
   TNLB_TRY_STATUS(err.alloc(sizeof(int32_t)));
   TNLB_CUDA_TRY(cudaMemsetAsync(err.ptr, 0, sizeof(int32_t), st));
   auto* kf = two_factor ? lf::k_features2<Real> : lf::k_features<Real>;
   kf<<<grid_for(n, 128), 128, 0, st>>>(M->F->a_rp.as<int32_t>(), M->F->a_cols.as<int32_t>(), M->F->a_vals.as<Real>(),
                                        M->F->g->offsets.as<int32_t>(), M->F->g_cols.as<int32_t>(), n,
                                        M->feat.as<float>(), M->s.as<Real>(), err.as<int32_t>());
   TNLB_CHECK_LAUNCH();
   int32_t h = 0;
   TNLB_CUDA_TRY(cudaMemcpyAsync(&h, err.ptr, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
   TNLB_CUDA_TRY(cudaStreamSynchronize(st));
   TNLB_REQUIRE(h == 0, TNLB_ERR_INVALID_ARGUMENT,
                two_factor ? "learned two-factor FSAI: a row of A's lower triangle holds more than 4 entries"
                           : "learned FSAI: a row of G's pattern holds more than 8 entries");
   return TNLB_OK;
}

}  // namespace

// Forward pass for all rows: o (n x 4); activations h1..h3 kept when `acts`.
tnlb_status lfsai_forward(const tnlb_lfsai* net, const float* feat, int64_t n, float* o, float* h1, float* h2,
                          float* h3, cudaStream_t st)
{
   if (net->use_tc) return lfsai_forward_tc(net, feat, n, o, h1, h2, h3, st);
   const float* wr = net->wround.as<float>();
   const unsigned g = grid_for(n, 128);
   lf::k_layer<kLfF, kLfH, true><<<g, 128, 0, st>>>(feat, n, wr + kLfW1, wr + kLfB1, h1);
   lf::k_layer<kLfH, kLfH, true><<<g, 128, 0, st>>>(h1, n, wr + kLfW2, wr + kLfB2, h2);
   lf::k_layer<kLfH, kLfH, true><<<g, 128, 0, st>>>(h2, n, wr + kLfW3, wr + kLfB3, h3);
   lf::k_layer<kLfH, kLfK, false><<<g, 128, 0, st>>>(h3, n, wr + kLfW4, wr + kLfB4, o);
   TNLB_CHECK_LAUNCH();
   return TNLB_OK;
}

namespace {

// dW, db of one layer from its output deltas and (BF16-rounded) inputs.
template <int FIN, int FOUT>
tnlb_status wgrad_layer(const float* dout, const float* in, int64_t n, int64_t rpb, int blocks, float* part, float* gW,
                        float* gb, cudaStream_t st)
{
   constexpr int nwW = FOUT * FIN;
   lf::k_wgrad<FIN, FOUT><<<blocks, 256, 0, st>>>(dout, in, n, rpb, part);
   lf::k_sum_partials<<<(nwW + FOUT + 255) / 256, 256, 0, st>>>(part, blocks, nwW + FOUT, gW, gb, nwW);
   TNLB_CHECK_LAUNCH();
   return TNLB_OK;
}

// Backward from dL/do through the network into net->grad.
tnlb_status lfsai_backward(tnlb_lfsai* net, const float* feat, int64_t n, const float* h1, const float* h2,
                           const float* h3, const float* dout, cudaStream_t st)
{
   if (net->use_tc) return lfsai_backward_tc(net, feat, n, h1, h2, h3, dout, st);
   const float* wr = net->wround.as<float>();
   DeviceBuffer d3, d2, d1, part;
   TNLB_TRY_STATUS(d3.alloc(sizeof(float) * n * kLfH));
   TNLB_TRY_STATUS(d2.alloc(sizeof(float) * n * kLfH));
   TNLB_TRY_STATUS(d1.alloc(sizeof(float) * n * kLfH));
   const unsigned g = grid_for(n, 128);
   lf::k_back_layer<kLfH, kLfK><<<g, 128, 0, st>>>(dout, h3, n, wr + kLfW4, d3.as<float>());
   lf::k_back_layer<kLfH, kLfH><<<g, 128, 0, st>>>(d3.as<float>(), h2, n, wr + kLfW3, d2.as<float>());
   lf::k_back_layer<kLfH, kLfH><<<g, 128, 0, st>>>(d2.as<float>(), h1, n, wr + kLfW2, d1.as<float>());
   TNLB_CHECK_LAUNCH();
   const int64_t rpb = 2048;
   const int blocks = (int)((n + rpb - 1) / rpb);
   TNLB_TRY_STATUS(part.alloc(sizeof(float) * (size_t)blocks * (kLfH * kLfH + kLfH)));
   float* gr = net->grad.as<float>();
   TNLB_TRY_STATUS(wgrad_layer<kLfH, kLfK>(dout, h3, n, rpb, blocks, part.as<float>(), gr + kLfW4, gr + kLfB4, st));
   TNLB_TRY_STATUS(wgrad_layer<kLfH, kLfH>(d3.as<float>(), h2, n, rpb, blocks, part.as<float>(), gr + kLfW3, gr + kLfB3, st));
   TNLB_TRY_STATUS(wgrad_layer<kLfH, kLfH>(d2.as<float>(), h1, n, rpb, blocks, part.as<float>(), gr + kLfW2, gr + kLfB2, st));
   TNLB_TRY_STATUS(wgrad_layer<kLfF, kLfH>(d1.as<float>(), feat, n, rpb, blocks, part.as<float>(), gr + kLfW1, gr + kLfB1, st));
   return TNLB_OK;
}

template <typename Real>
tnlb_status gradient_t(tnlb_lfsai* net, const tnlb_segments* seg, const int32_t* cols, const Real* vals,
                       const Real* probes, int32_t P, cudaStream_t st, double* h_loss, int mode)
{
   const int32_t n = seg->n;
   const tnlb_real real = sizeof(Real) == 8 ? TNLB_F64 : TNLB_F32;
   const bool fit = mode == 1;
   LfsaiMatrix M;
   TNLB_TRY_STATUS(build_matrix_ctx<Real>(seg, real, cols, vals, net->level, net->two_factor, st, &M));
   Fsai* F = M.F;
   const int64_t gnnz = F->g->elements;
   lf::k_round_weights<<<(kLfParams + 255) / 256, 256, 0, st>>>(net->theta.as<float>(), net->wround.as<float>());
   DeviceBuffer o, h1, h2, h3, dout, dg, red, cnt, loss;
   TNLB_TRY_STATUS(o.alloc(sizeof(float) * (size_t)n * kLfK));
   TNLB_TRY_STATUS(h1.alloc(sizeof(float) * (size_t)n * kLfH));
   TNLB_TRY_STATUS(h2.alloc(sizeof(float) * (size_t)n * kLfH));
   TNLB_TRY_STATUS(h3.alloc(sizeof(float) * (size_t)n * kLfH));
   TNLB_TRY_STATUS(dout.alloc(sizeof(float) * (size_t)n * kLfK));
   TNLB_TRY_STATUS(dg.alloc(sizeof(double) * gnnz));
   TNLB_TRY_STATUS(red.alloc(sizeof(double) * kRedMaxBlocks * kRedSlots));
   TNLB_TRY_STATUS(cnt.alloc(sizeof(unsigned) * 2));
   TNLB_TRY_STATUS(loss.alloc(sizeof(double)));
   TNLB_CUDA_TRY(cudaMemsetAsync(cnt.ptr, 0, sizeof(unsigned) * 2, st));
   TNLB_CUDA_TRY(cudaMemsetAsync(loss.ptr, 0, sizeof(double), st));
   TNLB_CUDA_TRY(cudaMemsetAsync(dg.ptr, 0, sizeof(double) * gnnz, st));
   RedWork rw{red.as<double>(), cnt.as<unsigned>()};
   TNLB_TRY_STATUS(lfsai_forward(net, M.feat.as<float>(), n, o.as<float>(), h1.as<float>(), h2.as<float>(),
                                 h3.as<float>(), st));
   double kap_n = 0.0;  // Kaporin loss: n, for the host-side value
   if (net->two_factor) {
      TNLB_REQUIRE(mode != 2, TNLB_ERR_INVALID_ARGUMENT,
                   "learned two-factor FSAI: the Kaporin loss is defined for the symmetric form only");
      DeviceBuffer tgl, th;
      TNLB_TRY_STATUS(tgl.alloc(sizeof(Real) * gnnz));
      TNLB_TRY_STATUS(th.alloc(sizeof(Real) * gnnz));
      if (fit) {
         // classical two-factor FSAI: G_L's values, and H's from G_U
         Fsai* C = nullptr;
         TNLB_TRY_STATUS(fsai_create(seg, real, cols, vals, true, st, &C, true));
         TNLB_CUDA_TRY(cudaMemcpyAsync(tgl.ptr, C->g_vals.ptr, sizeof(Real) * gnnz, cudaMemcpyDeviceToDevice, st));
         lf::k_scatter_src<Real><<<grid_for(gnnz, 1024), 256, 0, st>>>(C->gt_src.as<int32_t>(), gnnz,
                                                                       C->gt_vals.as<Real>(), th.as<Real>());
         TNLB_CHECK_LAUNCH();
         TNLB_CUDA_TRY(cudaStreamSynchronize(st));
         fsai_destroy(C);
         lf::k_fit2_do<Real><<<vec_grid(n), kRedThreads, 0, st>>>(o.as<float>(), tgl.as<Real>(), th.as<Real>(),
                                                                  M.s.as<Real>(), F->g->offsets.as<int32_t>(),
                                                                  F->g_cols.as<int32_t>(), n, dout.as<float>(), rw,
                                                                  loss.as<double>());
         TNLB_CHECK_LAUNCH();
         TNLB_CUDA_TRY(cudaStreamSynchronize(st));  // the targets are freed on leaving
      }
      else {
         lf::k_g2_values<Real><<<grid_for(n, 128), 128, 0, st>>>(o.as<float>(), M.s.as<Real>(),
                                                                 F->g->offsets.as<int32_t>(), F->g_cols.as<int32_t>(),
                                                                 n, tgl.as<Real>(), th.as<Real>());
         TNLB_CHECK_LAUNCH();
         TNLB_TRY_STATUS(fsai_set_values2(F, tgl.ptr, th.ptr, st));
         DeviceBuffer t, w, v, u, q, dh;
         for (auto* b : {&t, &w, &v, &u, &q}) TNLB_TRY_STATUS(b->alloc(sizeof(Real) * n));
         TNLB_TRY_STATUS(dh.alloc(sizeof(double) * gnnz));
         TNLB_CUDA_TRY(cudaMemsetAsync(dh.ptr, 0, sizeof(double) * gnnz, st));
         const double c = -2.0 / ((double)n * P);
         for (int32_t p = 0; p < P; p++) {
            const Real* z = probes + (int64_t)p * n;
            // w = A G_U z; v = G_L w; u = z - v; q = A^T G_L^T u
            TNLB_TRY_STATUS(spmv_dispatch(F->gt, real, F->gt_cols.as<int32_t>(), F->gt_vals.ptr, z, t.ptr, 1.0, 0.0, st));
            TNLB_TRY_STATUS(spmv_dispatch(seg, real, cols, vals, t.ptr, w.ptr, 1.0, 0.0, st));
            TNLB_TRY_STATUS(spmv_dispatch(F->g, real, F->g_cols.as<int32_t>(), F->g_vals.ptr, w.ptr, v.ptr, 1.0, 0.0, st));
            lf::k_resid<Real><<<vec_grid(n), kRedThreads, 0, st>>>(n, z, v.as<Real>(), u.as<Real>(), rw,
                                                                   loss.as<double>());
            TNLB_CHECK_LAUNCH();
            TNLB_TRY_STATUS(tnlb_spmv_transposed(F->g, real, F->g_cols.as<int32_t>(), F->g_vals.ptr, n, u.ptr, t.ptr,
                                                 1.0, 0.0, 0, 0, (tnlb_stream)st));
            TNLB_TRY_STATUS(tnlb_spmv_transposed(seg, real, cols, vals, n, t.ptr, q.ptr, 1.0, 0.0, 0, 0,
                                                 (tnlb_stream)st));
            lf::k_dg2<Real><<<grid_for(n, 256), 256, 0, st>>>(F->g->offsets.as<int32_t>(), F->g_cols.as<int32_t>(), n,
                                                              u.as<Real>(), w.as<Real>(), z, q.as<Real>(), c,
                                                              dg.as<double>(), dh.as<double>());
            TNLB_CHECK_LAUNCH();
         }
         lf::k_do2<Real><<<grid_for(n, 128), 128, 0, st>>>(dg.as<double>(), dh.as<double>(), o.as<float>(),
                                                           M.s.as<Real>(), F->g->offsets.as<int32_t>(),
                                                           F->g_cols.as<int32_t>(), n, dout.as<float>());
         TNLB_CHECK_LAUNCH();
         TNLB_CUDA_TRY(cudaStreamSynchronize(st));
      }
   }
   else if (fit) {
      // supervised warm start on the classical FSAI values of the level-0
      // pattern (zero on fill entries)
      DeviceBuffer tg;
      TNLB_TRY_STATUS(tg.alloc(sizeof(Real) * gnnz));
      Fsai* C = nullptr;
      TNLB_TRY_STATUS(fsai_create(seg, real, cols, vals, true, st, &C));
      lf::k_map_target<Real><<<grid_for(n, 128), 128, 0, st>>>(
         F->g->offsets.as<int32_t>(), F->g_cols.as<int32_t>(), C->g->offsets.as<int32_t>(), C->g_cols.as<int32_t>(),
         C->g_vals.as<Real>(), n, tg.as<Real>());
      TNLB_CHECK_LAUNCH();
      TNLB_CUDA_TRY(cudaStreamSynchronize(st));
      fsai_destroy(C);
      lf::k_fit_do<Real><<<vec_grid(n), kRedThreads, 0, st>>>(o.as<float>(), tg.as<Real>(), M.s.as<Real>(),
                                                              F->g->offsets.as<int32_t>(), F->g_cols.as<int32_t>(), n,
                                                              dout.as<float>(), rw, loss.as<double>());
      TNLB_CHECK_LAUNCH();
   }
   else if (mode == 2) {
      // Kaporin loss: T and sum log G'_ii, then dK/do
      DeviceBuffer tot;
      TNLB_TRY_STATUS(tot.alloc(sizeof(double) * 2));
      lf::k_kap_sums<Real><<<vec_grid(n), kRedThreads, 0, st>>>(
         F->a_rp.as<int32_t>(), F->a_cols.as<int32_t>(), F->a_vals.as<Real>(), F->g->offsets.as<int32_t>(),
         F->g_cols.as<int32_t>(), n, o.as<float>(), rw, tot.as<double>());
      TNLB_CHECK_LAUNCH();
      lf::k_kap_do<Real><<<grid_for(n, 128), 128, 0, st>>>(F->a_rp.as<int32_t>(), F->a_cols.as<int32_t>(),
                                                           F->a_vals.as<Real>(), F->g->offsets.as<int32_t>(),
                                                           F->g_cols.as<int32_t>(), n, o.as<float>(),
                                                           tot.as<double>(), dout.as<float>());
      TNLB_CHECK_LAUNCH();
      double ht[2] = {0, 0};
      TNLB_CUDA_TRY(cudaMemcpyAsync(ht, tot.ptr, sizeof(ht), cudaMemcpyDeviceToHost, st));
      TNLB_CUDA_TRY(cudaStreamSynchronize(st));
      TNLB_REQUIRE(ht[0] > 0, TNLB_ERR_BREAKDOWN, "learned FSAI: trace(G A G^T) is not positive");
      kap_n = std::log(ht[0] / n) - 2.0 * ht[1] / n;
   }
   else {
      lf::k_g_values<Real><<<grid_for(n, 128), 128, 0, st>>>(o.as<float>(), M.s.as<Real>(), F->g->offsets.as<int32_t>(),
                                                             F->g_cols.as<int32_t>(), n, F->g_vals.as<Real>());
      TNLB_CHECK_LAUNCH();
      TNLB_TRY_STATUS(fsai_set_values(F, F->g_vals.ptr, st));
      DeviceBuffer t, w, v, u, q;
      for (auto* b : {&t, &w, &v, &u, &q}) TNLB_TRY_STATUS(b->alloc(sizeof(Real) * n));
      const double c = -2.0 / ((double)n * P);
      for (int32_t p = 0; p < P; p++) {
         const Real* z = probes + (int64_t)p * n;
         // w = A G^T z; v = G w; u = z - v; q = A G^T u
         TNLB_TRY_STATUS(spmv_dispatch(F->gt, real, F->gt_cols.as<int32_t>(), F->gt_vals.ptr, z, t.ptr, 1.0, 0.0, st));
         TNLB_TRY_STATUS(spmv_dispatch(seg, real, cols, vals, t.ptr, w.ptr, 1.0, 0.0, st));
         TNLB_TRY_STATUS(spmv_dispatch(F->g, real, F->g_cols.as<int32_t>(), F->g_vals.ptr, w.ptr, v.ptr, 1.0, 0.0, st));
         lf::k_resid<Real><<<vec_grid(n), kRedThreads, 0, st>>>(n, z, v.as<Real>(), u.as<Real>(), rw, loss.as<double>());
         TNLB_TRY_STATUS(spmv_dispatch(F->gt, real, F->gt_cols.as<int32_t>(), F->gt_vals.ptr, u.ptr, t.ptr, 1.0, 0.0, st));
         TNLB_TRY_STATUS(spmv_dispatch(seg, real, cols, vals, t.ptr, q.ptr, 1.0, 0.0, st));
         lf::k_dg<Real><<<grid_for(n, 256), 256, 0, st>>>(F->g->offsets.as<int32_t>(), F->g_cols.as<int32_t>(), n,
                                                          u.as<Real>(), w.as<Real>(), z, q.as<Real>(), c,
                                                          dg.as<double>());
         TNLB_CHECK_LAUNCH();
      }
      lf::k_do<Real><<<grid_for(n, 128), 128, 0, st>>>(dg.as<double>(), o.as<float>(), M.s.as<Real>(),
                                                       F->g->offsets.as<int32_t>(), F->g_cols.as<int32_t>(), n,
                                                       dout.as<float>());
      TNLB_CHECK_LAUNCH();
   }
   TNLB_TRY_STATUS(lfsai_backward(net, M.feat.as<float>(), n, h1.as<float>(), h2.as<float>(), h3.as<float>(),
                                  dout.as<float>(), st));
   double hl = 0;
   TNLB_CUDA_TRY(cudaMemcpyAsync(&hl, loss.ptr, sizeof(double), cudaMemcpyDeviceToHost, st));
   TNLB_CUDA_TRY(cudaStreamSynchronize(st));
   *h_loss = mode == 2 ? kap_n : fit ? hl : hl / ((double)n * P);
   return TNLB_OK;
}

template <typename Real>
tnlb_status precond_t(const tnlb_lfsai* net, const tnlb_segments* seg, const int32_t* cols, const Real* vals,
                      cudaStream_t st, tnlb_precond** out)
{
   const tnlb_real real = sizeof(Real) == 8 ? TNLB_F64 : TNLB_F32;
   auto* M = new LfsaiMatrix();
   tnlb_status s = build_matrix_ctx<Real>(seg, real, cols, vals, net->level, net->two_factor, st, M);
   if (s != TNLB_OK) {
      delete M;
      return s;
   }
   const int32_t n = seg->n;
   DeviceBuffer o, h1, h2, h3;
   lf::k_round_weights<<<(kLfParams + 255) / 256, 256, 0, st>>>(net->theta.as<float>(), net->wround.as<float>());
   TNLB_TRY_STATUS(o.alloc(sizeof(float) * (size_t)n * kLfK));
   TNLB_TRY_STATUS(h1.alloc(sizeof(float) * (size_t)n * kLfH));
   TNLB_TRY_STATUS(h2.alloc(sizeof(float) * (size_t)n * kLfH));
   TNLB_TRY_STATUS(h3.alloc(sizeof(float) * (size_t)n * kLfH));
   TNLB_TRY_STATUS(lfsai_forward(net, M->feat.as<float>(), n, o.as<float>(), h1.as<float>(), h2.as<float>(),
                                 h3.as<float>(), st));
   if (net->two_factor) {
      DeviceBuffer h;
      TNLB_TRY_STATUS(h.alloc(sizeof(Real) * M->F->g->elements));
      lf::k_g2_values<Real><<<grid_for(n, 128), 128, 0, st>>>(o.as<float>(), M->s.as<Real>(),
                                                              M->F->g->offsets.as<int32_t>(),
                                                              M->F->g_cols.as<int32_t>(), n, M->F->g_vals.as<Real>(),
                                                              h.as<Real>());
      TNLB_CHECK_LAUNCH();
      TNLB_TRY_STATUS(fsai_set_values2(M->F, M->F->g_vals.ptr, h.ptr, st));
      TNLB_CUDA_TRY(cudaStreamSynchronize(st));
   }
   else {
      lf::k_g_values<Real><<<grid_for(n, 128), 128, 0, st>>>(o.as<float>(), M->s.as<Real>(),
                                                             M->F->g->offsets.as<int32_t>(),
                                                             M->F->g_cols.as<int32_t>(), n, M->F->g_vals.as<Real>());
      TNLB_CHECK_LAUNCH();
      TNLB_TRY_STATUS(fsai_set_values(M->F, M->F->g_vals.ptr, st));
   }
   TNLB_CUDA_TRY(cudaStreamSynchronize(st));
   auto* P = new tnlb_precond();
   P->kind = TNLB_PRECOND_FSAI;
   P->real = real;
   P->n = n;
   P->fsai = M->F;
   M->F = nullptr;
   delete M;
   *out = P;
   return TNLB_OK;
}

}  // namespace

tnlb_status lfsai_gradient(tnlb_lfsai* net, const tnlb_segments* seg, tnlb_real real, const int32_t* cols,
                           const void* vals, const void* probes, int32_t P, int mode, cudaStream_t st, double* loss)
{
   TNLB_REQUIRE(mode >= 0 && mode <= 2, TNLB_ERR_INVALID_ARGUMENT, "learned FSAI: unknown training mode");
   TNLB_REQUIRE(mode != 0 || (probes && P > 0), TNLB_ERR_INVALID_ARGUMENT, "learned FSAI: the probe loss needs probes");
   if (real == TNLB_F64)
      return gradient_t<double>(net, seg, cols, (const double*)vals, (const double*)probes, P, st, loss, mode);
   return gradient_t<float>(net, seg, cols, (const float*)vals, (const float*)probes, P, st, loss, mode);
}

tnlb_status lfsai_adam(tnlb_lfsai* net, double lr, cudaStream_t st)
{
   net->step++;
   const float b1 = 0.9f, b2 = 0.999f;
   const float c1 = 1.f - std::pow(b1, (float)net->step), c2 = 1.f - std::pow(b2, (float)net->step);
   lf::k_adam<<<(kLfParams + 255) / 256, 256, 0, st>>>(net->theta.as<float>(), net->grad.as<float>(),
                                                       net->m.as<float>(), net->v.as<float>(), kLfParams, (float)lr, b1,
                                                       b2, 1e-8f, c1, c2);
   TNLB_CHECK_LAUNCH();
   return TNLB_OK;
}

tnlb_status lfsai_init(tnlb_lfsai* net, uint64_t seed, cudaStream_t st)
{
   TNLB_TRY_STATUS(net->theta.alloc(sizeof(float) * kLfParams));
   TNLB_TRY_STATUS(net->wround.alloc(sizeof(float) * kLfParams));
   TNLB_TRY_STATUS(net->grad.alloc(sizeof(float) * kLfParams));
   TNLB_TRY_STATUS(net->m.alloc(sizeof(float) * kLfParams));
   TNLB_TRY_STATUS(net->v.alloc(sizeof(float) * kLfParams));
   TNLB_CUDA_TRY(cudaMemsetAsync(net->m.ptr, 0, sizeof(float) * kLfParams, st));
   TNLB_CUDA_TRY(cudaMemsetAsync(net->v.ptr, 0, sizeof(float) * kLfParams, st));
   TNLB_CUDA_TRY(cudaMemsetAsync(net->grad.ptr, 0, sizeof(float) * kLfParams, st));
   lf::k_init_params<<<(kLfParams + 255) / 256, 256, 0, st>>>(seed, net->theta.as<float>());
   TNLB_CHECK_LAUNCH();
   lf::k_round_weights<<<(kLfParams + 255) / 256, 256, 0, st>>>(net->theta.as<float>(), net->wround.as<float>());
   TNLB_CHECK_LAUNCH();
   TNLB_CUDA_TRY(cudaStreamSynchronize(st));
   return TNLB_OK;
}

tnlb_status lfsai_precond(const tnlb_lfsai* net, const tnlb_segments* seg, tnlb_real real, const int32_t* cols,
                          const void* vals, cudaStream_t st, tnlb_precond** out)
{
   if (real == TNLB_F64) return precond_t<double>(net, seg, cols, (const double*)vals, st, out);
   return precond_t<float>(net, seg, cols, (const float*)vals, st, out);
}

// Features and network outputs for inspection (tests).
tnlb_status lfsai_eval(const tnlb_lfsai* net, const tnlb_segments* seg, tnlb_real real, const int32_t* cols,
                       const void* vals, cudaStream_t st, float* h_feat, float* h_out)
{
   LfsaiMatrix M;
   if (real == TNLB_F64)
      TNLB_TRY_STATUS(
         build_matrix_ctx<double>(seg, real, cols, (const double*)vals, net->level, net->two_factor, st, &M));
   else
      TNLB_TRY_STATUS(
         build_matrix_ctx<float>(seg, real, cols, (const float*)vals, net->level, net->two_factor, st, &M));
   const int32_t n = seg->n;
   DeviceBuffer o, h1, h2, h3;
   lf::k_round_weights<<<(kLfParams + 255) / 256, 256, 0, st>>>(net->theta.as<float>(), net->wround.as<float>());
   TNLB_TRY_STATUS(o.alloc(sizeof(float) * (size_t)n * kLfK));
   TNLB_TRY_STATUS(h1.alloc(sizeof(float) * (size_t)n * kLfH));
   TNLB_TRY_STATUS(h2.alloc(sizeof(float) * (size_t)n * kLfH));
   TNLB_TRY_STATUS(h3.alloc(sizeof(float) * (size_t)n * kLfH));
   TNLB_TRY_STATUS(lfsai_forward(net, M.feat.as<float>(), n, o.as<float>(), h1.as<float>(), h2.as<float>(),
                                 h3.as<float>(), st));
   if (h_feat)
      TNLB_CUDA_TRY(cudaMemcpyAsync(h_feat, M.feat.ptr, sizeof(float) * (size_t)n * kLfF, cudaMemcpyDeviceToHost, st));
   if (h_out) TNLB_CUDA_TRY(cudaMemcpyAsync(h_out, o.ptr, sizeof(float) * (size_t)n * kLfK, cudaMemcpyDeviceToHost, st));
   TNLB_CUDA_TRY(cudaStreamSynchronize(st));
   return TNLB_OK;
}

}  // namespace tnlb
