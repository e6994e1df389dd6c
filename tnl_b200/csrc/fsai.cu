// fsai.cu -- factorised sparse approximate inverse preconditioner M^-1 = G^T G.
//
// No counterpart in the reference (it has Diagonal, ILU0 and ILUT only).
// G is lower triangular on a given sparsity pattern (here: the lower
// triangle of A including the diagonal).  The classical values are the
// Kolotilina-Yeremin FSAI: for row i with pattern J (sorted, i last) solve
// the small SPD system A[J,J] g = e_last and scale G_i = g / sqrt(g_last),
// so that diag(G A G^T) = 1 (L. Yu. Kolotilina, A. Yu. Yeremin, "Factorized
// sparse approximate inverse preconditionings I", SIAM J. Matrix Anal. Appl.
// 14 (1993)).  The learned preconditioner (lfsai.cu) writes G's values on the
// same pattern from a per-row network instead.
//
// Applying M^-1 costs two SpMVs through the library's CSR tile kernel:
// t = G r, z = G^T t, with G^T stored explicitly (transposed once).
#include <vector>

#include "fsai.cuh"
#include "internal.cuh"
#include "segview.cuh"

namespace tnlb {

namespace {

__global__ void k_count_lower(const int32_t* __restrict__ rp, const int32_t* __restrict__ cols, int32_t n,
                              int32_t* __restrict__ cnt)
{
   const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (i >= n) return;
   int32_t c = 0;
   for (int32_t q = rp[i]; q < rp[i + 1]; q++) c += (cols[q] >= 0 && cols[q] <= i);
   cnt[i] = c;
}

__global__ void k_copy_lower(const int32_t* __restrict__ rp, const int32_t* __restrict__ cols, int32_t n,
                             const int32_t* __restrict__ grp, int32_t* __restrict__ gcols)
{
   const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (i >= n) return;
   int32_t o = grp[i];
   for (int32_t q = rp[i]; q < rp[i + 1]; q++)
      if (cols[q] >= 0 && cols[q] <= i) gcols[o++] = cols[q];
}

// Level-1 lower pattern of row i: the columns j <= i reached from i in at
// most two steps through A's pattern (i itself, its neighbours, theirs),
// i.e. the lower triangle of the pattern of A^2, sorted.  Count pass
// (gcols == nullptr: cnt[i] = size) and fill pass.  More than kLevel1Max
// candidates in a row sets *err = 1.
constexpr int kLevel1Max = 64;

__global__ void k_level1_lower(const int32_t* __restrict__ rp, const int32_t* __restrict__ cols, int32_t n,
                               const int32_t* __restrict__ grp, int32_t* __restrict__ gcols, int32_t* __restrict__ cnt,
                               int32_t* __restrict__ err)
{
   const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (i >= n) return;
   int32_t cand[kLevel1Max];
   int k = 0;
   bool over = false;
   auto push = [&](int32_t j) {
      for (int q = 0; q < k; q++)
         if (cand[q] == j) return;
      if (k == kLevel1Max) {
         over = true;
         return;
      }
      // insertion keeps cand sorted
      int q = k++;
      while (q > 0 && cand[q - 1] > j) {
         cand[q] = cand[q - 1];
         q--;
      }
      cand[q] = j;
   };
   push((int32_t)i);
   for (int32_t a = rp[i]; a < rp[i + 1]; a++) {
      const int32_t l = cols[a];
      if (l < 0) continue;
      if (l <= i) push(l);
      for (int32_t b = rp[l]; b < rp[l + 1]; b++) {
         const int32_t j = cols[b];
         if (j >= 0 && j <= i) push(j);
      }
   }
   if (over) {
      atomicExch(err, 1);
      k = 0;
   }
   if (!gcols)
      cnt[i] = k;
   else
      for (int q = 0; q < k; q++) gcols[grp[i] + q] = cand[q];
}

// a(r, c) from a CSR row with ascending columns (0 if absent).
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

constexpr int kFsaiMaxRow = 32;

// Classical FSAI row: Cholesky of A[J,J] (k <= 32) in FP64, solve for e_last.
template <typename Real>
__global__ void k_fsai_rows(const int32_t* __restrict__ rp, const int32_t* __restrict__ cols,
                            const Real* __restrict__ vals, int32_t n, const int32_t* __restrict__ grp,
                            const int32_t* __restrict__ gcols, Real* __restrict__ gvals, int32_t* __restrict__ err)
{
   const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (i >= n) return;
   const int32_t b = grp[i], k = grp[i + 1] - b;
   if (k <= 0 || k > kFsaiMaxRow) {
      atomicExch(err, 1);
      return;
   }
   double L[kFsaiMaxRow * (kFsaiMaxRow + 1) / 2];
   // packed lower Cholesky factor of A[J,J]
   for (int r = 0; r < k; r++) {
      const int32_t jr = gcols[b + r];
      for (int c = 0; c <= r; c++) {
         const int32_t jc = gcols[b + c];
         double s = (double)lookup(rp, cols, vals, jr, jc);
         for (int q = 0; q < c; q++) s -= L[r * (r + 1) / 2 + q] * L[c * (c + 1) / 2 + q];
         if (r == c) {
            if (!(s > 0)) {
               atomicExch(err, 2);
               s = 1.0;
            }
            L[r * (r + 1) / 2 + r] = sqrt(s);
         }
         else
            L[r * (r + 1) / 2 + c] = s / L[c * (c + 1) / 2 + c];
      }
   }
   // A[J,J] g = e_last: forward (only the last entry of e is nonzero), back
   double y[kFsaiMaxRow];
   for (int r = 0; r < k; r++) {
      double s = (r == k - 1) ? 1.0 : 0.0;
      for (int q = 0; q < r; q++) s -= L[r * (r + 1) / 2 + q] * y[q];
      y[r] = s / L[r * (r + 1) / 2 + r];
   }
   for (int r = k - 1; r >= 0; r--) {
      double s = y[r];
      for (int q = r + 1; q < k; q++) s -= L[q * (q + 1) / 2 + r] * y[q];
      y[r] = s / L[r * (r + 1) / 2 + r];
   }
   const double scale = 1.0 / sqrt(y[k - 1]);
   for (int r = 0; r < k; r++) gvals[b + r] = (Real)(y[r] * scale);
}

// Two-factor FSAI row for a nonsymmetric A: with B = A[J,J] (J the lower
// pattern of row i, i last), g_L = B^-T e_last is row i of G_L and
// g_U = B^-1 e_last is column i of G_U; both are scaled by 1/sqrt(g_U,last)
// (= 1/sqrt((B^-1)_last,last)) so that diag(G_L A G_U) = 1 on the pattern.
// Row i of H = G_U^T (lower, same pattern) is written to hvals.  LU without
// pivoting (the local blocks of the diagonally dominant operators are).
template <typename Real>
__global__ void k_fsai2_rows(const int32_t* __restrict__ rp, const int32_t* __restrict__ cols,
                             const Real* __restrict__ vals, int32_t n, const int32_t* __restrict__ grp,
                             const int32_t* __restrict__ gcols, Real* __restrict__ gvals, Real* __restrict__ hvals,
                             int32_t* __restrict__ err)
{
   constexpr int KM = 12;
   const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (i >= n) return;
   const int32_t b = grp[i], k = grp[i + 1] - b;
   if (k <= 0 || k > KM) {
      atomicExch(err, 1);
      return;
   }
   double B[KM][KM];
   for (int r = 0; r < k; r++)
      for (int c = 0; c < k; c++) B[r][c] = (double)lookup(rp, cols, vals, gcols[b + r], gcols[b + c]);
   // in-place LU (Doolittle), B = L U
   for (int p = 0; p < k; p++) {
      if (B[p][p] == 0.0) {
         atomicExch(err, 2);
         return;
      }
      for (int r = p + 1; r < k; r++) {
         const double l = B[r][p] / B[p][p];
         B[r][p] = l;
         for (int c = p + 1; c < k; c++) B[r][c] -= l * B[p][c];
      }
   }
   // u = B^-1 e: L y = e, U u = y
   double u[KM], w[KM];
   for (int r = 0; r < k; r++) {
      double sacc = (r == k - 1) ? 1.0 : 0.0;
      for (int q = 0; q < r; q++) sacc -= B[r][q] * u[q];
      u[r] = sacc;
   }
   for (int r = k - 1; r >= 0; r--) {
      double sacc = u[r];
      for (int q = r + 1; q < k; q++) sacc -= B[r][q] * u[q];
      u[r] = sacc / B[r][r];
   }
   // w = B^-T e: U^T z = e, L^T w = z
   for (int r = 0; r < k; r++) {
      double sacc = (r == k - 1) ? 1.0 : 0.0;
      for (int q = 0; q < r; q++) sacc -= B[q][r] * w[q];
      w[r] = sacc / B[r][r];
   }
   for (int r = k - 1; r >= 0; r--) {
      double sacc = w[r];
      for (int q = r + 1; q < k; q++) sacc -= B[q][r] * w[q];
      w[r] = sacc;
   }
   if (!(u[k - 1] > 0)) {
      atomicExch(err, 2);
      return;
   }
   const double scale = 1.0 / sqrt(u[k - 1]);
   for (int r = 0; r < k; r++) {
      gvals[b + r] = (Real)(w[r] * scale);
      hvals[b + r] = (Real)(u[r] * scale);
   }
}

// Transpose of a CSR matrix with ascending columns: counting by column,
// then each row of the transpose is filled in ascending source-row order
// (one thread per transpose row scanning a precomputed list is avoided by
// placing entries with a per-column cursor and sorting each short row).
__global__ void k_col_count(const int32_t* __restrict__ cols, int64_t nnz, int32_t* __restrict__ cnt)
{
   for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < nnz; q += (int64_t)gridDim.x * blockDim.x)
      atomicAdd(cnt + cols[q], 1);
}

__global__ void k_scatter_t(const int32_t* __restrict__ rp, const int32_t* __restrict__ cols, int32_t n,
                            const int32_t* __restrict__ trp, int32_t* __restrict__ cursor, int32_t* __restrict__ tcols,
                            int32_t* __restrict__ tsrc)
{
   const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (i >= n) return;
   for (int32_t q = rp[i]; q < rp[i + 1]; q++) {
      const int32_t c = cols[q];
      const int32_t pos = trp[c] + atomicAdd(cursor + c, 1);
      tcols[pos] = (int32_t)i;
      tsrc[pos] = q;
   }
}

// Sort each transpose row by column (source row): insertion sort, rows are short.
__global__ void k_sort_rows(const int32_t* __restrict__ trp, int32_t n, int32_t* __restrict__ tcols,
                            int32_t* __restrict__ tsrc)
{
   const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (r >= n) return;
   const int32_t b = trp[r], e = trp[r + 1];
   for (int32_t a = b + 1; a < e; a++) {
      const int32_t kc = tcols[a], ks = tsrc[a];
      int32_t j = a - 1;
      while (j >= b && tcols[j] > kc) {
         tcols[j + 1] = tcols[j];
         tsrc[j + 1] = tsrc[j];
         j--;
      }
      tcols[j + 1] = kc;
      tsrc[j + 1] = ks;
   }
}

template <typename Real>
__global__ void k_gather_vals(const int32_t* __restrict__ src, int64_t nnz, const Real* __restrict__ from,
                              Real* __restrict__ to)
{
   for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < nnz; q += (int64_t)gridDim.x * blockDim.x)
      to[q] = from[src[q]];
}

__global__ void k_lengths(const int32_t* __restrict__ rp, int32_t n, int32_t* __restrict__ len)
{
   const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (i < n) len[i] = rp[i + 1] - rp[i];
}

// CSR segments object over an existing row-pointer array.
tnlb_status make_csr_segments(const int32_t* d_rowptr, int32_t n, cudaStream_t st, tnlb_segments** out)
{
   DeviceBuffer len;
   TNLB_TRY_STATUS(len.alloc(sizeof(int32_t) * (n > 0 ? n : 1)));
   if (n > 0) {
      k_lengths<<<grid_for(n, 256), 256, 0, st>>>(d_rowptr, n, len.as<int32_t>());
      TNLB_CHECK_LAUNCH();
   }
   auto* seg = new tnlb_segments();
   seg->format = TNLB_CSR;
   seg->organization = TNLB_COLUMN_MAJOR;
   seg->n = n;
   TNLB_CUDA_TRY(cudaGetDevice(&seg->device));
   tnlb_status s = build_segments(seg, len.as<int32_t>(), st);
   if (s != TNLB_OK) {
      delete seg;
      return s;
   }
   *out = seg;
   return TNLB_OK;
}

}  // namespace

// Gathers A into CSR (ascending columns), builds G's pattern (level 0: the
// lower triangle of A with the diagonal; level 1: the lower triangle of the
// pattern of A^2, one level of fill) and, when `classical`, the
// Kolotilina-Yeremin values; then G^T.  The values of a learned G are
// written later through fsai_set_values.
tnlb_status fsai_create(const tnlb_segments* seg, tnlb_real real, const int32_t* cols, const void* vals, bool classical,
                        cudaStream_t st, Fsai** out, bool two_factor, int level)
{
   TNLB_REQUIRE(level == 0 || level == 1, TNLB_ERR_INVALID_ARGUMENT, "FSAI: the pattern level must be 0 or 1");
   TNLB_REQUIRE(level == 0 || !two_factor, TNLB_ERR_INVALID_ARGUMENT,
                "FSAI: the two-factor form uses the level-0 pattern");
   const int32_t n = seg->n;
   TNLB_REQUIRE(n > 0, TNLB_ERR_INVALID_ARGUMENT, "FSAI: the matrix is empty");
   auto* F = new Fsai();
   F->n = n;
   F->real = real;
   F->two_factor = two_factor;
   const size_t rs = real == TNLB_F64 ? 8 : 4;
   // CSR copy of A
   {
      TNLB_TRY_STATUS(gather_csr(view_of(seg), real, cols, vals, F->a_rp, F->a_cols, F->a_vals, st));
   }
   // pattern of G
   DeviceBuffer cnt, grp;
   TNLB_TRY_STATUS(cnt.alloc(sizeof(int32_t) * n));
   TNLB_TRY_STATUS(grp.alloc(sizeof(int32_t) * ((size_t)n + 1)));
   DeviceBuffer perr;
   TNLB_TRY_STATUS(perr.alloc(sizeof(int32_t)));
   TNLB_CUDA_TRY(cudaMemsetAsync(perr.ptr, 0, sizeof(int32_t), st));
   if (level == 0)
      k_count_lower<<<grid_for(n, 256), 256, 0, st>>>(F->a_rp.as<int32_t>(), F->a_cols.as<int32_t>(), n,
                                                      cnt.as<int32_t>());
   else
      k_level1_lower<<<grid_for(n, 128), 128, 0, st>>>(F->a_rp.as<int32_t>(), F->a_cols.as<int32_t>(), n, nullptr,
                                                       nullptr, cnt.as<int32_t>(), perr.as<int32_t>());
   TNLB_CHECK_LAUNCH();
   int64_t gnnz = 0;
   TNLB_TRY_STATUS(exclusive_scan_i32(cnt.as<int32_t>(), grp.as<int32_t>(), n, &gnnz, st, true));
   {
      int32_t h = 0;
      TNLB_CUDA_TRY(cudaMemcpyAsync(&h, perr.ptr, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
      TNLB_CUDA_TRY(cudaStreamSynchronize(st));
      TNLB_REQUIRE(h == 0, TNLB_ERR_INVALID_ARGUMENT,
                   "FSAI: a row of the level-1 pattern reaches more than 64 candidate columns");
   }
   TNLB_TRY_STATUS(F->g_cols.alloc(sizeof(int32_t) * gnnz));
   TNLB_TRY_STATUS(F->g_vals.alloc(rs * gnnz));
   if (level == 0)
      k_copy_lower<<<grid_for(n, 256), 256, 0, st>>>(F->a_rp.as<int32_t>(), F->a_cols.as<int32_t>(), n,
                                                     grp.as<int32_t>(), F->g_cols.as<int32_t>());
   else
      k_level1_lower<<<grid_for(n, 128), 128, 0, st>>>(F->a_rp.as<int32_t>(), F->a_cols.as<int32_t>(), n,
                                                       grp.as<int32_t>(), F->g_cols.as<int32_t>(), nullptr,
                                                       perr.as<int32_t>());
   TNLB_CHECK_LAUNCH();
   TNLB_TRY_STATUS(make_csr_segments(grp.as<int32_t>(), n, st, &F->g));
   DeviceBuffer hvals;  // two-factor: row i of H = G_U^T on G's pattern
   if (two_factor) TNLB_TRY_STATUS(hvals.alloc(rs * gnnz));
   if (classical) {
      DeviceBuffer err;
      TNLB_TRY_STATUS(err.alloc(sizeof(int32_t)));
      TNLB_CUDA_TRY(cudaMemsetAsync(err.ptr, 0, sizeof(int32_t), st));
      if (two_factor) {
         if (real == TNLB_F64)
            k_fsai2_rows<double><<<grid_for(n, 128), 128, 0, st>>>(F->a_rp.as<int32_t>(), F->a_cols.as<int32_t>(),
                                                                  F->a_vals.as<double>(), n, grp.as<int32_t>(),
                                                                  F->g_cols.as<int32_t>(), F->g_vals.as<double>(),
                                                                  hvals.as<double>(), err.as<int32_t>());
         else
            k_fsai2_rows<float><<<grid_for(n, 128), 128, 0, st>>>(F->a_rp.as<int32_t>(), F->a_cols.as<int32_t>(),
                                                                 F->a_vals.as<float>(), n, grp.as<int32_t>(),
                                                                 F->g_cols.as<int32_t>(), F->g_vals.as<float>(),
                                                                 hvals.as<float>(), err.as<int32_t>());
      }
      else if (real == TNLB_F64)
         k_fsai_rows<double><<<grid_for(n, 128), 128, 0, st>>>(F->a_rp.as<int32_t>(), F->a_cols.as<int32_t>(),
                                                              F->a_vals.as<double>(), n, grp.as<int32_t>(),
                                                              F->g_cols.as<int32_t>(), F->g_vals.as<double>(),
                                                              err.as<int32_t>());
      else
         k_fsai_rows<float><<<grid_for(n, 128), 128, 0, st>>>(F->a_rp.as<int32_t>(), F->a_cols.as<int32_t>(),
                                                             F->a_vals.as<float>(), n, grp.as<int32_t>(),
                                                             F->g_cols.as<int32_t>(), F->g_vals.as<float>(),
                                                             err.as<int32_t>());
      TNLB_CHECK_LAUNCH();
      int32_t h = 0;
      TNLB_CUDA_TRY(cudaMemcpyAsync(&h, err.ptr, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
      TNLB_CUDA_TRY(cudaStreamSynchronize(st));
      TNLB_REQUIRE(h != 1, TNLB_ERR_INVALID_ARGUMENT, "FSAI: a row of the pattern holds too many entries");
      TNLB_REQUIRE(h != 2, TNLB_ERR_INVALID_ARGUMENT, "FSAI: a local block A[J,J] is singular or not positive definite");
   }
   // transpose pattern
   DeviceBuffer tcnt, cursor;
   TNLB_TRY_STATUS(tcnt.alloc(sizeof(int32_t) * n));
   TNLB_TRY_STATUS(cursor.alloc(sizeof(int32_t) * n));
   TNLB_CUDA_TRY(cudaMemsetAsync(tcnt.ptr, 0, sizeof(int32_t) * n, st));
   TNLB_CUDA_TRY(cudaMemsetAsync(cursor.ptr, 0, sizeof(int32_t) * n, st));
   k_col_count<<<grid_for(gnnz, 256), 256, 0, st>>>(F->g_cols.as<int32_t>(), gnnz, tcnt.as<int32_t>());
   TNLB_CHECK_LAUNCH();
   DeviceBuffer trp;
   TNLB_TRY_STATUS(trp.alloc(sizeof(int32_t) * ((size_t)n + 1)));
   TNLB_TRY_STATUS(exclusive_scan_i32(tcnt.as<int32_t>(), trp.as<int32_t>(), n, nullptr, st, true));
   TNLB_TRY_STATUS(F->gt_cols.alloc(sizeof(int32_t) * gnnz));
   TNLB_TRY_STATUS(F->gt_src.alloc(sizeof(int32_t) * gnnz));
   TNLB_TRY_STATUS(F->gt_vals.alloc(rs * gnnz));
   k_scatter_t<<<grid_for(n, 256), 256, 0, st>>>(grp.as<int32_t>(), F->g_cols.as<int32_t>(), n, trp.as<int32_t>(),
                                                 cursor.as<int32_t>(), F->gt_cols.as<int32_t>(), F->gt_src.as<int32_t>());
   TNLB_CHECK_LAUNCH();
   k_sort_rows<<<grid_for(n, 256), 256, 0, st>>>(trp.as<int32_t>(), n, F->gt_cols.as<int32_t>(),
                                                 F->gt_src.as<int32_t>());
   TNLB_CHECK_LAUNCH();
   TNLB_TRY_STATUS(make_csr_segments(trp.as<int32_t>(), n, st, &F->gt));
   TNLB_TRY_STATUS(F->tmp.alloc(rs * n));
   if (classical) {
      // G^T from G (symmetric case), or G_U = H^T (two factors)
      const void* src = two_factor ? hvals.ptr : F->g_vals.ptr;
      if (real == TNLB_F64)
         k_gather_vals<double><<<grid_for(gnnz, 1024), 256, 0, st>>>(F->gt_src.as<int32_t>(), gnnz,
                                                                     (const double*)src, F->gt_vals.as<double>());
      else
         k_gather_vals<float><<<grid_for(gnnz, 1024), 256, 0, st>>>(F->gt_src.as<int32_t>(), gnnz,
                                                                    (const float*)src, F->gt_vals.as<float>());
      TNLB_CHECK_LAUNCH();
   }
   TNLB_CUDA_TRY(cudaStreamSynchronize(st));
   *out = F;
   return TNLB_OK;
}

// New values of G (device array over G's pattern, same real type); G^T follows.
tnlb_status fsai_set_values(Fsai* F, const void* gvals, cudaStream_t st)
{
   const int64_t gnnz = F->g->elements;
   const size_t rs = F->real == TNLB_F64 ? 8 : 4;
   TNLB_CUDA_TRY(cudaMemcpyAsync(F->g_vals.ptr, gvals, rs * gnnz, cudaMemcpyDeviceToDevice, st));
   if (F->real == TNLB_F64)
      k_gather_vals<double><<<grid_for(gnnz, 1024), 256, 0, st>>>(F->gt_src.as<int32_t>(), gnnz, F->g_vals.as<double>(),
                                                                  F->gt_vals.as<double>());
   else
      k_gather_vals<float><<<grid_for(gnnz, 1024), 256, 0, st>>>(F->gt_src.as<int32_t>(), gnnz, F->g_vals.as<float>(),
                                                                 F->gt_vals.as<float>());
   TNLB_CHECK_LAUNCH();
   return TNLB_OK;
}

// New values of the two factors (device arrays over G's pattern): G_L's
// values, and H = G_U^T's, from which G_U (stored as CSR) is gathered.
tnlb_status fsai_set_values2(Fsai* F, const void* glvals, const void* hvals, cudaStream_t st)
{
   TNLB_REQUIRE(F->two_factor, TNLB_ERR_INVALID_ARGUMENT, "fsai_set_values2: not a two-factor FSAI");
   const int64_t gnnz = F->g->elements;
   const size_t rs = F->real == TNLB_F64 ? 8 : 4;
   TNLB_CUDA_TRY(cudaMemcpyAsync(F->g_vals.ptr, glvals, rs * gnnz, cudaMemcpyDeviceToDevice, st));
   if (F->real == TNLB_F64)
      k_gather_vals<double><<<grid_for(gnnz, 1024), 256, 0, st>>>(F->gt_src.as<int32_t>(), gnnz,
                                                                  (const double*)hvals, F->gt_vals.as<double>());
   else
      k_gather_vals<float><<<grid_for(gnnz, 1024), 256, 0, st>>>(F->gt_src.as<int32_t>(), gnnz,
                                                                 (const float*)hvals, F->gt_vals.as<float>());
   TNLB_CHECK_LAUNCH();
   return TNLB_OK;
}

// z = G^T (G r)
tnlb_status fsai_apply(const Fsai* F, const void* r, void* z, cudaStream_t st, const int32_t* skip)
{
   TNLB_TRY_STATUS(
      spmv_dispatch(F->g, F->real, F->g_cols.as<int32_t>(), F->g_vals.ptr, r, F->tmp.ptr, 1.0, 0.0, st, skip));
   return spmv_dispatch(F->gt, F->real, F->gt_cols.as<int32_t>(), F->gt_vals.ptr, F->tmp.ptr, z, 1.0, 0.0, st, skip);
}

bool fsai_two_factor(const Fsai* F) { return F->two_factor; }

FsaiView fsai_view(const Fsai* F)
{
   FsaiView v;
   v.g = F->g;
   v.gt = F->gt;
   v.gcols = F->g_cols.as<int32_t>();
   v.gtcols = F->gt_cols.as<int32_t>();
   v.gvals = F->g_vals.ptr;
   v.gtvals = F->gt_vals.ptr;
   v.tmp = F->tmp.ptr;
   return v;
}

bool fsai_dot_fusable(const Fsai* F) { return !F->two_factor && spmv_dot_fusable(F->g) && spmv_dot_fusable(F->gt); }

// t = G r with (t, t) = (r, G^T G r) summed in the same kernel; z = G^T t
tnlb_status fsai_apply_dot(const Fsai* F, const void* r, void* z, double* partials, unsigned* counter, double* rz_out,
                           cudaStream_t st, const int32_t* skip)
{
   TNLB_REQUIRE(fsai_dot_fusable(F), TNLB_ERR_INVALID_ARGUMENT, "fsai_apply_dot: not a symmetric short-row FSAI");
   TNLB_TRY_STATUS(spmv_dot(F->g, F->real, F->g_cols.as<int32_t>(), F->g_vals.ptr, r, F->tmp.ptr, partials, counter,
                            rz_out, st, skip, true));
   return spmv_dispatch(F->gt, F->real, F->gt_cols.as<int32_t>(), F->gt_vals.ptr, F->tmp.ptr, z, 1.0, 0.0, st, skip);
}

tnlb_status fsai_apply_dot_xpby(const Fsai* F, tnlb_real vec, const void* r, void* p, double* partials,
                                unsigned* counter, double* rz_out, const double* rz_old, cudaStream_t st,
                                const int32_t* skip)
{
   TNLB_REQUIRE(fsai_dot_fusable(F), TNLB_ERR_INVALID_ARGUMENT, "fsai_apply_dot_xpby: not a symmetric short-row FSAI");
   TNLB_TRY_STATUS(spmv_dot_mixed(F->g, F->real, vec, F->real, F->g_cols.as<int32_t>(), F->g_vals.ptr, r, F->tmp.ptr,
                                  partials, counter, rz_out, st, skip, true));
   return spmv_xpby_mixed(F->gt, F->real, F->real, vec, F->gt_cols.as<int32_t>(), F->gt_vals.ptr, F->tmp.ptr, p,
                          rz_out, rz_old, st, skip);
}

void fsai_destroy(Fsai* F) { delete F; }

}  // namespace tnlb
