// spmv_sym.cu -- the products of SparseMatrixBase that scatter with atomic
// additions, for every segment format:
//  * vectorProduct of a symmetric matrix (SparseMatrixBase.hpp:296-330):
//    one triangle is stored; a stored a_rc with c < r also adds
//    alpha a_rc x[r] to y[c];
//  * transposedVectorProduct (SparseMatrixBase.hpp:542-588):
//    y[c] += alpha x[r] a_rc over the stored elements.
// As in the reference, y is first multiplied by beta unless beta == 1 (read
// even when beta == 0), and the scattered additions are atomic, so their
// order -- and the last bits of y -- is not fixed.  G lanes take one row,
// G from the mean row length (as Light CSR picks it); elements are reached
// through the formats' getGlobalIndex (segview.cuh), so one kernel serves
// CSR, Ellpack, SlicedEllpack, ChunkedEllpack, BiEllpack and AdaptiveCSR.
#include "internal.cuh"
#include "segview.cuh"

namespace tnlb {
namespace {

template <typename Real>
__global__ void k_scale_in_place(int64_t n, Real b, Real* __restrict__ y)
{
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
      y[i] = y[i] * b;
}

template <typename Real, int G>
__global__ void k_spmv_symmetric(SegView v, const int32_t* __restrict__ cols, const Real* __restrict__ vals,
                                 const Real* __restrict__ x, Real* __restrict__ y, Real alpha, int32_t begin,
                                 int32_t end)
{
   const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   const int64_t row = begin + gid / G;
   const int lane = (int)(gid % G);
   Real sum = Real(0);
   if (row < end) {
      const Real xr = x[row];
      for (int32_t local = lane;; local += G) {
         const int64_t gi = global_index_of(v, (int32_t)row, local);
         if (gi < 0) break;
         const int32_t c = cols[gi];
         if (c < 0) continue;  // padding
         const Real a = vals[gi];
         if (c < row) atomicAdd(y + c, alpha * a * xr);
         sum += a * x[c];
      }
   }
   sum = group_sum<G>(sum);
   if (row < end && lane == 0) atomicAdd(y + row, alpha * sum);
}

template <typename Real, int G>
__global__ void k_spmv_transposed(SegView v, const int32_t* __restrict__ cols, const Real* __restrict__ vals,
                                  const Real* __restrict__ x, Real* __restrict__ y, Real alpha, int32_t n,
                                  int32_t begin, int32_t end)
{
   const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   const int64_t row = gid / G;
   const int lane = (int)(gid % G);
   if (row >= n) return;
   const Real axr = alpha * x[row];
   for (int32_t local = lane;; local += G) {
      const int64_t gi = global_index_of(v, (int32_t)row, local);
      if (gi < 0) break;
      const int32_t c = cols[gi];
      if (c >= begin && c < end && c != -1) atomicAdd(y + c, axr * vals[gi]);
   }
}

int lanes_for(const tnlb_segments* seg)
{
   if (seg->n <= 0) return 2;
   const int64_t e = (seg->storage + seg->n - 1) / seg->n;
   if (e <= 2) return 2;
   if (e <= 4) return 4;
   if (e <= 8) return 8;
   if (e <= 16) return 16;
   return 32;
}

template <typename Real>
tnlb_status symmetric_t(const tnlb_segments* seg, const int32_t* cols, const Real* vals, const Real* x, Real* y,
                        Real alpha, Real beta, int32_t begin, int32_t end, cudaStream_t st)
{
   const int64_t n = seg->n;
   if (beta != Real(1)) {
      k_scale_in_place<Real><<<grid_for(n, 256 * 4), 256, 0, st>>>(n, beta, y);
      TNLB_CHECK_LAUNCH();
   }
   const int64_t rows = (int64_t)end - begin;
   if (rows <= 0) return TNLB_OK;
   const SegView v = view_of(seg);
   const int G = lanes_for(seg);
#define TNLB_SYM(GG)                                                                                           \
   case GG:                                                                                                    \
      k_spmv_symmetric<Real, GG><<<grid_for(rows * GG, 256), 256, 0, st>>>(v, cols, vals, x, y, alpha, begin, \
                                                                            end);                              \
      break;
   switch (G) {
      TNLB_SYM(2)
      TNLB_SYM(4)
      TNLB_SYM(8)
      TNLB_SYM(16)
      TNLB_SYM(32)
   }
#undef TNLB_SYM
   TNLB_CHECK_LAUNCH();
   return TNLB_OK;
}

template <typename Real>
tnlb_status transposed_t(const tnlb_segments* seg, const int32_t* cols, const Real* vals, int32_t columns,
                         const Real* x, Real* y, Real alpha, Real beta, int32_t begin, int32_t end, cudaStream_t st)
{
   if (beta != Real(1) && columns > 0) {
      k_scale_in_place<Real><<<grid_for(columns, 256 * 4), 256, 0, st>>>(columns, beta, y);
      TNLB_CHECK_LAUNCH();
   }
   const int64_t n = seg->n;
   if (n <= 0 || end <= begin) return TNLB_OK;
   const SegView v = view_of(seg);
   const int G = lanes_for(seg);
#define TNLB_TR(GG)                                                                                              \
   case GG:                                                                                                      \
      k_spmv_transposed<Real, GG><<<grid_for(n * GG, 256), 256, 0, st>>>(v, cols, vals, x, y, alpha, (int32_t)n, \
                                                                          begin, end);                           \
      break;
   switch (G) {
      TNLB_TR(2)
      TNLB_TR(4)
      TNLB_TR(8)
      TNLB_TR(16)
      TNLB_TR(32)
   }
#undef TNLB_TR
   TNLB_CHECK_LAUNCH();
   return TNLB_OK;
}

}  // namespace
}  // namespace tnlb

using namespace tnlb;

extern "C" tnlb_status tnlb_spmv_symmetric(const tnlb_segments* seg, tnlb_real real, const int32_t* d_cols,
                                          const void* d_values, const void* d_x, void* d_y, double alpha,
                                          double beta, int32_t begin, int32_t end, tnlb_stream stream)
{
   clear_error();
   TNLB_REQUIRE(seg != nullptr, TNLB_ERR_INVALID_ARGUMENT, "null segments");
   TNLB_REQUIRE(real == TNLB_F32 || real == TNLB_F64, TNLB_ERR_INVALID_ARGUMENT, "unknown real type");
   if (end == 0) end = seg->n;
   TNLB_REQUIRE(begin >= 0 && begin <= end && end <= seg->n, TNLB_ERR_INVALID_ARGUMENT,
                "vectorProduct: row range [begin, end) outside the matrix");
   if (seg->n == 0) return TNLB_OK;
   TNLB_REQUIRE(d_y != nullptr && (seg->storage == 0 || (d_cols && d_values && d_x)), TNLB_ERR_INVALID_ARGUMENT,
                "null array");
   const cudaStream_t st = (cudaStream_t)stream;
   if (real == TNLB_F64)
      return symmetric_t<double>(seg, d_cols, (const double*)d_values, (const double*)d_x, (double*)d_y, alpha, beta,
                                 begin, end, st);
   return symmetric_t<float>(seg, d_cols, (const float*)d_values, (const float*)d_x, (float*)d_y, (float)alpha,
                             (float)beta, begin, end, st);
}

extern "C" tnlb_status tnlb_spmv_transposed(const tnlb_segments* seg, tnlb_real real, const int32_t* d_cols,
                                           const void* d_values, int32_t columns, const void* d_x, void* d_y,
                                           double alpha, double beta, int32_t begin, int32_t end, tnlb_stream stream)
{
   clear_error();
   TNLB_REQUIRE(seg != nullptr, TNLB_ERR_INVALID_ARGUMENT, "null segments");
   TNLB_REQUIRE(real == TNLB_F32 || real == TNLB_F64, TNLB_ERR_INVALID_ARGUMENT, "unknown real type");
   TNLB_REQUIRE(columns >= 0, TNLB_ERR_INVALID_ARGUMENT,
                "transposedVectorProduct: size of the output vector does not match the number of matrix columns");
   if (end == 0) end = columns;
   TNLB_REQUIRE(begin >= 0 && begin <= end && end <= columns, TNLB_ERR_INVALID_ARGUMENT,
                "transposedVectorProduct: column range [begin, end) outside the matrix");
   if (columns == 0) return TNLB_OK;
   TNLB_REQUIRE(d_y != nullptr && (seg->storage == 0 || (d_cols && d_values && d_x)), TNLB_ERR_INVALID_ARGUMENT,
                "null array");
   const cudaStream_t st = (cudaStream_t)stream;
   if (real == TNLB_F64)
      return transposed_t<double>(seg, d_cols, (const double*)d_values, columns, (const double*)d_x, (double*)d_y,
                                  alpha, beta, begin, end, st);
   return transposed_t<float>(seg, d_cols, (const float*)d_values, columns, (const float*)d_x, (float*)d_y,
                              (float)alpha, (float)beta, begin, end, st);
}
