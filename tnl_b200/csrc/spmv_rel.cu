// spmv_rel.cu -- compact copies of short-row CSR matrices for the FP32
// iterations of the reliable-update PCG (solvers.cu): each column stored as
// a 16-bit offset from its row (every |column - row| < 32768, as in the
// stencils and their FSAI factors) and the values in FP32 or FP16.  The
// solver builds them from its own FP32 copies; the caller's matrix and the
// public formats are untouched.
//
// Per entry the product then reads 6 bytes (FP32 value + offset) or 4 (FP16
// value + offset) instead of 8, on the bandwidth-bound FP32 iteration.
// Rows are summed in FP32 in entry order, as the CSR short-row kernels do.
#include <cuda_fp16.h>

#include "internal.cuh"
#include "reduce.cuh"
#include "spmv_rel.cuh"

namespace tnlb {

namespace {

// offsets[k] = cols[k] - row(k); *bad = 1 if one does not fit in int16
__global__ void k_rel_offsets(const int32_t* __restrict__ rowptr, const int32_t* __restrict__ cols, int32_t n,
                              int16_t* __restrict__ off, int32_t* __restrict__ bad)
{
   const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (r >= n) return;
   for (int32_t k = rowptr[r]; k < rowptr[r + 1]; k++) {
      const int64_t d = (int64_t)cols[k] - r;
      if (cols[k] < 0 || d < -32768 || d > 32767) {
         *bad = 1;
         off[k] = 0;
      }
      else
         off[k] = (int16_t)d;
   }
}

__global__ void k_to_half(const float* __restrict__ a, int64_t n, __half* __restrict__ b)
{
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
      b[i] = __float2half_rn(a[i]);
}

// y = A x and (x, y) -- or (y, y) with `self` -- as k_csr_short_dot does.
template <typename TV, int L, int R>
__global__ void __launch_bounds__(256) k_rel_dot(const int32_t* __restrict__ rowptr, const int16_t* __restrict__ off,
                                                 const TV* __restrict__ vals, const float* __restrict__ x,
                                                 float* __restrict__ y, int32_t n, RedWork w,
                                                 double* __restrict__ dot_out, const int32_t* __restrict__ skip,
                                                 int self)
{
   if (skip && *skip) return;
   double d = 0.0;
   const int64_t stride = (int64_t)gridDim.x * blockDim.x * R;
   for (int64_t r0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) * R; r0 < n; r0 += stride) {
      float s[R];
      rel_rows<TV, L, R>(rowptr, off, vals, x, r0, n, s);
#pragma unroll
      for (int k = 0; k < R; k++)
         if (r0 + k < n) {
            y[r0 + k] = s[k];
            d += (double)s[k] * (self ? (double)s[k] : (double)__ldg(x + r0 + k));
         }
   }
   double vv[1] = {d};
   if (publish_and_arrive<1>(vv, w)) {
      double t[1];
      gather_totals<1>(t, w);
      if (threadIdx.x == 0) *dot_out = t[0];
   }
}

// y = A x + (num / den) y, as k_csr_short_xpby does.
template <typename TV, int L, int R>
__global__ void __launch_bounds__(256) k_rel_xpby(const int32_t* __restrict__ rowptr, const int16_t* __restrict__ off,
                                                  const TV* __restrict__ vals, const float* __restrict__ x,
                                                  float* __restrict__ y, int32_t n, const double* __restrict__ num,
                                                  const double* __restrict__ den, const int32_t* __restrict__ skip)
{
   if (skip && *skip) return;
   const float beta = (float)(*num / *den);
   const int64_t stride = (int64_t)gridDim.x * blockDim.x * R;
   for (int64_t r0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) * R; r0 < n; r0 += stride) {
      float s[R];
      rel_rows<TV, L, R>(rowptr, off, vals, x, r0, n, s);
#pragma unroll
      for (int k = 0; k < R; k++)
         if (r0 + k < n) y[r0 + k] = s[k] + beta * y[r0 + k];
   }
}

}  // namespace

tnlb_status rel_csr_build(const tnlb_segments* seg, const int32_t* cols, const float* vals, bool half,
                          cudaStream_t st, RelCsr* out, bool* ok)
{
   *ok = false;
   if (!spmv_dot_fusable(seg)) return TNLB_OK;
   const int32_t n = seg->n;
   const int64_t nnz = seg->elements;
   out->n = n;
   out->max_row = seg->max_row;
   out->rowptr = seg->offsets.as<int32_t>();
   out->half = half;
   DeviceBuffer bad;
   TNLB_TRY_STATUS(bad.alloc(sizeof(int32_t)));
   TNLB_CUDA_TRY(cudaMemsetAsync(bad.ptr, 0, sizeof(int32_t), st));
   TNLB_TRY_STATUS(out->off.alloc(sizeof(int16_t) * (nnz > 0 ? nnz : 1)));
   k_rel_offsets<<<grid_for(n, 256), 256, 0, st>>>(out->rowptr, cols, n, out->off.as<int16_t>(), bad.as<int32_t>());
   TNLB_CHECK_LAUNCH();
   if (half) {
      TNLB_TRY_STATUS(out->vals.alloc(sizeof(__half) * (nnz > 0 ? nnz : 1)));
      k_to_half<<<grid_for(nnz, 256 * 8), 256, 0, st>>>(vals, nnz, out->vals.as<__half>());
      TNLB_CHECK_LAUNCH();
   }
   else {
      TNLB_TRY_STATUS(out->vals.alloc(sizeof(float) * (nnz > 0 ? nnz : 1)));
      if (nnz) TNLB_CUDA_TRY(cudaMemcpyAsync(out->vals.ptr, vals, sizeof(float) * nnz, cudaMemcpyDeviceToDevice, st));
   }
   int32_t h = 0;
   TNLB_CUDA_TRY(cudaMemcpyAsync(&h, bad.ptr, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
   TNLB_CUDA_TRY(cudaStreamSynchronize(st));
   *ok = h == 0;
   return TNLB_OK;
}

tnlb_status rel_spmv_dot(const RelCsr& A, const float* x, float* y, double* partials, unsigned* counter,
                         double* dot_out, cudaStream_t st, const int32_t* skip, bool self_dot)
{
   RedWork w{partials, counter};
   const int self = self_dot ? 1 : 0;
   if (A.half)
      TNLB_REL_WIDTH(A.max_row, {
         constexpr int R = rel_rows_per_thread<L>();
         auto* k = k_rel_dot<__half, L, R>;
         const unsigned g = resident_grid((const void*)k, 256, A.n, R);
         k<<<g, 256, 0, st>>>(A.rowptr, A.off.as<int16_t>(), A.vals.as<__half>(), x, y, A.n, w, dot_out, skip, self);
      });
   else
      TNLB_REL_WIDTH(A.max_row, {
         constexpr int R = rel_rows_per_thread<L>();
         auto* k = k_rel_dot<float, L, R>;
         const unsigned g = resident_grid((const void*)k, 256, A.n, R);
         k<<<g, 256, 0, st>>>(A.rowptr, A.off.as<int16_t>(), A.vals.as<float>(), x, y, A.n, w, dot_out, skip, self);
      });
   TNLB_CHECK_LAUNCH();
   return TNLB_OK;
}

tnlb_status rel_spmv_xpby(const RelCsr& A, const float* x, float* y, const double* num, const double* den,
                          cudaStream_t st, const int32_t* skip)
{
   if (A.half)
      TNLB_REL_WIDTH(A.max_row, {
         constexpr int R = rel_rows_per_thread<L>();
         auto* k = k_rel_xpby<__half, L, R>;
         const unsigned g = resident_grid((const void*)k, 256, A.n, R);
         k<<<g, 256, 0, st>>>(A.rowptr, A.off.as<int16_t>(), A.vals.as<__half>(), x, y, A.n, num, den, skip);
      });
   else
      TNLB_REL_WIDTH(A.max_row, {
         constexpr int R = rel_rows_per_thread<L>();
         auto* k = k_rel_xpby<float, L, R>;
         const unsigned g = resident_grid((const void*)k, 256, A.n, R);
         k<<<g, 256, 0, st>>>(A.rowptr, A.off.as<int16_t>(), A.vals.as<float>(), x, y, A.n, num, den, skip);
      });
   TNLB_CHECK_LAUNCH();
   return TNLB_OK;
}

}  // namespace tnlb
