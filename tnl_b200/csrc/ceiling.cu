// ceiling.cu -- the attainable rate of a CSR product's memory traffic on this
// GPU, for reporting a kernel against it (no counterpart in the reference).
//
// k_stream_gather moves exactly the bytes of y = A x for a CSR matrix and
// does the same random gathers, with no reduction by rows: each warp streams
// 256 consecutive column indexes and values (the loads and L2 policies of
// the tile kernel: non-caching, evict-first), gathers x at every column
// (evict-last), and keeps one running sum per thread; the row pointer is
// read once and y written once by a thread-per-row pass over the same grid.
// Mode 0 skips the gathers (the streaming rate alone).  On a matrix whose
// columns are uniformly random the gathers, one 32-byte sector each, bound
// the product well below the copy bandwidth: this kernel measures that
// bound.
#include "internal.cuh"

namespace tnlb {
namespace {

__device__ __forceinline__ uint64_t pol_first()
{
   uint64_t p;
   asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
   return p;
}
__device__ __forceinline__ uint64_t pol_last()
{
   uint64_t p;
   asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
   return p;
}
__device__ __forceinline__ int32_t ldh(const int32_t* a, uint64_t pol)
{
   int32_t v;
   asm("ld.global.nc.L1::no_allocate.L2::cache_hint.s32 %0, [%1], %2;" : "=r"(v) : "l"(a), "l"(pol));
   return v;
}
__device__ __forceinline__ double ldh(const double* a, uint64_t pol)
{
   double v;
   asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(a), "l"(pol));
   return v;
}
__device__ __forceinline__ float ldh(const float* a, uint64_t pol)
{
   float v;
   asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(a), "l"(pol));
   return v;
}

template <typename Real, bool Gather>
__global__ void __launch_bounds__(256) k_stream_gather(const int32_t* __restrict__ rowptr,
                                                       const int32_t* __restrict__ cols, const Real* __restrict__ vals,
                                                       const Real* __restrict__ x, Real* __restrict__ y, int32_t n,
                                                       int64_t nnz)
{
   constexpr int kItems = 8;
   const int lane = threadIdx.x & 31;
   const int64_t base = (((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32 * kItems;
   const uint64_t pf = pol_first(), pl = pol_last();
   Real s = Real(0);
   if (base < nnz) {
      int32_t c[kItems];
      Real v[kItems];
#pragma unroll
      for (int j = 0; j < kItems; j++) {
         const int64_t e = base + j * 32 + lane;
         c[j] = -1;
         v[j] = Real(0);
         if (e < nnz) {
            c[j] = ldh(cols + e, pf);
            v[j] = ldh(vals + e, pf);
         }
      }
#pragma unroll
      for (int j = 0; j < kItems; j++) {
         if (Gather) {
            if (c[j] >= 0) s += v[j] * ldh(x + c[j], pl);
         }
         else
            s += v[j] * (Real)c[j];
      }
   }
   // rows: the row pointer read and y written once, thread per row
   const int64_t nthreads = (int64_t)gridDim.x * blockDim.x;
   for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += nthreads)
      y[r] = (Real)ldh(rowptr + r, pf) + s;
}

template <typename Real>
void launch(int mode, const int32_t* rowptr, const int32_t* cols, const Real* vals, const Real* x, Real* y,
            int32_t n, int64_t nnz, cudaStream_t st)
{
   const unsigned g = grid_for((nnz + 255) / 256, 8);
   if (mode == 1)
      k_stream_gather<Real, true><<<g, 256, 0, st>>>(rowptr, cols, vals, x, y, n, nnz);
   else
      k_stream_gather<Real, false><<<g, 256, 0, st>>>(rowptr, cols, vals, x, y, n, nnz);
}

}  // namespace
}  // namespace tnlb

extern "C" tnlb_status tnlb_bench_stream_gather(tnlb_real real, int32_t mode, int32_t rows, int64_t nnz,
                                                const int32_t* d_rowptr, const int32_t* d_cols, const void* d_values,
                                                const void* d_x, void* d_y, tnlb_stream stream)
{
   using namespace tnlb;
   clear_error();
   TNLB_REQUIRE(real == TNLB_F32 || real == TNLB_F64, TNLB_ERR_INVALID_ARGUMENT, "unknown real type");
   TNLB_REQUIRE(mode == 0 || mode == 1, TNLB_ERR_INVALID_ARGUMENT, "mode must be 0 (stream) or 1 (stream + gather)");
   TNLB_REQUIRE(rows > 0 && nnz > 0 && d_rowptr && d_cols && d_values && d_x && d_y, TNLB_ERR_INVALID_ARGUMENT,
                "bad arguments");
   cudaStream_t st = (cudaStream_t)stream;
   if (real == TNLB_F64)
      launch<double>(mode, d_rowptr, d_cols, (const double*)d_values, (const double*)d_x, (double*)d_y, rows, nnz, st);
   else
      launch<float>(mode, d_rowptr, d_cols, (const float*)d_values, (const float*)d_x, (float*)d_y, rows, nnz, st);
   TNLB_CHECK_LAUNCH();
   return TNLB_OK;
}
