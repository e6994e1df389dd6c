// spmv_rel.cuh -- device helpers of the compact short-row CSR copies
// (16-bit column offsets from the row, FP32 or FP16 values; spmv_rel.cu),
// shared by their products and by the fused reliable-update kernels of
// solvers.cu.
#pragma once

#include <cuda_fp16.h>

#include <cstdint>

namespace tnlb {

__device__ __forceinline__ float rel_to_f(float v) { return v; }
__device__ __forceinline__ float rel_to_f(__half v) { return __half2float(v); }

// Rows r0 .. r0 + R - 1 (consecutive: R + 1 row offsets, then every entry
// load of the R rows is issued before the x gathers); xv(c) is x[c].  Rows
// at or past n give 0.
template <typename TV, int L, int R, typename XV>
__device__ __forceinline__ void rel_rows_f(const int32_t* __restrict__ rowptr, const int16_t* __restrict__ off,
                                           const TV* __restrict__ vals, const XV& xv, int64_t r0, int32_t n,
                                           float (&s)[R])
{
   int32_t bnd[R + 1];
#pragma unroll
   for (int k = 0; k <= R; k++) bnd[k] = r0 + k <= n ? __ldg(rowptr + r0 + k) : 0;
   int32_t c[R][L];
   float v[R][L];
#pragma unroll
   for (int k = 0; k < R; k++)
#pragma unroll
      for (int j = 0; j < L; j++) {
         c[k][j] = -1;
         v[k][j] = 0.0f;
         if (r0 + k < n && bnd[k] + j < bnd[k + 1]) {
            c[k][j] = (int32_t)(r0 + k) + (int32_t)__ldg(off + bnd[k] + j);
            v[k][j] = rel_to_f(__ldg(vals + bnd[k] + j));
         }
      }
#pragma unroll
   for (int k = 0; k < R; k++) {
      float t = 0.0f;
#pragma unroll
      for (int j = 0; j < L; j++)
         if (c[k][j] >= 0) t += v[k][j] * xv(c[k][j]);
      s[k] = t;
   }
}

template <typename TV, int L, int R>
__device__ __forceinline__ void rel_rows(const int32_t* __restrict__ rowptr, const int16_t* __restrict__ off,
                                         const TV* __restrict__ vals, const float* __restrict__ x, int64_t r0,
                                         int32_t n, float (&s)[R])
{
   rel_rows_f<TV, L, R>(rowptr, off, vals, [x](int32_t c) { return __ldg(x + c); }, r0, n, s);
}

// Rows per thread: two consecutive rows for up to 8 entries a row, as the
// short-row sweep on the 5-point operator and its triangular factor favoured
// (FP16 values: 25 -> 19 us on the factor).
template <int L>
constexpr int rel_rows_per_thread()
{
   return L <= 8 ? 2 : 1;
}

#define TNLB_REL_WIDTH(m, ...)   \
   do {                          \
      if ((m) <= 4) {            \
         constexpr int L = 4;    \
         __VA_ARGS__;            \
      }                          \
      else if ((m) <= 5) {       \
         constexpr int L = 5;    \
         __VA_ARGS__;            \
      }                          \
      else if ((m) <= 7) {       \
         constexpr int L = 7;    \
         __VA_ARGS__;            \
      }                          \
      else if ((m) <= 8) {       \
         constexpr int L = 8;    \
         __VA_ARGS__;            \
      }                          \
      else {                     \
         constexpr int L = 16;   \
         __VA_ARGS__;            \
      }                          \
   } while (0)


}  // namespace tnlb
