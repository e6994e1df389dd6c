// compact.cuh -- device side of the compact matrix copies (compact.cu):
// the two row layouts as "row policies" that the products of compact.cu and
// the fused reliable-update kernels of solvers.cu are templated on.
//
// A policy gives each thread R rows per pass of a grid-stride loop (kept
// rolled with `#pragma unroll 1`: left to the compiler, the loop around an
// FP64 dot accumulator was unrolled into a schedule that took the diagonal
// product on the 2048^2 5-point operator from 28.5 to 61.8 us):
//   first(), step()   the loop over pass bases;
//   row(base, k)      row k of the pass (rows at or past n are skipped);
//   rows(base, n, xv, s)  s[k] = sum over the row's entries of v * xv(c),
//                     xv(c) the input at column c, summed in FP32 in
//                     ascending column order;
//   prefetch(base, n) an L2 prefetch of the values of the pass at `base`
//                     (issued a pass ahead; a no-op where it did not pay);
//   kQuad             four consecutive full rows may be read and written
//                     as 16-byte vectors by the kernel's epilogue;
//   kMinBlocks        resident blocks per SM the kernels ask for (0: none).
// Policies: RelRows (16-bit offsets, two consecutive rows per thread),
// DiaRows (diagonals, four consecutive rows, up to 5 diagonals), DiaRow1
// (diagonals, one row, 6 to 8 diagonals).  All sum the same terms in the
// same order -- a missing diagonal slot adds fma(0, x, s) = s -- so for
// finite inputs their row sums are bitwise equal.
//
// Row-excess form (`self` >= 0 / `excess`): the diagonal entry holds the
// row's excess s_i = a_ii + sum_{j != i} a_ij instead of a_ii, and a row
// sums s_i x_i + sum_{j != i} a_ij (x_j - x_i).  On a diagonally dominant
// operator with nonpositive off-diagonals (a diffusion stencil) rounding
// the a_ij to FP32 then perturbs the operator by a Laplacian of relative
// size 2^-24, instead of by 2^-24 ||A|| on every eigenvalue, and x_j - x_i
// of a smooth x is exact (Sterbenz), so the FP32 product keeps the small
// eigenvalues that high-contrast coefficients create.
#pragma once

#include <cuda_fp16.h>

#include <cstdint>
#include <type_traits>

namespace tnlb {

__device__ __forceinline__ float rel_to_f(float v) { return v; }
__device__ __forceinline__ float rel_to_f(__half v) { return __half2float(v); }

// CSR with 16-bit column offsets, R consecutive rows per thread (R + 1 row
// offsets, then every entry load of the R rows issued before the gathers).
template <typename TV, int L, int R>
struct RelRows {
   static constexpr int kR = R;
   static constexpr bool kQuad = false;
   static constexpr int kMinBlocks = 0;  // no residency asked for
   const int32_t* __restrict__ rowptr;
   const int16_t* __restrict__ off;
   const TV* __restrict__ vals;
   bool excess;  // row-excess form

   __device__ __forceinline__ int64_t first() const { return ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) * R; }
   __device__ __forceinline__ int64_t step() const { return (int64_t)gridDim.x * blockDim.x * R; }
   __device__ __forceinline__ int64_t row(int64_t base, int k) const { return base + k; }
   __device__ __forceinline__ void prefetch(int64_t, int32_t) const {}

   template <typename XV>
   __device__ __forceinline__ void rows(int64_t r0, int32_t n, const XV& xv, float (&s)[R]) const
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
         const int32_t row = (int32_t)(r0 + k);
         const float xi = excess && r0 + k < n ? xv(row) : 0.0f;
         float t = 0.0f;
#pragma unroll
         for (int j = 0; j < L; j++)
            if (c[k][j] >= 0) {
               float xx = xv(c[k][j]);
               if (excess && c[k][j] != row) xx -= xi;
               t += v[k][j] * xx;
            }
         s[k] = t;
      }
   }
};

// Column offsets of the diagonals (ascending).
struct DiaOffsets {
   int32_t o[8];
};

// Four consecutive values of a 16-byte-aligned (FP32) or 8-byte-aligned
// (FP16) array.
__device__ __forceinline__ void ld_quad(const float* p, float (&o)[4])
{
   const float4 t = __ldg(reinterpret_cast<const float4*>(p));
   o[0] = t.x;
   o[1] = t.y;
   o[2] = t.z;
   o[3] = t.w;
}
__device__ __forceinline__ void ld_quad(const __half* p, float (&o)[4])
{
   const uint2 t = __ldg(reinterpret_cast<const uint2*>(p));
   const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&t.x));
   const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&t.y));
   o[0] = a.x;
   o[1] = a.y;
   o[2] = b.x;
   o[3] = b.y;
}

// The input of a product: x[c], and x[c .. c+3] for c a multiple of 4.
struct PlainInput {
   const float* __restrict__ x;
   __device__ __forceinline__ float operator()(int32_t c) const { return __ldg(x + c); }
   __device__ __forceinline__ void quad(int32_t c, float (&o)[4]) const { ld_quad(x + c, o); }
};

// Diagonal layout, four consecutive rows per thread (kQuad): the value
// pitch is a multiple of 4, so each diagonal's four values are one vector
// load, and so is the input of a diagonal whose offset is a multiple of 4
// (0 and +-N on an N-wide grid); the other diagonals' inputs are four
// scalar loads that mostly hit the same sectors.  A column outside [0, n)
// has a zero value and reads nothing.  Columns are formed in 32 bits
// (n < 2^31).  The input functor needs operator()(c) and quad(c, o).
template <typename TV, int D>
struct DiaRows {
   static constexpr int kR = 4;
   static constexpr bool kQuad = true;
   // resident 256-thread blocks per SM asked for (0: none); 5 for the
   // 3-diagonal FSAI factors of a 5-point operator (48 registers)
   static constexpr int kMinBlocks = D <= 3 ? 5 : 0;
   const TV* __restrict__ vals;
   DiaOffsets d;
   int64_t pitch;
   int32_t self;  // row-excess form: the slot of offset 0; -1 plain

   __device__ __forceinline__ int64_t first() const
   {
      return ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) * 4;
   }
   __device__ __forceinline__ int64_t step() const { return (int64_t)gridDim.x * blockDim.x * 4; }
   __device__ __forceinline__ int64_t row(int64_t base, int k) const { return base + k; }
   // L2 prefetch of the value lines of the pass at `base` (one thread per
   // 128-byte line), issued a pass ahead so that its loads find them in L2.
   __device__ __forceinline__ void prefetch(int64_t base, int32_t nr) const
   {
      constexpr int kPerLine = 128 / (4 * (int)sizeof(TV));
      if (base >= nr || (threadIdx.x & (kPerLine - 1)) != 0) return;
#pragma unroll
      for (int j = 0; j < D; j++)
         asm volatile("prefetch.global.L2 [%0];" ::"l"(vals + (int64_t)j * pitch + base));
   }

   template <typename XV>
   __device__ __forceinline__ void rows(int64_t base, int32_t nr, const XV& xv, float (&s)[4]) const
   {
      const int32_t i0 = (int32_t)base;
      const bool full = base + 3 < nr;
      float v[D][4], x[D][4];
#pragma unroll
      for (int j = 0; j < D; j++) {
         const TV* vp = vals + (int64_t)j * pitch + i0;
         const int32_t c0 = i0 + d.o[j];
         if (full)
            ld_quad(vp, v[j]);
         else
#pragma unroll
            for (int k = 0; k < 4; k++) v[j][k] = i0 + k < nr ? rel_to_f(__ldg(vp + k)) : 0.0f;
         if (full && (d.o[j] & 3) == 0 && c0 >= 0 && c0 + 3 < nr)
            xv.quad(c0, x[j]);
         else
#pragma unroll
            for (int k = 0; k < 4; k++) {
               const int32_t c = c0 + k;
               const bool in = i0 + k < nr && (uint32_t)c < (uint32_t)nr;
               x[j][k] = in ? xv(c) : 0.0f;
               if (!in) v[j][k] = 0.0f;
            }
      }
      if (self >= 0) {
         float xi[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
         for (int j = 0; j < D; j++)
            if (j == self)
#pragma unroll
               for (int k = 0; k < 4; k++) xi[k] = x[j][k];
#pragma unroll
         for (int j = 0; j < D; j++)
            if (j != self)
#pragma unroll
               for (int k = 0; k < 4; k++) x[j][k] -= xi[k];
      }
#pragma unroll
      for (int k = 0; k < 4; k++) {
         float t = 0.0f;
#pragma unroll
         for (int j = 0; j < D; j++) t += v[j][k] * x[j][k];
         s[k] = t;
      }
   }
};

// Diagonal layout, one row per thread (for 6 to 8 diagonals, where the
// four-row form's registers -- 77 at 7 diagonals -- cut the resident warps
// and measured slower on the 7-point 256^3 operator): every load of a warp
// one contiguous run, the D value and D input loads issued before the sum.
template <typename TV, int D>
struct DiaRow1 {
   static constexpr int kR = 1;
   static constexpr bool kQuad = false;
   static constexpr int kMinBlocks = 0;  // no residency asked for
   const TV* __restrict__ vals;
   DiaOffsets d;
   int64_t pitch;
   int32_t self;  // row-excess form: the slot of offset 0; -1 plain

   __device__ __forceinline__ int64_t first() const { return (int64_t)blockIdx.x * blockDim.x + threadIdx.x; }
   __device__ __forceinline__ int64_t step() const { return (int64_t)gridDim.x * blockDim.x; }
   __device__ __forceinline__ int64_t row(int64_t base, int) const { return base; }
   __device__ __forceinline__ void prefetch(int64_t, int32_t) const {}

   template <typename XV>
   __device__ __forceinline__ void rows(int64_t base, int32_t nr, const XV& xv, float (&s)[1]) const
   {
      const int32_t i = (int32_t)base;
      const bool rin = base < nr;
      const TV* vp = vals + i;
      float v[D], x[D];
#pragma unroll
      for (int j = 0; j < D; j++) {
         const int32_t c = i + d.o[j];
         const bool in = rin && (uint32_t)c < (uint32_t)nr;
         v[j] = in ? rel_to_f(__ldg(vp + (int64_t)j * pitch)) : 0.0f;
         x[j] = in ? xv(c) : 0.0f;
      }
      if (self >= 0) {
         float xi = 0.0f;
#pragma unroll
         for (int j = 0; j < D; j++)
            if (j == self) xi = x[j];
#pragma unroll
         for (int j = 0; j < D; j++)
            if (j != self) x[j] -= xi;
      }
      float t = 0.0f;
#pragma unroll
      for (int j = 0; j < D; j++) t += v[j] * x[j];
      s[0] = t;
   }
};

// Rows per thread: two for up to 8 entries a row, as the short-row sweep on
// the 5-point operator and its triangular factor favoured (FP16 values:
// 25 -> 19 us on the factor).
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

#define TNLB_DIA_CASE(DD, ...)   \
   case DD: {                    \
      constexpr int D = DD;      \
      __VA_ARGS__;               \
      break;                     \
   }
#define TNLB_DIA_WIDTH(m, ...)                    \
   do {                                           \
      switch (m) {                                \
         TNLB_DIA_CASE(1, __VA_ARGS__)            \
         TNLB_DIA_CASE(2, __VA_ARGS__)            \
         TNLB_DIA_CASE(3, __VA_ARGS__)            \
         TNLB_DIA_CASE(4, __VA_ARGS__)            \
         TNLB_DIA_CASE(5, __VA_ARGS__)            \
         TNLB_DIA_CASE(6, __VA_ARGS__)            \
         TNLB_DIA_CASE(7, __VA_ARGS__)            \
         default: {                               \
            constexpr int D = 8;                  \
            __VA_ARGS__;                          \
         }                                        \
      }                                           \
   } while (0)

// `using Rows = <the policy of copy C with values TV>;` then the body.
#define TNLB_COMPACT_ROWS(C, TV, ...)                                                                  \
   do {                                                                                                \
      if ((C).kind == CompactCopy::kDia) {                                                             \
         TNLB_DIA_WIDTH((C).width, {                                                                   \
            using Rows = std::conditional_t<(D <= 5), DiaRows<TV, D>, DiaRow1<TV, D>>;                 \
            DiaOffsets dd_;                                                                            \
            for (int q_ = 0; q_ < 8; q_++) dd_.o[q_] = (C).diag[q_];                                   \
            const Rows rows_{(C).vals.template as<TV>(), dd_, (C).pitch, (C).self_slot};              \
            __VA_ARGS__;                                                                               \
         });                                                                                           \
      }                                                                                                \
      else {                                                                                           \
         TNLB_REL_WIDTH((C).width, {                                                                   \
            using Rows = RelRows<TV, L, rel_rows_per_thread<L>()>;                                     \
            const Rows rows_{(C).rowptr, (C).off.template as<int16_t>(), (C).vals.template as<TV>(),   \
                             (C).self_slot >= 0};                                                      \
            __VA_ARGS__;                                                                               \
         });                                                                                           \
      }                                                                                                \
   } while (0)

}  // namespace tnlb
