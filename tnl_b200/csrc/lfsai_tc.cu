// lfsai_tc.cu -- the learned-FSAI network's dense layers on the 5th-generation
// tensor cores (tcgen05, sm_100a).
//
// One CTA of 128 threads processes tiles of 128 rows: thread t owns row t.
// Per layer the row activations (BF16) and the weights (BF16) sit in shared
// memory in the canonical K-major, non-swizzled core-matrix layout (8 rows x
// 16 bytes per core matrix; neighbouring core matrices 128 B apart along K,
// 8-row groups K/8*128 B apart); one elected thread issues
// tcgen05.mma.cta_group::1.kind::f16 (M=128, N=64 or 16, K=16 per
// instruction; 2 instructions for the 32 features of layer 1) into an FP32 accumulator in tensor memory, commits to an
// mbarrier, and every thread reads its row back with tcgen05.ld (32x32b: warp
// w reads TMEM lanes 32w..32w+31), adds the bias, applies ReLU and writes the
// next layer's BF16 input.  Waits on the mbarrier are bounded: on timeout the
// CTA records an error, releases its TMEM and returns.
//
// The same arithmetic as the CUDA-core kernels of lfsai.cu (BF16 products,
// FP32 sums) up to the summation order inside the tensor core.
//
// Training runs on the tensor cores too:
//  * k_backward_tc: per 128-row tile, the deltas d3 = (dL/do W4) .* (h3 > 0),
//    d2 = (d3 W3) .* (h2 > 0), d1 = (d2 W2) .* (h1 > 0) as three MMAs with
//    the transposed weights as B operands (K = 16, 64, 64), the deltas
//    rounded to BF16 as the next MMA's A operand and kept in FP32 for the
//    weight gradients;
//  * k_wgrad_tc: dW = sum_r d_r^T bf16(x_r) with the rows as the K
//    dimension: A = d^T (FOUT <= 64 of the 128 M rows used), B = x^T plus a
//    row of ones, so the bias gradient sum_r d_r comes out of the same MMA
//    as column FIN; each CTA accumulates its rows in TMEM and writes one
//    partial, summed in a fixed order afterwards.
#include <cuda_bf16.h>

#include "internal.cuh"
#include "lfsai.cuh"

namespace tnlb {
namespace tc {

constexpr int kRows = 128;     // rows per tile (MMA M)
constexpr int kTmemCols = 128;  // accumulator columns allocated per CTA (N=64 layers, N=16 output)
constexpr uint32_t kSpinLimit = 1u << 24;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor (tcgen05 format): start address, leading
// (K-direction core-matrix) byte offset, stride (8-row-group) byte offset,
// descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
   return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
          ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor, kind::f16: D FP32, A and B BF16, both K-major.
__host__ __device__ constexpr uint32_t instr_desc(int M, int N)
{
   return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// Byte offset of element (r, k) in a K-major core-matrix tile with KC
// 8-element chunks along K.
__device__ __forceinline__ uint32_t core_off(int r, int k, int KC)
{
   return (uint32_t)((((r >> 3) * KC + (k >> 3)) << 7) + ((r & 7) << 4) + ((k & 7) << 1));
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate)
{
   asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void commit(uint64_t* bar)
{
   asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                : "memory");
}

// Bounded wait for the mbarrier phase with parity `phase`; false on timeout.
__device__ __forceinline__ bool wait_bar(uint64_t* bar, uint32_t phase)
{
   const uint32_t a = smem_u32(bar);
   for (uint32_t it = 0; it < kSpinLimit; it++) {
      uint32_t ok;
      asm volatile(
         "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
         : "=r"(ok)
         : "r"(a), "r"(phase)
         : "memory");
      if (ok) return true;
   }
   return false;
}

__device__ __forceinline__ void ld16(uint32_t taddr, float (&v)[16])
{
   uint32_t r[16];
   asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
      "[%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
   for (int q = 0; q < 16; q++) v[q] = __uint_as_float(r[q]);
}

__device__ __forceinline__ void wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void store_bf16(uint8_t* base, uint32_t off, float v)
{
   *reinterpret_cast<__nv_bfloat16*>(base + off) = __float2bfloat16_rn(v);
}

struct Smem {
   alignas(1024) uint8_t a[kRows * kLfH * 2];  // layer input tile, 128 x 64 BF16 (layer 1 uses 128 x 32)
   alignas(1024) uint8_t w1[kLfH * kLfF * 2];  // 64 x 32
   alignas(1024) uint8_t w2[kLfH * kLfH * 2];  // 64 x 64
   alignas(1024) uint8_t w3[kLfH * kLfH * 2];
   alignas(1024) uint8_t w4[16 * kLfH * 2];    // 8 x 64 padded to 16 rows
   float b[3 * kLfH + 16];
   alignas(8) uint64_t bar;
   uint32_t taddr;
   int32_t fail;
};

// Forward pass of the network over n rows.  h1..h3 (n x 64, FP32 after ReLU)
// are written when non-null; o (n x 8) always.
__global__ void __launch_bounds__(kRows) k_forward_tc(const float* __restrict__ feat, int64_t n,
                                                      const float* __restrict__ wr, float* __restrict__ h1,
                                                      float* __restrict__ h2, float* __restrict__ h3,
                                                      float* __restrict__ o, int32_t* __restrict__ err)
{
   extern __shared__ uint8_t dyn[];
   Smem& S = *reinterpret_cast<Smem*>((reinterpret_cast<uintptr_t>(dyn) + 1023) & ~uintptr_t(1023));
   const int t = threadIdx.x, warp = t >> 5;
   // weights (BF16-rounded FP32 copies) into the core-matrix layout
   for (int e = t; e < kLfH * kLfF; e += kRows) store_bf16(S.w1, core_off(e / kLfF, e % kLfF, kLfF / 8), wr[kLfW1 + e]);
   for (int e = t; e < kLfH * kLfH; e += kRows) {
      store_bf16(S.w2, core_off(e / kLfH, e % kLfH, kLfH / 8), wr[kLfW2 + e]);
      store_bf16(S.w3, core_off(e / kLfH, e % kLfH, kLfH / 8), wr[kLfW3 + e]);
   }
   for (int e = t; e < 16 * kLfH; e += kRows) {
      const int r = e / kLfH, c = e % kLfH;
      store_bf16(S.w4, core_off(r, c, kLfH / 8), r < kLfK ? wr[kLfW4 + r * kLfH + c] : 0.f);
   }
   for (int e = t; e < kLfH; e += kRows) {
      S.b[e] = wr[kLfB1 + e];
      S.b[kLfH + e] = wr[kLfB2 + e];
      S.b[2 * kLfH + e] = wr[kLfB3 + e];
   }
   if (t < 16) S.b[3 * kLfH + t] = t < kLfK ? wr[kLfB4 + t] : 0.f;
   if (t == 0) {
      S.fail = 0;
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&S.bar)), "r"(1));
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
   }
   if (warp == 0) {
      asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&S.taddr)),
                   "r"(kTmemCols));
      asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
   }
   fence_before();
   __syncthreads();
   fence_after();
   const uint32_t tmem = S.taddr;
   const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
   const uint32_t a_addr = smem_u32(S.a);
   uint32_t phase = 0;
   bool ok = true;

   for (int64_t tile = blockIdx.x; ok && tile * kRows < n; tile += gridDim.x) {
      const int64_t row = tile * kRows + t;
      const bool live = row < n;
      // layer-1 input: features, BF16, K = 16
#pragma unroll
      for (int k = 0; k < kLfF; k++) store_bf16(S.a, core_off(t, k, kLfF / 8), live ? feat[row * kLfF + k] : 0.f);
      for (int layer = 0; layer < 4 && ok; layer++) {
         const int K = layer == 0 ? kLfF : kLfH;
         const int N = layer == 3 ? 16 : kLfH;
         const uint8_t* W = layer == 0 ? S.w1 : layer == 1 ? S.w2 : layer == 2 ? S.w3 : S.w4;
         fence_async_smem();
         fence_before();
         __syncthreads();
         if (t == 0) {
            fence_after();
            const uint32_t idesc = instr_desc(kRows, N);
            const uint32_t sbo = (uint32_t)(K / 8) * 128u;
            for (int kk = 0; kk < K / 16; kk++) {
               const uint64_t ad = smem_desc(a_addr + kk * 256u, 128u, sbo);
               const uint64_t bd = smem_desc(smem_u32(W) + kk * 256u, 128u, sbo);
               mma_bf16(tmem, ad, bd, idesc, kk > 0 ? 1u : 0u);
            }
            commit(&S.bar);
         }
         // every thread waits; the decision to go on is taken by the whole block
         const int mine = wait_bar(&S.bar, phase) ? 1 : 0;
         if (!__syncthreads_and(mine)) {
            ok = false;
            if (t == 0) S.fail = 1;
            break;
         }
         phase ^= 1u;
         fence_after();
         if (layer < 3) {
            float* hout = layer == 0 ? h1 : layer == 1 ? h2 : h3;
            const float* bias = S.b + layer * kLfH;
            for (int c0 = 0; c0 < kLfH; c0 += 16) {
               float v[16];
               ld16(tmem + lane_base + (uint32_t)c0, v);
               wait_ld();
#pragma unroll
               for (int q = 0; q < 16; q++) {
                  const float h = fmaxf(v[q] + bias[c0 + q], 0.f);
                  if (live && hout) hout[row * kLfH + c0 + q] = h;
                  store_bf16(S.a, core_off(t, c0 + q, kLfH / 8), h);
               }
            }
         }
         else {
            float v[16];
            ld16(tmem + lane_base, v);
            wait_ld();
            if (live)
#pragma unroll
               for (int q = 0; q < kLfK; q++) o[row * kLfK + q] = v[q] + S.b[3 * kLfH + q];
         }
      }
   }
   fence_before();
   __syncthreads();
   if (S.fail && t == 0) atomicExch(err, 1);
   if (warp == 0) {
      fence_after();
      asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
   }
}

struct SmemBack {
   alignas(1024) uint8_t a[kRows * kLfH * 2];  // delta tile, 128 x 64 BF16 (first MMA: 128 x 16)
   alignas(1024) uint8_t w4t[kLfH * 16 * 2];   // W4^T, 64 x 16 (K = outputs, 8 used)
   alignas(1024) uint8_t w3t[kLfH * kLfH * 2]; // W3^T, 64 x 64
   alignas(1024) uint8_t w2t[kLfH * kLfH * 2]; // W2^T
   alignas(8) uint64_t bar;
   uint32_t taddr;
   int32_t fail;
};

// Deltas of the three hidden layers for all rows (see the file comment).
__global__ void __launch_bounds__(kRows) k_backward_tc(const float* __restrict__ dout, int64_t n,
                                                       const float* __restrict__ wr, const float* __restrict__ h1,
                                                       const float* __restrict__ h2, const float* __restrict__ h3,
                                                       float* __restrict__ d1, float* __restrict__ d2,
                                                       float* __restrict__ d3, int32_t* __restrict__ err)
{
   extern __shared__ uint8_t dyn[];
   SmemBack& S = *reinterpret_cast<SmemBack*>((reinterpret_cast<uintptr_t>(dyn) + 1023) & ~uintptr_t(1023));
   const int t = threadIdx.x, warp = t >> 5;
   // B operands: element (n, k) = W[k][n], K-major core-matrix layout
   for (int e = t; e < kLfH * 16; e += kRows) {
      const int nn = e / 16, k = e % 16;
      store_bf16(S.w4t, core_off(nn, k, 2), k < kLfK ? wr[kLfW4 + k * kLfH + nn] : 0.f);
   }
   for (int e = t; e < kLfH * kLfH; e += kRows) {
      const int nn = e / kLfH, k = e % kLfH;
      store_bf16(S.w3t, core_off(nn, k, kLfH / 8), wr[kLfW3 + k * kLfH + nn]);
      store_bf16(S.w2t, core_off(nn, k, kLfH / 8), wr[kLfW2 + k * kLfH + nn]);
   }
   if (t == 0) {
      S.fail = 0;
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&S.bar)), "r"(1));
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
   }
   if (warp == 0) {
      asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&S.taddr)),
                   "r"(kTmemCols));
      asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
   }
   fence_before();
   __syncthreads();
   fence_after();
   const uint32_t tmem = S.taddr;
   const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
   const uint32_t a_addr = smem_u32(S.a);
   uint32_t phase = 0;
   bool ok = true;
   for (int64_t tile = blockIdx.x; ok && tile * kRows < n; tile += gridDim.x) {
      const int64_t row = tile * kRows + t;
      const bool live = row < n;
      // first A operand: dL/do (8 outputs) padded to K = 16
#pragma unroll
      for (int k = 0; k < 16; k++) store_bf16(S.a, core_off(t, k, 2), (live && k < kLfK) ? dout[row * kLfK + k] : 0.f);
      for (int layer = 3; layer >= 1 && ok; layer--) {
         const int K = layer == 3 ? 16 : kLfH;
         const uint8_t* W = layer == 3 ? S.w4t : layer == 2 ? S.w3t : S.w2t;
         fence_async_smem();
         fence_before();
         __syncthreads();
         if (t == 0) {
            fence_after();
            const uint32_t idesc = instr_desc(kRows, kLfH);
            const uint32_t sbo = (uint32_t)(K / 8) * 128u;
            for (int kk = 0; kk < K / 16; kk++) {
               const uint64_t ad = smem_desc(a_addr + kk * 256u, 128u, sbo);
               const uint64_t bd = smem_desc(smem_u32(W) + kk * 256u, 128u, sbo);
               mma_bf16(tmem, ad, bd, idesc, kk > 0 ? 1u : 0u);
            }
            commit(&S.bar);
         }
         const int mine = wait_bar(&S.bar, phase) ? 1 : 0;
         if (!__syncthreads_and(mine)) {
            ok = false;
            if (t == 0) S.fail = 1;
            break;
         }
         phase ^= 1u;
         fence_after();
         const float* hin = layer == 3 ? h3 : layer == 2 ? h2 : h1;
         float* dst = layer == 3 ? d3 : layer == 2 ? d2 : d1;
         for (int c0 = 0; c0 < kLfH; c0 += 16) {
            float v[16];
            ld16(tmem + lane_base + (uint32_t)c0, v);
            wait_ld();
#pragma unroll
            for (int q = 0; q < 16; q++) {
               const float d = (live && hin[row * kLfH + c0 + q] > 0.f) ? v[q] : 0.f;
               if (live) dst[row * kLfH + c0 + q] = d;
               store_bf16(S.a, core_off(t, c0 + q, kLfH / 8), d);
            }
         }
      }
   }
   fence_before();
   __syncthreads();
   if (S.fail && t == 0) atomicExch(err, 1);
   if (warp == 0) {
      fence_after();
      asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
   }
}

struct SmemWgrad {
   alignas(1024) uint8_t a[kRows * kRows * 2];        // d^T: 128 (M, outputs) x 128 (K, rows)
   alignas(1024) uint8_t b[(kLfH + 16) * kRows * 2];  // x^T and a row of ones: (FIN + 16) x 128
   alignas(8) uint64_t bar;
   uint32_t taddr;
   int32_t fail;
};

// Weight and bias gradient of one layer, one partial per CTA:
// partial[cta] = [dW (FOUT x FIN) | db (FOUT)] over rows
// [cta * rows_per_cta, (cta + 1) * rows_per_cta) (a multiple of 128).
template <int FIN, int FOUT>
__global__ void __launch_bounds__(kRows) k_wgrad_tc(const float* __restrict__ d, const float* __restrict__ x,
                                                    int64_t n, int64_t rows_per_cta, float* __restrict__ partial,
                                                    int32_t* __restrict__ err)
{
   constexpr int N = FIN + 16;  // x^T rows, then the ones row and padding
   static_assert(N % 16 == 0 && N <= 256 && FOUT <= kRows, "MMA shape");
   extern __shared__ uint8_t dyn[];
   SmemWgrad& S = *reinterpret_cast<SmemWgrad*>((reinterpret_cast<uintptr_t>(dyn) + 1023) & ~uintptr_t(1023));
   const int t = threadIdx.x, warp = t >> 5;
   // the M rows FOUT..127 of A and the padding rows of B stay zero; the
   // ones row of B is set once
   for (int e = t; e < kRows * kRows; e += kRows) {
      const int m = e / kRows, k = e % kRows;
      if (m >= FOUT) store_bf16(S.a, core_off(m, k, kRows / 8), 0.f);
   }
   for (int e = t; e < 16 * kRows; e += kRows) {
      const int nn = FIN + e / kRows, k = e % kRows;
      store_bf16(S.b, core_off(nn, k, kRows / 8), nn == FIN ? 1.f : 0.f);
   }
   if (t == 0) {
      S.fail = 0;
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&S.bar)), "r"(1));
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
   }
   if (warp == 0) {
      asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&S.taddr)),
                   "r"(kTmemCols));
      asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
   }
   fence_before();
   __syncthreads();
   fence_after();
   const uint32_t tmem = S.taddr;
   const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
   uint32_t phase = 0;
   bool ok = true;
   const int64_t r0 = (int64_t)blockIdx.x * rows_per_cta;
   const int64_t r1 = imin64(n, r0 + rows_per_cta);
   bool first = true;
   for (int64_t rb = r0; ok && rb < r1; rb += kRows) {
      // thread t stages row rb + t: its deltas into column t of A, its
      // inputs into column t of B (zero beyond the last row)
      const int64_t row = rb + t;
      const bool live = row < r1;
#pragma unroll 4
      for (int m = 0; m < FOUT; m++) store_bf16(S.a, core_off(m, t, kRows / 8), live ? d[row * FOUT + m] : 0.f);
#pragma unroll 4
      for (int c = 0; c < FIN; c++) store_bf16(S.b, core_off(c, t, kRows / 8), live ? x[row * FIN + c] : 0.f);
      if (!live) store_bf16(S.b, core_off(FIN, t, kRows / 8), 0.f);
      else store_bf16(S.b, core_off(FIN, t, kRows / 8), 1.f);
      fence_async_smem();
      fence_before();
      __syncthreads();
      if (t == 0) {
         fence_after();
         const uint32_t idesc = instr_desc(kRows, N);
         const uint32_t sbo = (uint32_t)(kRows / 8) * 128u;
         for (int kk = 0; kk < kRows / 16; kk++) {
            const uint64_t ad = smem_desc(smem_u32(S.a) + kk * 256u, 128u, sbo);
            const uint64_t bd = smem_desc(smem_u32(S.b) + kk * 256u, 128u, sbo);
            mma_bf16(tmem, ad, bd, idesc, (first && kk == 0) ? 0u : 1u);
         }
         commit(&S.bar);
      }
      first = false;
      const int mine = wait_bar(&S.bar, phase) ? 1 : 0;
      if (!__syncthreads_and(mine)) {
         ok = false;
         if (t == 0) S.fail = 1;
         break;
      }
      phase ^= 1u;
      fence_after();
   }
   if (ok) {
      // TMEM lane m holds dW row m (columns 0..FIN-1) and db[m] (column FIN)
      constexpr int NW = FOUT * FIN + FOUT;
      float* out = partial + (int64_t)blockIdx.x * NW;
      if (r0 >= r1) {
         for (int e = t; e < NW; e += kRows) out[e] = 0.f;
      }
      else if (warp * 32 < FOUT) {
         for (int c0 = 0; c0 < N; c0 += 16) {
            float v[16];
            ld16(tmem + lane_base + (uint32_t)c0, v);
            wait_ld();
            if (t < FOUT)
#pragma unroll
               for (int q = 0; q < 16; q++) {
                  const int c = c0 + q;
                  if (c < FIN)
                     out[t * FIN + c] = v[q];
                  else if (c == FIN)
                     out[FOUT * FIN + t] = v[q];
               }
         }
      }
   }
   fence_before();
   __syncthreads();
   if (S.fail && t == 0) atomicExch(err, 1);
   if (warp == 0) {
      fence_after();
      asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
   }
}

}  // namespace tc

size_t lfsai_tc_smem_bytes() { return sizeof(tc::Smem) + 1024; }

tnlb_status lfsai_forward_tc(const tnlb_lfsai* net, const float* feat, int64_t n, float* o, float* h1, float* h2,
                             float* h3, cudaStream_t st)
{
   static bool attr_set = false;
   const size_t smem = lfsai_tc_smem_bytes();
   if (!attr_set) {
      TNLB_CUDA_TRY(cudaFuncSetAttribute(tc::k_forward_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      attr_set = true;
   }
   DeviceBuffer err;
   TNLB_TRY_STATUS(err.alloc(sizeof(int32_t)));
   TNLB_CUDA_TRY(cudaMemsetAsync(err.ptr, 0, sizeof(int32_t), st));
   const int64_t tiles = (n + tc::kRows - 1) / tc::kRows;
   const unsigned grid = (unsigned)imin64(tiles, 148 * 4);
   tc::k_forward_tc<<<grid, tc::kRows, smem, st>>>(feat, n, net->wround.as<float>(), h1, h2, h3, o, err.as<int32_t>());
   TNLB_CHECK_LAUNCH();
   int32_t h = 0;
   TNLB_CUDA_TRY(cudaMemcpyAsync(&h, err.ptr, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
   TNLB_CUDA_TRY(cudaStreamSynchronize(st));
   TNLB_REQUIRE(h == 0, TNLB_ERR_TIMEOUT, "tensor-core network pass: an mbarrier wait timed out");
   return TNLB_OK;
}


namespace {

__global__ void k_sum_partials_tc(const float* __restrict__ partial, int blocks, int nw, float* __restrict__ gW,
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

template <int FIN, int FOUT>
tnlb_status wgrad_tc(const float* d, const float* x, int64_t n, float* gW, float* gb, int32_t* err, cudaStream_t st)
{
   static bool attr_set = false;
   const size_t smem = sizeof(tc::SmemWgrad) + 1024;
   if (!attr_set) {
      TNLB_CUDA_TRY(cudaFuncSetAttribute(tc::k_wgrad_tc<FIN, FOUT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem));
      attr_set = true;
   }
   const int64_t chunks = (n + tc::kRows - 1) / tc::kRows;
   const int64_t ctas = imin64(chunks, 148 * 4);
   const int64_t rows_per_cta = ((chunks + ctas - 1) / ctas) * tc::kRows;
   const int blocks = (int)((n + rows_per_cta - 1) / rows_per_cta);
   constexpr int NW = FOUT * FIN + FOUT;
   DeviceBuffer part;
   TNLB_TRY_STATUS(part.alloc(sizeof(float) * (size_t)blocks * NW));
   tc::k_wgrad_tc<FIN, FOUT><<<blocks, tc::kRows, smem, st>>>(d, x, n, rows_per_cta, part.as<float>(), err);
   TNLB_CHECK_LAUNCH();
   k_sum_partials_tc<<<(NW + 255) / 256, 256, 0, st>>>(part.as<float>(), blocks, NW, gW, gb, FOUT * FIN);
   TNLB_CHECK_LAUNCH();
   // the partial buffer is freed on return: wait for its readers
   TNLB_CUDA_TRY(cudaStreamSynchronize(st));
   return TNLB_OK;
}

}  // namespace

tnlb_status lfsai_backward_tc(tnlb_lfsai* net, const float* feat, int64_t n, const float* h1, const float* h2,
                              const float* h3, const float* dout, cudaStream_t st)
{
   static bool attr_set = false;
   const size_t smem = sizeof(tc::SmemBack) + 1024;
   if (!attr_set) {
      TNLB_CUDA_TRY(cudaFuncSetAttribute(tc::k_backward_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      attr_set = true;
   }
   DeviceBuffer d3, d2, d1, err;
   TNLB_TRY_STATUS(d3.alloc(sizeof(float) * n * kLfH));
   TNLB_TRY_STATUS(d2.alloc(sizeof(float) * n * kLfH));
   TNLB_TRY_STATUS(d1.alloc(sizeof(float) * n * kLfH));
   TNLB_TRY_STATUS(err.alloc(sizeof(int32_t)));
   TNLB_CUDA_TRY(cudaMemsetAsync(err.ptr, 0, sizeof(int32_t), st));
   const int64_t tiles = (n + tc::kRows - 1) / tc::kRows;
   const unsigned grid = (unsigned)imin64(tiles, 148 * 4);
   tc::k_backward_tc<<<grid, tc::kRows, smem, st>>>(dout, n, net->wround.as<float>(), h1, h2, h3, d1.as<float>(),
                                                    d2.as<float>(), d3.as<float>(), err.as<int32_t>());
   TNLB_CHECK_LAUNCH();
   float* gr = net->grad.as<float>();
   TNLB_TRY_STATUS(wgrad_tc<kLfH, kLfK>(dout, h3, n, gr + kLfW4, gr + kLfB4, err.as<int32_t>(), st));
   TNLB_TRY_STATUS(wgrad_tc<kLfH, kLfH>(d3.as<float>(), h2, n, gr + kLfW3, gr + kLfB3, err.as<int32_t>(), st));
   TNLB_TRY_STATUS(wgrad_tc<kLfH, kLfH>(d2.as<float>(), h1, n, gr + kLfW2, gr + kLfB2, err.as<int32_t>(), st));
   TNLB_TRY_STATUS(wgrad_tc<kLfF, kLfH>(d1.as<float>(), feat, n, gr + kLfW1, gr + kLfB1, err.as<int32_t>(), st));
   int32_t h = 0;
   TNLB_CUDA_TRY(cudaMemcpyAsync(&h, err.ptr, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
   TNLB_CUDA_TRY(cudaStreamSynchronize(st));
   TNLB_REQUIRE(h == 0, TNLB_ERR_TIMEOUT, "tensor-core network backward pass: an mbarrier wait timed out");
   return TNLB_OK;
}

}  // namespace tnlb
