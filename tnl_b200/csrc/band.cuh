// band.cuh -- products on a diagonal (DIA) copy with every operand staged in
// shared memory by bulk copies (cp.async.bulk, the TMA's one-dimensional
// form; no multicast), for the FP32 iterations of the reliable-update PCG.
//
// The diagonal kernels of compact.cuh read each row's D values and gather
// D inputs with ordinary loads.  Profiled on the 2048^2 5-point operator
// and its FSAI factors they ran at 28-47% of the DRAM bandwidth, their
// warps stalled on long-scoreboard loads: latency-bound, too few bytes in
// flight per SM.  Here a block works on tiles of kBandT consecutive rows.
// One thread issues, for the next tile, bulk copies of
//   * the D value runs of the tile's rows (contiguous in the DIA layout),
//   * for every input vector, one run per "band" -- a group of diagonals
//     whose offsets lie within kBandGap of each other (a 5-point operator
//     has three: -N; -1, 0, 1; +N) -- covering the inputs of all the
//     tile's rows on those diagonals, and
//   * for some kernels, the tile's own entries of vectors it updates,
// all completing on one mbarrier, while the block computes the current
// tile from the other of two stages.  Up to two stages of tens of KB are
// in flight per block, against a few KB for the register-staged kernels.
// A tile's rows are spread over the threads with a stride of the block
// size, so that the shared-memory reads of a warp are consecutive words.
// Each row sums the same terms in the same order as DiaRows / DiaRow1.
//
// Bulk copies need 16-byte-aligned addresses and sizes: the value pitch is
// a multiple of 8 rows, tiles start at multiples of kBandT, band runs are
// widened to multiples of 4 floats, and every vector read this way is
// allocated to a multiple of 4 entries (`npad`); the padding is read but
// never used.  Waits on the mbarrier are bounded: on a timeout the kernel
// records an error (the caller turns it into a breakdown) and stops after
// its copies in flight have landed, or have been given up on.
#pragma once

#include <cuda_fp16.h>

#include <cstdint>

#include "compact.cuh"

namespace tnlb {

constexpr int kBandT = 1024;       // rows of a tile
constexpr int kBandThreads = 256;  // threads of a block
constexpr int kBandGap = 16;       // diagonals closer than this share a band
constexpr int kBandRows = kBandT / kBandThreads;
constexpr long kBandSpin = 1L << 24;  // mbarrier polls before a wait gives up

// The plan of a banded product, built on the host and passed by value:
// the bands (band b covers offsets [lo[b], hi[b]]), the byte offsets of one
// stage's parts (the D value runs; per banded input vector k one run per
// band; the own-row runs), and per diagonal j the lower offset of its band
// and that band's run, so that the per-row loop reads only fixed
// parameter slots (no dynamically indexed arrays, no local memory).
struct BandPlan {
   int32_t D = 0, nb = 0;
   int32_t lo[8] = {}, hi[8] = {};
   uint32_t vals = 0, band[2][8] = {}, own[2] = {}, bytes = 0;
   int32_t dlo[8] = {};        // lo of diagonal j's band
   uint32_t dband[2][8] = {};  // its run for input k
   int32_t zlo = 0;            // the band of offset 0
   uint32_t zband[2] = {};
   bool zero = false;  // offset 0 among the diagonals
};

// The plan for ascending offsets o[0..D-1] (D <= 8), values of vbytes
// bytes, KB banded input vectors and KO own-row vectors (KB, KO <= 2).
inline BandPlan band_plan(const int32_t* o, int D, int vbytes, int KB, int KO)
{
   BandPlan P;
   P.D = D;
   int32_t of[8] = {};
   for (int j = 0; j < D; j++) {
      if (P.nb == 0 || o[j] - P.hi[P.nb - 1] >= kBandGap) {
         P.lo[P.nb] = P.hi[P.nb] = o[j];
         P.nb++;
      }
      else
         P.hi[P.nb - 1] = o[j];
      of[j] = P.nb - 1;
   }
   uint32_t off = (uint32_t)((D * kBandT * vbytes + 127) & ~127);
   for (int k = 0; k < KB; k++)
      for (int b = 0; b < P.nb; b++) {
         P.band[k][b] = off;
         // the run [floor4(i0 + lo), ceil4(i0 + T + hi)) holds at most
         // T + (hi - lo) + 6 entries
         const uint32_t span = (uint32_t)((kBandT + (P.hi[b] - P.lo[b]) + 8 + 3) & ~3);
         off += (span * 4 + 127) & ~127u;
      }
   for (int k = 0; k < KO; k++) {
      P.own[k] = off;
      off += kBandT * 4;
   }
   P.bytes = (off + 127) & ~127u;
   for (int j = 0; j < D; j++) {
      P.dlo[j] = P.lo[of[j]];
      for (int k = 0; k < KB; k++) P.dband[k][j] = P.band[k][of[j]];
      if (o[j] == 0) {
         P.zero = true;
         P.zlo = P.lo[of[j]];
         for (int k = 0; k < KB; k++) P.zband[k] = P.band[k][of[j]];
      }
   }
   return P;
}

// First entry of the run of a band with lower offset lo, for the tile at
// i0 (a multiple of 4, >= 0).
__device__ __forceinline__ int64_t band_start(int32_t lo, int64_t i0)
{
   const int64_t s = (i0 + lo) & ~(int64_t)3;
   return s < 0 ? 0 : s;
}

__device__ __forceinline__ uint32_t band_smem(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void band_bar_init(uint64_t* bar)
{
   asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(band_smem(bar)) : "memory");
}

__device__ __forceinline__ void band_expect(uint64_t* bar, uint32_t bytes)
{
   asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(band_smem(bar)), "r"(bytes)
                : "memory");
}

__device__ __forceinline__ void band_copy(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
   asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   band_smem(dst)),
                "l"(src), "r"(bytes), "r"(band_smem(bar))
                : "memory");
}

// Polls the mbarrier's phase `parity` at most kBandSpin times.
__device__ __forceinline__ bool band_wait(uint64_t* bar, uint32_t parity)
{
   const uint32_t a = band_smem(bar);
   for (long it = 0; it < kBandSpin; it++) {
      uint32_t done;
      asm volatile(
         "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
         : "=r"(done)
         : "r"(a), "r"(parity)
         : "memory");
      if (done) return true;
   }
   return false;
}

// *flag read once per block (thread 0, broadcast): a flag that another
// block may raise while this one starts must not split the block.
__device__ __forceinline__ bool band_block_flag(const int32_t* flag)
{
   __shared__ int32_t s_flag;
   if (threadIdx.x == 0) s_flag = flag ? *reinterpret_cast<const volatile int32_t*>(flag) : 0;
   __syncthreads();
   return s_flag != 0;
}

// Issues the copies of the tile at i0 into stage `st` (one thread).  The
// band loop runs over all 8 slots with a guard, so that the plan's arrays
// are read at fixed indexes.
template <typename TV, int D, int KB, int KO>
__device__ __forceinline__ void band_issue(unsigned char* st, uint64_t* bar, const BandPlan& P, const TV* vals,
                                           int64_t pitch, const float* const (&bin)[KB > 0 ? KB : 1],
                                           const float* const (&oin)[KO > 0 ? KO : 1], int64_t npad, int64_t i0)
{
   const int64_t vrows = pitch - i0 < kBandT ? pitch - i0 : kBandT;
   const int64_t orows = npad - i0 < kBandT ? npad - i0 : kBandT;
   int64_t gs[8], ge[8];
   uint32_t total = (uint32_t)(D * vrows * (int64_t)sizeof(TV)) + (uint32_t)(KO * orows * 4);
#pragma unroll
   for (int b = 0; b < 8; b++) {
      gs[b] = band_start(P.lo[b], i0);
      const int64_t e = (i0 + kBandT + P.hi[b] + 3) & ~(int64_t)3;
      ge[b] = b < P.nb ? (e > npad ? npad : e) : 0;
      if (ge[b] > gs[b]) total += (uint32_t)(KB * (ge[b] - gs[b]) * 4);
   }
   band_expect(bar, total);
#pragma unroll
   for (int j = 0; j < D; j++)
      band_copy(st + P.vals + (size_t)j * kBandT * sizeof(TV), vals + (int64_t)j * pitch + i0,
                (uint32_t)(vrows * sizeof(TV)), bar);
#pragma unroll
   for (int k = 0; k < KB; k++)
#pragma unroll
      for (int b = 0; b < 8; b++)
         if (ge[b] > gs[b]) band_copy(st + P.band[k][b], bin[k] + gs[b], (uint32_t)((ge[b] - gs[b]) * 4), bar);
#pragma unroll
   for (int k = 0; k < KO; k++) band_copy(st + P.own[k], oin[k] + i0, (uint32_t)(orows * 4), bar);
}

// The tile loop: stage s of tile k, the next tile's copies issued before
// the current one is computed.  tile(i0, stage) computes a tile.  Returns
// false, in every thread, after a wait gave up (the block then stops
// taking tiles).
template <typename TV, int D, int KB, int KO, typename Tile>
__device__ __forceinline__ bool band_loop(unsigned char* smem, uint64_t* bars, const BandPlan& P, const TV* vals,
                                          int64_t pitch, const float* const (&bin)[KB > 0 ? KB : 1],
                                          const float* const (&oin)[KO > 0 ? KO : 1], int64_t n, int64_t npad,
                                          Tile&& tile)
{
   const int64_t tiles = (n + kBandT - 1) / kBandT;
   if (threadIdx.x == 0) {
      band_bar_init(&bars[0]);
      band_bar_init(&bars[1]);
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
   }
   __syncthreads();
   int64_t t = blockIdx.x;
   if (threadIdx.x == 0 && t < tiles)
      band_issue<TV, D, KB, KO>(smem, &bars[0], P, vals, pitch, bin, oin, npad, t * kBandT);
   uint32_t phase[2] = {0u, 0u};
   bool ok = true;
   for (int k = 0; t < tiles; k++, t += gridDim.x) {
      const int s = k & 1;
      const int64_t next = t + gridDim.x;
      const bool issued_next = next < tiles;
      if (issued_next && threadIdx.x == 0) {
         // the stage was last read by the generic proxy (the tile before)
         asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
         band_issue<TV, D, KB, KO>(smem + (size_t)(s ^ 1) * P.bytes, &bars[s ^ 1], P, vals, pitch, bin, oin, npad,
                                   next * kBandT);
      }
      // every thread polls; the block goes on only when all saw the phase
      if (!__syncthreads_and(band_wait(&bars[s], phase[s]) ? 1 : 0)) {
         // let the other stage's copies land (or give up on them) before
         // the block's shared memory is released
         if (issued_next && threadIdx.x == 0) band_wait(&bars[s ^ 1], phase[s ^ 1]);
         ok = false;
         break;
      }
      phase[s] ^= 1u;
      tile(t * kBandT, smem + (size_t)s * P.bytes);
      __syncthreads();
   }
   __syncthreads();
   return ok;
}

// Blocks of a band kernel with `smem` bytes of dynamic shared memory kept
// resident on the device, at most one per tile and at most max_blocks.
// Raises the kernel's dynamic shared memory limit first.
inline unsigned band_grid(const void* kernel, size_t smem, int64_t n, int max_blocks)
{
   int dev = 0, sms = 148, occ = 0;
   if (cudaGetDevice(&dev) != cudaSuccess ||
       cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
      sms = 148;
   cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
   if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, kBandThreads, smem) != cudaSuccess || occ < 1) {
      cudaGetLastError();
      occ = 1;
   }
   int64_t g = (n + kBandT - 1) / kBandT;
   if (g > (int64_t)occ * sms) g = (int64_t)occ * sms;
   if (g > max_blocks) g = max_blocks;
   return (unsigned)(g < 1 ? 1 : g);
}

// The staged operands of one tile.
template <typename TV>
struct BandStage {
   const unsigned char* st;
   const BandPlan* P;
   int64_t i0;
   __device__ __forceinline__ float val(int j, int rl) const
   {
      return rel_to_f(reinterpret_cast<const TV*>(st + P->vals)[(size_t)j * kBandT + rl]);
   }
   // input vector k at column c on diagonal j (c inside its band's run)
   __device__ __forceinline__ float in(int k, int j, int64_t c) const
   {
      return reinterpret_cast<const float*>(st + P->dband[k][j])[c - band_start(P->dlo[j], i0)];
   }
   // input vector k at the own row i (the band of offset 0)
   __device__ __forceinline__ float self(int k, int64_t i) const
   {
      return reinterpret_cast<const float*>(st + P->zband[k])[i - band_start(P->zlo, i0)];
   }
   __device__ __forceinline__ float own(int k, int rl) const
   {
      return reinterpret_cast<const float*>(st + P->own[k])[rl];
   }
};

}  // namespace tnlb
