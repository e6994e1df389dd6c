// band.cuh -- products on a diagonal (DIA) copy with every operand staged in
// shared memory by bulk copies (cp.async.bulk, the TMA's one-dimensional
// form; no multicast), for the FP32 iterations of the reliable-update PCG:
// the two FSAI factor products of an iteration when the factors have more
// than 5 diagonals (the level-1 pattern of a 5-point operator has 7).
//
// The diagonal kernels of compact.cuh read each row's D values and gather
// D inputs with ordinary loads.  Profiled on the 2048^2 5-point operator
// and its FSAI factors they ran at 28-47% of the DRAM bandwidth, their
// warps stalled on long-scoreboard loads: latency-bound, too few bytes in
// flight per SM.  Here a block works on tiles of kBandT consecutive rows
// held in up to kBandStages shared-memory stages.  A producer warp issues,
// for each tile, bulk copies of
//   * the D value runs of the tile's rows (contiguous in the DIA layout),
//   * for every input vector, one run per "band" -- a group of diagonals
//     whose offsets lie within kBandGap of each other (a 5-point operator
//     has three: -N; -1, 0, 1; +N) -- covering the inputs of all the
//     tile's rows on those diagonals, and
//   * for some kernels, the tile's own entries of vectors it updates,
// all completing on the stage's "full" mbarrier; eight consumer warps wait
// on it, compute the tile and release the stage on its "empty" mbarrier,
// which the producer waits on before it refills the stage.  No block-wide
// barrier separates the tiles: with two blocks of 2-3 stages of 30-40 KB
// per SM, about 100 KB are in flight per SM (a microbenchmark of this
// scheme streamed 6.3-6.7 TB/s out of DRAM).  A tile's rows are spread
// over the consumer threads with a stride of their count, so that the
// shared-memory reads of a warp are consecutive words.
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
#include "internal.cuh"
#include "reduce.cuh"

namespace tnlb {

constexpr int kBandT = 1024;                    // rows of a tile
constexpr int kBandThreads = 256;               // consumer threads of a block (8 warps)
constexpr int kBandBlock = kBandThreads + 32;   // and one producer warp
constexpr int kBandStages = 4;                  // at most this many tiles a block holds
constexpr uint32_t kBandSmem = 110 * 1024;      // stage bytes a block may take (two blocks per SM)
constexpr int kBandGap = 16;                    // diagonals closer than this share a band
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
   uint32_t vals = 0, band[2][8] = {}, own[2] = {}, ownd[1] = {}, bytes = 0;
   int32_t dlo[8] = {};        // lo of diagonal j's band
   uint32_t dband[2][8] = {};  // its run for input k
   int32_t zlo = 0;            // the band of offset 0
   uint32_t zband[2] = {};
   bool zero = false;  // offset 0 among the diagonals
   int32_t minlo = 0, maxhi = 0;  // the smallest and largest offsets
   // interior tiles (no band run clipped at row 0): the byte offset, from
   // the stage, of input k on diagonal j at the tile's row 0, and of input
   // k at the own row 0; independent of the tile
   uint32_t xoff[2][8] = {}, selfoff[2] = {};
   int32_t stages = 2;  // stages a block holds (<= kBandStages)
};

// The plan for ascending offsets o[0..D-1] (D <= 8), values of vbytes
// bytes, KB banded input vectors, KO own-row FP32 vectors and KD own-row
// FP64 vectors (KB, KO <= 2, KD <= 1).
inline BandPlan band_plan(const int32_t* o, int D, int vbytes, int KB, int KO, int KD = 0)
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
   for (int k = 0; k < KD; k++) {
      P.ownd[k] = off;
      off += kBandT * 8;
   }
   P.bytes = (off + 127) & ~127u;
   P.minlo = D > 0 ? o[0] : 0;
   P.maxhi = D > 0 ? o[D - 1] : 0;
   for (int j = 0; j < D; j++) {
      P.dlo[j] = P.lo[of[j]];
      for (int k = 0; k < KB; k++) {
         P.dband[k][j] = P.band[k][of[j]];
         // run start i0 + (lo & ~3) when i0 + lo >= 0 (i0 a multiple of 4)
         P.xoff[k][j] = P.band[k][of[j]] + 4u * (uint32_t)(o[j] - (P.lo[of[j]] & ~3));
      }
      if (o[j] == 0) {
         P.zero = true;
         P.zlo = P.lo[of[j]];
         for (int k = 0; k < KB; k++) {
            P.zband[k] = P.band[k][of[j]];
            P.selfoff[k] = P.band[k][of[j]] + 4u * (uint32_t)(-(P.lo[of[j]] & ~3));
         }
      }
   }
   const uint32_t fit = kBandSmem / (P.bytes > 0 ? P.bytes : 1);
   P.stages = (int32_t)(fit < 2 ? 2 : fit > (uint32_t)kBandStages ? (uint32_t)kBandStages : fit);
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
template <typename TV, int D, int KB, int KO, int KD>
__device__ __forceinline__ void band_issue(unsigned char* st, uint64_t* bar, const BandPlan& P, const TV* vals,
                                           int64_t pitch, const float* const (&bin)[KB > 0 ? KB : 1],
                                           const float* const (&oin)[KO > 0 ? KO : 1],
                                           const double* const (&din)[KD > 0 ? KD : 1], int64_t npad, int64_t i0)
{
   const int64_t vrows = pitch - i0 < kBandT ? pitch - i0 : kBandT;
   const int64_t orows = npad - i0 < kBandT ? npad - i0 : kBandT;
   int64_t gs[8], ge[8];
   uint32_t total =
      (uint32_t)(D * vrows * (int64_t)sizeof(TV)) + (uint32_t)(KO * orows * 4) + (uint32_t)(KD * orows * 8);
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
#pragma unroll
   for (int k = 0; k < KD; k++) band_copy(st + P.ownd[k], din[k] + i0, (uint32_t)(orows * 8), bar);
}

__device__ __forceinline__ void band_arrive(uint64_t* bar)
{
   asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(band_smem(bar)) : "memory");
}

// The tile loop.  Warp kBandThreads / 32 (lane 0) produces: tile k goes to
// stage k % kBandStages once the consumers released the tile before it in
// that stage.  The other warps consume: wait for the stage, tile(i0,
// stage), release it.  Returns false in every thread after a wait gave up;
// the producer then waits (bounded) for its copies still in flight before
// the block's shared memory is released.
template <typename TV, int D, int KB, int KO, int KD, typename Tile>
__device__ __forceinline__ bool band_loop(unsigned char* smem, uint64_t* full, uint64_t* empty, const BandPlan& P,
                                          const TV* vals, int64_t pitch, const float* const (&bin)[KB > 0 ? KB : 1],
                                          const float* const (&oin)[KO > 0 ? KO : 1],
                                          const double* const (&din)[KD > 0 ? KD : 1], int64_t n, int64_t npad,
                                          Tile&& tile)
{
   const int64_t tiles = (n + kBandT - 1) / kBandT;
   const int S = P.stages;
   const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
   if (threadIdx.x == 0) {
      for (int s = 0; s < S; s++) {
         band_bar_init(&full[s]);
         asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(band_smem(&empty[s])), "r"(kBandThreads / 32)
                      : "memory");
      }
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
   }
   __syncthreads();
   bool ok = true;
   if (warp == kBandThreads / 32) {
      if (lane == 0) {
         int64_t k = 0;  // tiles issued
         for (int64_t t = blockIdx.x; t < tiles; t += gridDim.x, k++) {
            const int s = (int)(k % S);
            if (k >= S && !band_wait(&empty[s], (uint32_t)((k / S - 1) & 1))) {
               ok = false;
               break;
            }
            // the stage was last read by the generic proxy
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            band_issue<TV, D, KB, KO, KD>(smem + (size_t)s * P.bytes, &full[s], P, vals, pitch, bin, oin, din,
                                          npad, t * kBandT);
         }
         if (!ok)  // the last tile issued to each stage: k - 1, k - 2, ...
            for (int64_t q = k - 1; q >= 0 && q >= k - S; q--) band_wait(&full[q % S], (uint32_t)((q / S) & 1));
      }
   }
   else {
      int64_t k = 0;
      for (int64_t t = blockIdx.x; t < tiles; t += gridDim.x, k++) {
         const int s = (int)(k % S);
         if (!__all_sync(0xffffffffu, band_wait(&full[s], (uint32_t)((k / S) & 1)))) {
            ok = false;
            break;
         }
         tile(t * kBandT, smem + (size_t)s * P.bytes);
         __syncwarp();
         if (lane == 0) band_arrive(&empty[s]);
      }
   }
   return __syncthreads_and(ok ? 1 : 0) != 0;
}

// Block and grid sums of the band kernels (any block size): as
// publish_and_arrive / gather_totals of reduce.cuh.
template <int K>
__device__ __forceinline__ bool band_publish(const double (&v)[K], RedWork w)
{
   __shared__ double s_ws[K][kBandBlock / 32];
   __shared__ bool s_last;
   const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
   for (int k = 0; k < K; k++) {
      const double x = warp_sum(v[k]);
      if (lane == 0) s_ws[k][wid] = x;
   }
   __syncthreads();
   if (threadIdx.x == 0) {
#pragma unroll
      for (int k = 0; k < K; k++) {
         double r = 0.0;
         for (int q = 0; q < (int)(blockDim.x >> 5); q++) r += s_ws[k][q];
         w.partials[(size_t)k * kRedMaxBlocks + blockIdx.x] = r;
      }
      __threadfence();
      const unsigned t = atomicAdd(w.counter, 1u);
      s_last = (t == gridDim.x - 1);
   }
   __syncthreads();
   return s_last;
}

template <int K>
__device__ __forceinline__ void band_totals(double (&out)[K], RedWork w)
{
   __shared__ double s_ws[K][kBandBlock / 32];
   const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
   for (int k = 0; k < K; k++) {
      double v = 0.0;
      for (unsigned i = threadIdx.x; i < gridDim.x; i += blockDim.x)
         v += __ldcg(w.partials + (size_t)k * kRedMaxBlocks + i);
      v = warp_sum(v);
      if (lane == 0) s_ws[k][wid] = v;
   }
   __syncthreads();
   if (threadIdx.x == 0) {
#pragma unroll
      for (int k = 0; k < K; k++) {
         double r = 0.0;
         for (int q = 0; q < (int)(blockDim.x >> 5); q++) r += s_ws[k][q];
         out[k] = r;
      }
      *w.counter = 0;
   }
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
   if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, kBandBlock, smem) != cudaSuccess || occ < 1) {
      cudaGetLastError();
      occ = 1;
   }
   int64_t g = (n + kBandT - 1) / kBandT;
   if (g > (int64_t)occ * sms) g = (int64_t)occ * sms;
   if (g > max_blocks) g = max_blocks;
   return (unsigned)(g < 1 ? 1 : g);
}

// Per-tile pointers into a stage, at this thread's first row (the tile's
// row threadIdx.x; its rows q follow at + q * kBandThreads): the value run
// of diagonal 0 (diagonal j at + j * kBandT), input k on diagonal j, and
// input k at the own row.  `interior`: every column of the tile's rows lies
// in [0, n) and the tile is full, so no row or column needs a check.  The
// pointers are formed once per tile; each tap is then one shared-memory
// load at a fixed offset.
template <typename TV, int D, int KB>
struct BandPtrs {
   const TV* v;
   const float* x[KB > 0 ? KB : 1][D];
   const float* self[KB > 0 ? KB : 1];
   const float* own[2];
   const double* ownd;
   bool interior;
   __device__ __forceinline__ BandPtrs(const unsigned char* st, const BandPlan& P, const DiaOffsets& o, int64_t i0,
                                       int64_t n)
   {
      interior = i0 + P.minlo >= 0 && i0 + kBandT + P.maxhi <= n && i0 + kBandT <= n;
      const unsigned char* me = st + 4 * threadIdx.x;
      v = reinterpret_cast<const TV*>(st + P.vals) + threadIdx.x;
      if (interior) {
#pragma unroll
         for (int k = 0; k < KB; k++) {
#pragma unroll
            for (int j = 0; j < D; j++) x[k][j] = reinterpret_cast<const float*>(me + P.xoff[k][j]);
            self[k] = reinterpret_cast<const float*>(me + P.selfoff[k]);
         }
      }
      else {
#pragma unroll
         for (int k = 0; k < KB; k++) {
#pragma unroll
            for (int j = 0; j < D; j++)
               x[k][j] = reinterpret_cast<const float*>(st + P.dband[k][j]) +
                         (int32_t)(i0 + o.o[j] - band_start(P.dlo[j], i0)) + (int32_t)threadIdx.x;
            self[k] = reinterpret_cast<const float*>(st + P.zband[k]) + (int32_t)(i0 - band_start(P.zlo, i0)) +
                      (int32_t)threadIdx.x;
         }
      }
      own[0] = reinterpret_cast<const float*>(me + P.own[0]);
      own[1] = reinterpret_cast<const float*>(me + P.own[1]);
      ownd = reinterpret_cast<const double*>(st + P.ownd[0]) + threadIdx.x;
   }
};

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
