// spmv_csr.cu -- y = alpha*A*x + beta*y for CSR (and AdaptiveCSR) segments.
//
// Kernels (the names of Algorithms/SegmentsReductionKernels and the
// ThreadsToSegmentsMapping of Segments/LaunchConfiguration.h):
//  * scalar   -- one thread per row (Fixed, TPS 1; ReducingOperations_CSR.h:33-77)
//  * vector   -- G = 2..32 lanes per row, shuffle reduction
//                (reduceSegmentsCSRVariableVectorKernel, ReducingKernels_CSR.h:63-118)
//  * block    -- 64/128/256 threads per row through shared memory
//                (reduceSegmentsCSRLightMultivectorKernel, :120-189)
//  * light    -- G chosen from the mean row length
//                (LaunchConfigurationSetter_LightCSR.h:30-58)
//  * adaptive -- AdaptiveCSR STREAM / VECTOR / LONG block descriptors
//                (ReducingKernels_AdaptiveCSR.h:16-134)
//  * tile     -- the default: nnz-balanced merge-path tiles.  The merge of
//                the row-end offsets with the nonzero indices is cut into
//                tiles of 256 items (rows + nonzeros), one per warp, so that
//                every warp does the same work whatever the row-length
//                distribution (Merrill & Garland, "Merge-based parallel
//                sparse matrix-vector multiplication", SC16).  A warp keeps
//                its tile's products in registers, marks the rows ending in
//                the tile in a bit mask and sums rows with segmented shuffle
//                scans.  A row split between tiles leaves a partial sum per
//                tile in a carry array; a second small kernel adds them (in
//                tile order, so results are deterministic).  The tile
//                coordinates are computed once per matrix, when the
//                segments are built.
#include <climits>

#include "internal.cuh"
#include "reduce.cuh"

namespace tnlb {
namespace {

// Sum of v[k] x[c[k]] over k = k0, k0 + stride, ... < k1 for one lane, four
// entries loaded before any is used (four independent chains in flight).
template <typename Real>
__device__ __forceinline__ Real strided_dot(const int32_t* __restrict__ cols, const Real* __restrict__ vals,
                                            const Real* __restrict__ x, int32_t k0, int32_t k1, int32_t stride)
{
   Real s = 0;
   int32_t k = k0;
   for (; k + 3 * stride < k1; k += 4 * stride) {
      int32_t c[4];
      Real v[4];
#pragma unroll
      for (int u = 0; u < 4; u++) {
         c[u] = ld_stream(cols + k + u * stride);
         v[u] = ld_stream(vals + k + u * stride);
      }
#pragma unroll
      for (int u = 0; u < 4; u++)
         if (c[u] >= 0) s += v[u] * ld_gather(x + c[u]);
   }
   for (; k < k1; k += stride) {
      const int32_t c = ld_stream(cols + k);
      const Real v = ld_stream(vals + k);
      if (c >= 0) s += v * ld_gather(x + c);
   }
   return s;
}

// ------------------------------------------------------------- scalar

template <typename Real>
__global__ void k_csr_scalar(const int32_t* __restrict__ rowptr, const int32_t* __restrict__ cols,
                             const Real* __restrict__ vals, const Real* __restrict__ x, Real* __restrict__ y,
                             int32_t begin, int32_t end, Real alpha, Real beta)
{
   const int64_t row = begin + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (row >= end) return;
   keep(y, (int32_t)row, strided_dot(cols, vals, x, rowptr[row], rowptr[row + 1], 1), alpha, beta);
}

// ------------------------------------------------- vector (G lanes/row)

template <typename Real, int G>
__global__ void k_csr_vector(const int32_t* __restrict__ rowptr, const int32_t* __restrict__ cols,
                             const Real* __restrict__ vals, const Real* __restrict__ x, Real* __restrict__ y,
                             int32_t begin, int32_t end, Real alpha, Real beta)
{
   const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   const int64_t row = begin + gid / G;
   const int lane = (int)(gid % G);
   Real sum = 0;
   if (row < end) sum = strided_dot(cols, vals, x, rowptr[row] + lane, rowptr[row + 1], G);
   sum = group_sum<G>(sum);
   if (row < end && lane == 0) keep(y, (int32_t)row, sum, alpha, beta);
}

// ---------------------------------------- block (64/128/256 threads/row)

template <typename Real, int G>
__global__ void k_csr_block(const int32_t* __restrict__ rowptr, const int32_t* __restrict__ cols,
                            const Real* __restrict__ vals, const Real* __restrict__ x, Real* __restrict__ y,
                            int32_t begin, int32_t end, Real alpha, Real beta)
{
   constexpr int kRowsPerBlock = 256 / G;
   constexpr int kWarpsPerRow = G / 32;
   __shared__ Real part[8];
   const int r_in_block = threadIdx.x / G;
   const int t = threadIdx.x % G;
   const int64_t row = begin + (int64_t)blockIdx.x * kRowsPerBlock + r_in_block;
   Real sum = 0;
   if (row < end) sum = strided_dot(cols, vals, x, rowptr[row] + t, rowptr[row + 1], G);
   sum = warp_sum(sum);
   if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = sum;
   __syncthreads();
   if (t == 0 && row < end) {
      Real s = 0;
      for (int w = 0; w < kWarpsPerRow; w++) s += part[r_in_block * kWarpsPerRow + w];
      keep(y, (int32_t)row, s, alpha, beta);
   }
}

// ------------------------------------------------------------ adaptive

template <typename Real>
struct AcsrParams {
   static constexpr int kStreamPerWarp = (24576 / (int)sizeof(Real)) / 8;
};

template <typename Real>
__global__ void __launch_bounds__(256) k_csr_adaptive(const tnlb_acsr_block* __restrict__ blocks, int64_t count,
                                                      const int32_t* __restrict__ rowptr,
                                                      const int32_t* __restrict__ cols, const Real* __restrict__ vals,
                                                      const Real* __restrict__ x, Real* __restrict__ y, Real alpha,
                                                      Real beta)
{
   constexpr int S = AcsrParams<Real>::kStreamPerWarp;
   __shared__ Real stream_buf[8][S];
   __shared__ Real long_part[8];
   const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
   const int64_t w = (int64_t)blockIdx.x * 8 + wib;
   const bool active = w < count;
   tnlb_acsr_block d{};
   if (active) d = blocks[w];
   if (active && d.type == 1) {  // STREAM: many short rows, staged per warp
      // the block's entries 12 per lane and pass (FP64: the whole block in
      // one pass), every load and then every x gather issued before any is
      // used: 3x the gathers in flight of a 4-wide loop, which left the
      // kernel at a third of the tile kernel's rate on power-law rows
      constexpr int U = 12;
      const int32_t first = d.first_segment;
      const int32_t b = rowptr[first];
      for (int32_t k = lane; k < d.block_size; k += 32 * U) {
         int32_t c[U];
         Real v[U], g[U];
#pragma unroll
         for (int u = 0; u < U; u++) {
            c[u] = -1;
            v[u] = Real(0);
            if (k + 32 * u < d.block_size) {
               c[u] = ld_stream(cols + b + k + 32 * u);
               v[u] = ld_stream(vals + b + k + 32 * u);
            }
         }
#pragma unroll
         for (int u = 0; u < U; u++) g[u] = c[u] >= 0 ? ld_gather(x + c[u]) : Real(0);
#pragma unroll
         for (int u = 0; u < U; u++)
            if (k + 32 * u < d.block_size) stream_buf[wib][k + 32 * u] = v[u] * g[u];
      }
      __syncwarp();
      for (int32_t r = first + lane; r < first + d.segments_in_block; r += 32) {
         Real s = 0;
         const int32_t e = rowptr[r + 1] - b;
         for (int32_t k = rowptr[r] - b; k < e; k++) s += stream_buf[wib][k];
         keep(y, r, s, alpha, beta);
      }
   }
   else if (active && d.type == 2) {  // VECTOR: one row per warp
      const int32_t r = d.first_segment;
      const int32_t b = rowptr[r], e = b + d.block_size;
      Real s = strided_dot(cols, vals, x, b + lane, e, 32);
      s = warp_sum(s);
      if (lane == 0) keep(y, r, s, alpha, beta);
   }
   else if (active && d.type == 0) {  // LONG: several warps of this block per row
      const int32_t r = d.first_segment;
      const int32_t b = rowptr[r], e = rowptr[r + 1];
      Real s = strided_dot(cols, vals, x, b + lane + 32 * d.warp_idx, e, 32 * d.warps_count);
      s = warp_sum(s);
      if (lane == 0) long_part[wib] = s;
   }
   __syncthreads();
   if (active && d.type == 0 && d.warp_idx == 0 && lane == 0) {
      Real s = 0;
      for (int k = 0; k < d.warps_count; k++) s += long_part[wib + k];
      keep(y, d.first_segment, s, alpha, beta);
   }
}

// ------------------------------------------------------------ short rows

// One thread per row for matrices whose rows hold at most L entries
// (stencils, FSAI factors): all of a row's loads are issued before any is
// used; consecutive threads read consecutive rows, so a warp's loads of
// entry j share cache lines with those of entry j-1.  Sums in entry order.
// Grid-stride: a matrix of a few resident waves runs on the resident blocks
// only (no ramp of block launches), a larger one one row per thread.
template <typename Real, int L>
__global__ void __launch_bounds__(256) k_csr_short(const int32_t* __restrict__ rowptr, const int32_t* __restrict__ cols,
                                                   const Real* __restrict__ vals, const Real* __restrict__ x,
                                                   Real* __restrict__ y, int32_t n, Real alpha, Real beta,
                                                   const int32_t* __restrict__ skip)
{
   if (skip && *skip) return;
   for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
      const int32_t b = rowptr[r], e = rowptr[r + 1];
      int32_t c[L];
      Real v[L];
#pragma unroll
      for (int j = 0; j < L; j++) {
         c[j] = -1;
         v[j] = Real(0);
         if (b + j < e) {
            c[j] = __ldg(cols + b + j);
            v[j] = __ldg(vals + b + j);
         }
      }
      Real s = Real(0);
#pragma unroll
      for (int j = 0; j < L; j++)
         if (c[j] >= 0) s += v[j] * __ldg(x + c[j]);
      keep(y, (int32_t)r, s, alpha, beta);
   }
}

// k_csr_short with the dot product (x, y) of the product's input and output
// fused into it (the (p, A p) of CG): a grid-stride loop over rows on at most
// kRedMaxBlocks blocks, each block's sum of x[r] * y[r] published, the last
// block to arrive adding them in block order (deterministic) into *dot_out.
// With `self`, the sum is (y, y) instead (the (r, G^T G r) = |G r|^2 of an
// FSAI application).  Values TV, input TX, output TY (mixed storage: FP32
// values with FP64 vectors); rows are summed in TX.  Needs alpha = 1,
// beta = 0.
template <typename TV, typename TX, typename TY, int L, int R>
__global__ void __launch_bounds__(256) k_csr_short_dot(const int32_t* __restrict__ rowptr,
                                                       const int32_t* __restrict__ cols, const TV* __restrict__ vals,
                                                       const TX* __restrict__ x, TY* __restrict__ y, int32_t n,
                                                       RedWork w, double* __restrict__ dot_out,
                                                       const int32_t* __restrict__ skip, int self)
{
   if (skip && *skip) return;  // every block returns: no ticket is taken
   double d = 0.0;
   const int64_t stride = (int64_t)gridDim.x * blockDim.x;
   // R rows per thread and pass (r0 + k * stride), all their loads issued
   // before any is used: R times the loads in flight of one row
   for (int64_t r0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r0 < n; r0 += R * stride) {
      int32_t b[R], e[R];
#pragma unroll
      for (int k = 0; k < R; k++) {
         const int64_t r = r0 + k * stride;
         b[k] = r < n ? rowptr[r] : 0;
         e[k] = r < n ? rowptr[r + 1] : 0;
      }
      int32_t c[R][L];
      TV v[R][L];
#pragma unroll
      for (int k = 0; k < R; k++)
#pragma unroll
         for (int j = 0; j < L; j++) {
            c[k][j] = -1;
            v[k][j] = TV(0);
            if (b[k] + j < e[k]) {
               c[k][j] = __ldg(cols + b[k] + j);
               v[k][j] = __ldg(vals + b[k] + j);
            }
         }
      TX s[R];
#pragma unroll
      for (int k = 0; k < R; k++) {
         s[k] = TX(0);
#pragma unroll
         for (int j = 0; j < L; j++)
            if (c[k][j] >= 0) s[k] += (TX)v[k][j] * __ldg(x + c[k][j]);
      }
#pragma unroll
      for (int k = 0; k < R; k++) {
         const int64_t r = r0 + k * stride;
         if (r < n) {
            const TY ys = (TY)s[k];
            y[r] = ys;
            d += (double)ys * (self ? (double)ys : (double)__ldg(x + r));
         }
      }
   }
   double vv[1] = {d};
   if (publish_and_arrive<1>(vv, w)) {
      double t[1];
      gather_totals<1>(t, w);
      if (threadIdx.x == 0) *dot_out = t[0];
   }
}

// k_csr_short with the update y = A x + (num / den) y fused into it (the
// p = G^T t + beta p of FSAI-preconditioned CG, beta = num / den from two
// device scalars); one thread per row; types as k_csr_short_dot.
template <typename TV, typename TX, typename TY, int L, int R>
__global__ void __launch_bounds__(256) k_csr_short_xpby(const int32_t* __restrict__ rowptr,
                                                        const int32_t* __restrict__ cols, const TV* __restrict__ vals,
                                                        const TX* __restrict__ x, TY* __restrict__ y, int32_t n,
                                                        const double* __restrict__ num, const double* __restrict__ den,
                                                        const int32_t* __restrict__ skip)
{
   if (skip && *skip) return;
   const TY beta = (TY)(*num / *den);
   const int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t r0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r0 < n; r0 += R * stride) {
      int32_t b[R], e[R];
      TY yo[R];
#pragma unroll
      for (int k = 0; k < R; k++) {
         const int64_t r = r0 + k * stride;
         b[k] = r < n ? rowptr[r] : 0;
         e[k] = r < n ? rowptr[r + 1] : 0;
         yo[k] = r < n ? y[r] : TY(0);
      }
      int32_t c[R][L];
      TV v[R][L];
#pragma unroll
      for (int k = 0; k < R; k++)
#pragma unroll
         for (int j = 0; j < L; j++) {
            c[k][j] = -1;
            v[k][j] = TV(0);
            if (b[k] + j < e[k]) {
               c[k][j] = __ldg(cols + b[k] + j);
               v[k][j] = __ldg(vals + b[k] + j);
            }
         }
#pragma unroll
      for (int k = 0; k < R; k++) {
         TX s = TX(0);
#pragma unroll
         for (int j = 0; j < L; j++)
            if (c[k][j] >= 0) s += (TX)v[k][j] * __ldg(x + c[k][j]);
         const int64_t r = r0 + k * stride;
         if (r < n) y[r] = (TY)s + beta * yo[k];
      }
   }
}

// ---------------------------------------------------------------- tile

__global__ void k_max_row(const int32_t* __restrict__ rowptr, int32_t n, int32_t* __restrict__ out)
{
   int32_t m = 0;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
      m = max(m, rowptr[i + 1] - rowptr[i]);
#pragma unroll
   for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
   if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

__global__ void k_tile_plan(const int32_t* __restrict__ rowptr, int32_t n, int64_t nnz, int32_t tiles,
                            int32_t* __restrict__ tile_row, int32_t* __restrict__ tile_nnz, int32_t* __restrict__ carry_row)
{
   const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (t > tiles) return;
   const int64_t total = (int64_t)n + nnz;
   const int64_t D = ::tnlb::imin64(t * kTileSize, total);
   int64_t lo = ::tnlb::imax64(0, D - nnz), hi = ::tnlb::imin64(D, n);
   while (lo < hi) {
      const int64_t mid = (lo + hi) >> 1;
      if ((int64_t)rowptr[mid + 1] <= D - mid - 1)
         lo = mid + 1;
      else
         hi = mid;
   }
   tile_row[t] = (int32_t)lo;
   tile_nnz[t] = (int32_t)(D - lo);
   if (t < tiles) carry_row[t] = -1;
}

// L2 policies: the streamed values and column indexes are evicted first, the
// gathered vector is kept (it is re-read once per nonzero that points at it);
// no load allocates in L1 (the tile kernel serves irregular matrices, whose
// gathers rarely hit there).
__device__ __forceinline__ uint64_t policy_evict_first()
{
   uint64_t p;
   asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
   return p;
}
__device__ __forceinline__ uint64_t policy_evict_last()
{
   uint64_t p;
   asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
   return p;
}
__device__ __forceinline__ int32_t ld_stream_hint(const int32_t* a, uint64_t pol)
{
   int32_t v;
   asm("ld.global.nc.L1::no_allocate.L2::cache_hint.s32 %0, [%1], %2;" : "=r"(v) : "l"(a), "l"(pol));
   return v;
}
__device__ __forceinline__ double ld_stream_hint(const double* a, uint64_t pol)
{
   double v;
   asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(a), "l"(pol));
   return v;
}
__device__ __forceinline__ float ld_stream_hint(const float* a, uint64_t pol)
{
   float v;
   asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(a), "l"(pol));
   return v;
}
__device__ __forceinline__ double ld_keep(const double* a, uint64_t pol)
{
   double v;
   asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(a), "l"(pol));
   return v;
}
__device__ __forceinline__ float ld_keep(const float* a, uint64_t pol)
{
   float v;
   asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(a), "l"(pol));
   return v;
}

// Merge-path tile of one warp: at most kTileSize = 256 rows + nonzeros.
// Warps work independently (no block-wide barrier), and blocks are small
// (four warps), so a block's slot frees as soon as its few warps are done.
// The tile's nonzeros stay in registers in striped order (lane l holds
// nonzeros k0 + 32 j + l, j < 8): all loads and x gathers are issued before
// any is used.  Everything else stays in registers too:
//  * the rows ending in the tile are marked in a 256-bit mask (eight words,
//    one per 32-nonzero step) at the position of their last nonzero, each
//    word an OR-reduction over the warp of the lanes holding those rows;
//    rows with no nonzero in the tile are written at once;
//  * step j sums its 32 products per row by a segmented shuffle scan whose
//    segments the mask delimits, and keeps the scanned values in place of
//    the products; the row still open at the end of a step carries into the
//    next (a step with no row end only adds each lane's product to a
//    per-lane partial, reduced when the row ends);
//  * the lane of each row then fetches the row's sum from its row-end lane
//    (one shuffle per step) and the rows are written together;
//  * the row open at the end of the tile goes to the carry array.
// Every sum is taken in a fixed order, so results are deterministic.  A
// row-pointer array inconsistent with the tile plan can misplace sums but
// never writes outside rows [r0, r1) of the tile.
template <typename Real>
__global__ void __launch_bounds__(kTileThreads) k_csr_tile(const int32_t* __restrict__ rowptr,
                                                         const int32_t* __restrict__ cols,
                                                         const Real* __restrict__ vals, const Real* __restrict__ x,
                                                         Real* __restrict__ y, const int32_t* __restrict__ tile_row,
                                                         const int32_t* __restrict__ tile_nnz, int32_t tiles, int32_t n,
                                                         int32_t* __restrict__ carry_row, Real* __restrict__ carry_val,
                                                         Real alpha, Real beta, const int32_t* __restrict__ skip)
{
   constexpr int kWarps = kTileThreads / 32;
   constexpr unsigned kAll = 0xffffffffu;
   // solvers pass their device `done` flag: nothing to do once they stopped
   if (skip && *skip) return;
   const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
   const int64_t t = (int64_t)blockIdx.x * kWarps + warp;
   if (t >= tiles) return;  // warp-uniform
   const int32_t r0 = tile_row[t], r1 = tile_row[t + 1];
   const int32_t k0 = tile_nnz[t], k1 = tile_nnz[t + 1];
   const int32_t nrows = r1 - r0, nk = k1 - k0;
   const uint64_t pol_stream = policy_evict_first(), pol_keep = policy_evict_last();

   int32_t c[kTileItems];
   Real v[kTileItems];
#pragma unroll
   for (int j = 0; j < kTileItems; j++) {
      const int32_t e = k0 + j * 32 + lane;
      c[j] = -1;
      v[j] = Real(0);
      if (e < k1) {
         c[j] = ld_stream_hint(cols + e, pol_stream);
         v[j] = ld_stream_hint(vals + e, pol_stream);
      }
   }
   // the first 32 row ends of the tile, loaded before the x gathers are
   // issued so that both latencies overlap (the gathers need only c)
   int32_t eb0 = 0, ee0 = 0;
   if (lane < nrows) {
      eb0 = rowptr[r0 + lane];
      ee0 = rowptr[r0 + lane + 1];
   }
#pragma unroll
   for (int j = 0; j < kTileItems; j++) v[j] = c[j] >= 0 ? v[j] * ld_keep(x + c[j], pol_keep) : Real(0);

   // row-end masks, chunks of 32 rows; a row of chunk q > 0 reloads its ends
   auto row_ends = [&](int32_t q, int32_t& eb, int32_t& ee) {
      eb = eb0;
      ee = ee0;
      if (q > 0) {
         const int32_t i = q * 32 + lane;
         eb = ee = 0;
         if (i < nrows) {
            eb = rowptr[r0 + i];
            ee = rowptr[r0 + i + 1];
         }
      }
   };
   uint32_t m[kTileItems];
#pragma unroll
   for (int j = 0; j < kTileItems; j++) m[j] = 0u;
   bool all_marked = true;  // every row of the tile ends in it (no empty row)
   for (int32_t q = 0; q * 32 < nrows; q++) {
      const int32_t i = q * 32 + lane;
      int32_t eb, ee;
      row_ends(q, eb, ee);
      const bool mark = i < nrows && ee > k0 && ee > eb;
      if (i < nrows && !mark) keep(y, r0 + i, Real(0), alpha, beta);
      all_marked = all_marked && (i >= nrows || mark);
      const int32_t pos = mark ? ee - k0 - 1 : -1;
#pragma unroll
      for (int j = 0; j < kTileItems; j++) {
         const uint32_t bit = (mark && (pos >> 5) == j) ? (1u << (pos & 31)) : 0u;
         m[j] |= __reduce_or_sync(kAll, bit);
      }
   }

   // Blocked form (FP32), for tiles whose rows all end in them (then the
   // k-th marked position ends row r0 + k): the products go through shared
   // memory from striped to blocked order (lane l takes positions 8l ..
   // 8l + 7; one pad word every 32 keeps the stores free of bank
   // conflicts), each lane sums its positions in order, writing the rows
   // that start and end among them, and one segmented scan over the lanes
   // finishes the rows that cross lanes, in place of the striped form's
   // segmented scan per 32-nonzero step.  On the power-law matrix it took
   // the FP32 product from 319 to 292 us; in FP64 it measured 351 against
   // 344 us (the load pipe that serves the gathers, not the issue slots,
   // binds the FP64 product), so FP64 keeps the striped form.
   if (sizeof(Real) == 4 && __all_sync(kAll, all_marked)) {
      __shared__ Real s_prod[kWarps][kTileSize + kTileItems];
      __shared__ uint32_t s_mask[kWarps][kTileItems];
      Real* sp = s_prod[warp];
#pragma unroll
      for (int j = 0; j < kTileItems; j++) sp[j * 33 + lane] = v[j];  // position k = 32 j + lane at k + (k >> 5)
      uint32_t mw = 0u, lm = 0u;
#pragma unroll
      for (int j = 0; j < kTileItems; j++) {
         if (lane == j) mw = m[j];
         if (((nk - 1) >> 5) == j) lm = m[j];
      }
      if (lane < kTileItems) s_mask[warp][lane] = mw;
      __syncwarp();
      const uint32_t bits = (s_mask[warp][lane >> 2] >> ((lane & 3) * 8)) & 0xffu;
      Real pv[kTileItems];
#pragma unroll
      for (int i = 0; i < kTileItems; i++) pv[i] = sp[8 * lane + i + (lane >> 2)];
      // rank of this lane's first row end among the tile's
      const int nends = __popc(bits);
      int incl = nends;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
         const int u = __shfl_up_sync(kAll, incl, o);
         if (lane >= o) incl += u;
      }
      const int32_t row0 = r0 + incl - nends;
      Real run = Real(0), head = Real(0);
      int ended = 0;
#pragma unroll
      for (int i = 0; i < kTileItems; i++) {
         run += pv[i];
         if ((bits >> i) & 1u) {
            if (ended == 0)
               head = run;
            else
               keep(y, row0 + ended, run, alpha, beta);
            ended++;
            run = Real(0);
         }
      }
      // (open sum, row ended) scanned over the lanes: the sum carried into
      // a lane's first row end
      Real sc = run;
      bool fl = ended > 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
         const Real su = __shfl_up_sync(kAll, sc, o);
         const bool fu = __shfl_up_sync(kAll, fl, o);
         if (lane >= o) {
            if (!fl) sc += su;
            fl = fl || fu;
         }
      }
      Real cin = __shfl_up_sync(kAll, sc, 1);
      if (lane == 0) cin = Real(0);
      if (ended > 0) keep(y, row0, head + cin, alpha, beta);
      const Real open_sum = __shfl_sync(kAll, sc, 31);
      if (lane == 0) {
         const bool has = nk > 0 && !((lm >> ((nk - 1) & 31)) & 1u);
         carry_row[t] = (has && r1 < n) ? r1 : -1;
         carry_val[t] = open_sum;
      }
      return;
   }

   // The open row's partial sum: `carry` (one value) plus, after steps with
   // no row end, the per-lane partials `part`, reduced only when the row
   // ends (most nonzeros of a power-law matrix lie in steps without one).
   Real carry = Real(0), part = Real(0);
   bool parts = false;
   uint32_t last_mask = 0u;  // the mask word of the tile's last nonzero
#pragma unroll
   for (int j = 0; j < kTileItems; j++) {
      if (j * 32 < nk) {  // warp-uniform
         const uint32_t mj = m[j];
         if (((nk - 1) >> 5) == j) last_mask = mj;
         if (mj == 0u) {
            part += v[j];
            parts = true;
            continue;
         }
         Real open = carry;
         if (parts) {
            Real s = part;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(kAll, s, o);
            open += s;
            part = Real(0);
            parts = false;
         }
         const uint32_t below = mj & ((1u << lane) - 1u);
         const int seg0 = below ? 32 - __clz(below) : 0;  // first lane of this lane's row
         Real val = v[j];
#pragma unroll
         for (int o = 1; o < 32; o <<= 1) {
            const Real vv = __shfl_up_sync(kAll, val, o);
            if (lane - o >= seg0) val += vv;
         }
         if (seg0 == 0) val += open;
         v[j] = val;
         const Real last = __shfl_sync(kAll, val, 31);
         carry = (mj >> 31) ? Real(0) : last;
      }
   }
   if (parts) {
      Real s = part;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(kAll, s, o);
      carry += s;
   }
   // each row's lane fetches the sum from its row-end lane
   for (int32_t q = 0; q * 32 < nrows; q++) {
      const int32_t i = q * 32 + lane;
      int32_t eb, ee;
      row_ends(q, eb, ee);
      const bool mark = i < nrows && ee > k0 && ee > eb;
      const int32_t pos = mark ? ee - k0 - 1 : 0;
      Real res = Real(0);
#pragma unroll
      for (int j = 0; j < kTileItems; j++) {
         if (j * 32 < nk) {
            const Real tv = __shfl_sync(kAll, v[j], pos & 31);
            if ((pos >> 5) == j) res = tv;
         }
      }
      if (mark) keep(y, r0 + i, res, alpha, beta);
   }
   if (lane == 0) {
      // the row open at the end of the tile (row r1) carries on
      const bool has = nk > 0 && !((last_mask >> ((nk - 1) & 31)) & 1u);
      carry_row[t] = (has && r1 < n) ? r1 : -1;
      carry_val[t] = carry;
   }
}

// Adds the partial sums of rows split between tiles, in tile order.
template <typename Real>
__global__ void k_csr_tile_fixup(const int32_t* __restrict__ carry_row, const Real* __restrict__ carry_val,
                                 int32_t tiles, Real* __restrict__ y, Real alpha, const int32_t* __restrict__ skip)
{
   if (skip && *skip) return;
   const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (t >= tiles) return;
   const int32_t r = carry_row[t];
   if (r < 0) return;
   if (t > 0 && carry_row[t - 1] == r) return;
   Real s = carry_val[t];
   for (int64_t u = t + 1; u < tiles && carry_row[u] == r; u++) s += carry_val[u];
   y[r] += (alpha == Real(1)) ? s : alpha * s;
}

// --------------------------------------------------------------- launch

template <typename Real>
tnlb_status launch_vector(const int32_t* rowptr, const int32_t* cols, const Real* vals, const Real* x, Real* y,
                          int32_t begin, int32_t end, Real alpha, Real beta, int G, cudaStream_t st)
{
   const int64_t rows = (int64_t)end - begin;
   if (rows <= 0) return TNLB_OK;
#define TNLB_VEC(GG)                                                                                    \
   case GG:                                                                                             \
      k_csr_vector<Real, GG><<<grid_for(rows * GG, 256), 256, 0, st>>>(rowptr, cols, vals, x, y, begin, end, \
                                                                         alpha, beta);                  \
      break;
   switch (G) {
      case 1:
         k_csr_scalar<Real><<<grid_for(rows, 256), 256, 0, st>>>(rowptr, cols, vals, x, y, begin, end, alpha, beta);
         break;
         TNLB_VEC(2)
         TNLB_VEC(4)
         TNLB_VEC(8)
         TNLB_VEC(16)
         TNLB_VEC(32)
      case 64:
         k_csr_block<Real, 64><<<grid_for(rows, 4), 256, 0, st>>>(rowptr, cols, vals, x, y, begin, end, alpha, beta);
         break;
      case 128:
         k_csr_block<Real, 128><<<grid_for(rows, 2), 256, 0, st>>>(rowptr, cols, vals, x, y, begin, end, alpha, beta);
         break;
      case 256:
         k_csr_block<Real, 256><<<grid_for(rows, 1), 256, 0, st>>>(rowptr, cols, vals, x, y, begin, end, alpha, beta);
         break;
      default: set_error("threads per segment must be a power of two in 1..256"); return TNLB_ERR_INVALID_ARGUMENT;
   }
#undef TNLB_VEC
   TNLB_CHECK_LAUNCH();
   return TNLB_OK;
}

// Light CSR: TPS from the mean row length (LaunchConfigurationSetter_LightCSR.h:30-58).
int light_tps(int64_t storage, int32_t rows)
{
   if (rows <= 0) return 1;
   const int64_t e = (storage + rows - 1) / rows;
   if (e <= 2) return 2;
   if (e <= 4) return 4;
   if (e <= 8) return 8;
   if (e <= 16) return 16;
   return 32;
}

// The short-row product with the row width L in {4, 5, 7, 8, 16} (5 and 7:
// the 2D and 3D stencils).  Up to four resident waves of rows run on the
// resident blocks (measured on the 1024^2 Laplacian: 5% faster than a
// block per 256 rows); beyond that one thread per row (the 256^3 stencil:
// 7% faster than the resident grid).
template <typename Real>
void launch_csr_short(const tnlb_segments* seg, const int32_t* rowptr, const int32_t* cols, const Real* vals,
                      const Real* x, Real* y, Real alpha, Real beta, cudaStream_t st, const int32_t* skip)
{
   auto go = [&](auto* k) {
      const unsigned full = grid_for(seg->n, 256);
      const unsigned res = resident_grid((const void*)k, 256, seg->n, 1);
      const unsigned g = (int64_t)seg->n <= 4ll * res * 256 ? res : full;
      k<<<g, 256, 0, st>>>(rowptr, cols, vals, x, y, seg->n, alpha, beta, skip);
   };
   if (seg->max_row <= 4) go(k_csr_short<Real, 4>);
   else if (seg->max_row <= 5) go(k_csr_short<Real, 5>);
   else if (seg->max_row <= 7) go(k_csr_short<Real, 7>);
   else if (seg->max_row <= 8) go(k_csr_short<Real, 8>);
   else go(k_csr_short<Real, 16>);
}

template <typename Real>
tnlb_status spmv_csr_t(const tnlb_segments* seg, const int32_t* cols, const Real* vals, const Real* x, Real* y,
                       Real alpha, Real beta, int32_t begin, int32_t end, tnlb_kernel kernel, int32_t tps,
                       cudaStream_t st, int* launches, const int32_t* skip)
{
   const int32_t* rowptr = seg->offsets.as<int32_t>();
   const bool full = begin == 0 && end == seg->n;
   *launches = 0;
   if (end <= begin) return TNLB_OK;
   switch (kernel) {
      case TNLB_KERNEL_SCALAR:
         *launches = 1;
         return launch_vector<Real>(rowptr, cols, vals, x, y, begin, end, alpha, beta, 1, st);
      case TNLB_KERNEL_VECTOR:
         *launches = 1;
         return launch_vector<Real>(rowptr, cols, vals, x, y, begin, end, alpha, beta, tps > 0 ? tps : 32, st);
      case TNLB_KERNEL_LIGHT:
         *launches = 1;
         return launch_vector<Real>(rowptr, cols, vals, x, y, begin, end, alpha, beta,
                                    tps > 0 ? tps : light_tps(seg->elements, seg->n), st);
      case TNLB_KERNEL_ADAPTIVE: {
         const int k = sizeof(Real) == 8 ? 3 : 2;
         if (!full || seg->acsr_count[k] == 0 || seg->format != TNLB_ADAPTIVE_CSR) {
            // the reference falls back to the CSR kernels (ReducingOperations_AdaptiveCSR.h:51-57)
            *launches = 1;
            return launch_vector<Real>(rowptr, cols, vals, x, y, begin, end, alpha, beta,
                                       light_tps(seg->elements, seg->n), st);
         }
         const int64_t warps = seg->acsr_count[k] - 1;
         k_csr_adaptive<Real><<<grid_for(warps, 8), 256, 0, st>>>(seg->acsr_blocks[k].as<tnlb_acsr_block>(), warps,
                                                                  rowptr, cols, vals, x, y, alpha, beta);
         TNLB_CHECK_LAUNCH();
         *launches = 1;
         return TNLB_OK;
      }
      case TNLB_KERNEL_DEFAULT:
      case TNLB_KERNEL_TILE:
      default: {
         if (!full || seg->tiles == 0) {
            *launches = 1;
            return launch_vector<Real>(rowptr, cols, vals, x, y, begin, end, alpha, beta,
                                       light_tps(seg->elements, seg->n), st);
         }
         if (kernel != TNLB_KERNEL_TILE && seg->max_row >= 0 && seg->max_row <= 16) {
            launch_csr_short<Real>(seg, rowptr, cols, vals, x, y, alpha, beta, st, skip);
            TNLB_CHECK_LAUNCH();
            *launches = 1;
            return TNLB_OK;
         }
         k_csr_tile<Real><<<grid_for(seg->tiles, kTileThreads / 32), kTileThreads, 0, st>>>(
            rowptr, cols, vals, x, y, seg->tile_row.as<int32_t>(), seg->tile_nnz.as<int32_t>(), seg->tiles, seg->n,
            seg->carry_row.as<int32_t>(), seg->carry_val.as<Real>(), alpha, beta, skip);
         TNLB_CHECK_LAUNCH();
         k_csr_tile_fixup<Real><<<grid_for(seg->tiles, 256), 256, 0, st>>>(
            seg->carry_row.as<int32_t>(), seg->carry_val.as<Real>(), seg->tiles, y, alpha, skip);
         TNLB_CHECK_LAUNCH();
         *launches = 2;
         return TNLB_OK;
      }
   }
}

}  // namespace

tnlb_status build_csr_tile_plan(tnlb_segments* seg, cudaStream_t stream)
{
   const int64_t total = (int64_t)seg->n + seg->elements;
   const int64_t tiles = (total + kTileSize - 1) / kTileSize;
   TNLB_REQUIRE(tiles < INT32_MAX, TNLB_ERR_OVERFLOW, "too many tiles");
   seg->tiles = (int32_t)tiles;
   TNLB_TRY_STATUS(seg->tile_row.alloc(sizeof(int32_t) * (tiles + 1)));
   TNLB_TRY_STATUS(seg->tile_nnz.alloc(sizeof(int32_t) * (tiles + 1)));
   TNLB_TRY_STATUS(seg->carry_row.alloc(sizeof(int32_t) * (tiles + 1)));
   TNLB_TRY_STATUS(seg->carry_val.alloc(sizeof(double) * (tiles + 1)));
   k_tile_plan<<<grid_for(tiles + 1, 256), 256, 0, stream>>>(seg->offsets.as<int32_t>(), seg->n, seg->elements,
                                                              (int32_t)tiles, seg->tile_row.as<int32_t>(),
                                                              seg->tile_nnz.as<int32_t>(), seg->carry_row.as<int32_t>());
   TNLB_CHECK_LAUNCH();
   // longest row, for the choice of the default kernel
   DeviceBuffer mx;
   TNLB_TRY_STATUS(mx.alloc(sizeof(int32_t)));
   TNLB_CUDA_TRY(cudaMemsetAsync(mx.ptr, 0, sizeof(int32_t), stream));
   if (seg->n > 0) {
      k_max_row<<<grid_for(seg->n, 256 * 8), 256, 0, stream>>>(seg->offsets.as<int32_t>(), seg->n, mx.as<int32_t>());
      TNLB_CHECK_LAUNCH();
   }
   int32_t h = 0;
   TNLB_CUDA_TRY(cudaMemcpyAsync(&h, mx.ptr, sizeof(int32_t), cudaMemcpyDeviceToHost, stream));
   TNLB_CUDA_TRY(cudaStreamSynchronize(stream));
   seg->max_row = h;
   return TNLB_OK;
}

bool spmv_dot_fusable(const tnlb_segments* seg)
{
   return seg->format == TNLB_CSR && seg->n > 0 && seg->max_row >= 0 && seg->max_row <= 16;
}

int64_t spmv_dot_partials(const tnlb_segments*) { return kRedMaxBlocks; }


namespace {

// Rows per thread and pass of the fused short-row kernels (measured on the
// 2048^2 diffusion matrix and its FSAI factors, 4.2M rows): the FP64
// products gain from two rows in flight per thread, the FP32 product with
// (x, y) runs fastest with one, the FP32 product with the p update with
// four.  The row arrays are L wide (L = 5 and 7: the 2D and 3D stencils).
template <typename TV, int L, bool Dot>
constexpr int short_rows()
{
   return L > 8 ? 1 : sizeof(TV) == 8 ? (L > 5 ? 1 : 2) : Dot ? 1 : (L > 5 ? 2 : 4);
}

// The row width for seg->max_row: 4, 5, 7, 8 or 16.
#define TNLB_SHORT_WIDTH(seg, ...)  \
   do {                              \
      if ((seg)->max_row <= 4) {     \
         constexpr int L = 4;        \
         __VA_ARGS__;                \
      }                              \
      else if ((seg)->max_row <= 5) { \
         constexpr int L = 5;        \
         __VA_ARGS__;                \
      }                              \
      else if ((seg)->max_row <= 7) { \
         constexpr int L = 7;        \
         __VA_ARGS__;                \
      }                              \
      else if ((seg)->max_row <= 8) { \
         constexpr int L = 8;        \
         __VA_ARGS__;                \
      }                              \
      else {                         \
         constexpr int L = 16;       \
         __VA_ARGS__;                \
      }                              \
   } while (0)

template <typename TV, typename TX, typename TY>
void launch_short_dot(const tnlb_segments* seg, const int32_t* cols, const void* vals, const void* x, void* y, RedWork w,
                      double* dot_out, cudaStream_t st, const int32_t* skip, int self)
{
   const int32_t* rp = seg->offsets.as<int32_t>();
   const TV* v = (const TV*)vals;
   TNLB_SHORT_WIDTH(seg, {
      constexpr int R = short_rows<TV, L, true>();
      auto* k = k_csr_short_dot<TV, TX, TY, L, R>;
      const unsigned g = resident_grid((const void*)k, 256, seg->n, R);
      k<<<g, 256, 0, st>>>(rp, cols, v, (const TX*)x, (TY*)y, seg->n, w, dot_out, skip, self);
   });
}

template <typename TV, typename TX, typename TY>
void launch_short_xpby(const tnlb_segments* seg, const int32_t* cols, const void* vals, const void* x, void* y,
                       const double* num, const double* den, cudaStream_t st, const int32_t* skip)
{
   const int32_t* rp = seg->offsets.as<int32_t>();
   const TV* v = (const TV*)vals;
   TNLB_SHORT_WIDTH(seg, {
      constexpr int R = short_rows<TV, L, false>();
      auto* k = k_csr_short_xpby<TV, TX, TY, L, R>;
      const unsigned g = resident_grid((const void*)k, 256, seg->n, R);
      k<<<g, 256, 0, st>>>(rp, cols, v, (const TX*)x, (TY*)y, seg->n, num, den, skip);
   });
}
#undef TNLB_SHORT_WIDTH

}  // namespace

tnlb_status spmv_dot_mixed(const tnlb_segments* seg, tnlb_real tv, tnlb_real tx, tnlb_real ty, const int32_t* cols,
                           const void* vals, const void* x, void* y, double* partials, unsigned* counter,
                           double* dot_out, cudaStream_t st, const int32_t* skip, bool self_dot)
{
   TNLB_REQUIRE(spmv_dot_fusable(seg), TNLB_ERR_INVALID_ARGUMENT, "spmv_dot: not a short-row CSR matrix");
   RedWork w{partials, counter};
   const int self = self_dot ? 1 : 0;
   if (tv == TNLB_F64 && tx == TNLB_F64 && ty == TNLB_F64)
      launch_short_dot<double, double, double>(seg, cols, vals, x, y, w, dot_out, st, skip, self);
   else if (tv == TNLB_F32 && tx == TNLB_F32 && ty == TNLB_F32)
      launch_short_dot<float, float, float>(seg, cols, vals, x, y, w, dot_out, st, skip, self);
   else if (tv == TNLB_F32 && tx == TNLB_F64 && ty == TNLB_F64)
      launch_short_dot<float, double, double>(seg, cols, vals, x, y, w, dot_out, st, skip, self);
   else if (tv == TNLB_F32 && tx == TNLB_F64 && ty == TNLB_F32)
      launch_short_dot<float, double, float>(seg, cols, vals, x, y, w, dot_out, st, skip, self);
   else {
      set_error("spmv_dot: unsupported combination of value and vector types");
      return TNLB_ERR_INVALID_ARGUMENT;
   }
   TNLB_CHECK_LAUNCH();
   return TNLB_OK;
}

tnlb_status spmv_dot(const tnlb_segments* seg, tnlb_real real, const int32_t* cols, const void* vals, const void* x,
                     void* y, double* partials, unsigned* counter, double* dot_out, cudaStream_t st,
                     const int32_t* skip, bool self_dot)
{
   return spmv_dot_mixed(seg, real, real, real, cols, vals, x, y, partials, counter, dot_out, st, skip, self_dot);
}

tnlb_status spmv_xpby_mixed(const tnlb_segments* seg, tnlb_real tv, tnlb_real tx, tnlb_real ty, const int32_t* cols,
                            const void* vals, const void* x, void* y, const double* num, const double* den,
                            cudaStream_t st, const int32_t* skip)
{
   TNLB_REQUIRE(spmv_dot_fusable(seg), TNLB_ERR_INVALID_ARGUMENT, "spmv_xpby: not a short-row CSR matrix");
   if (tv == TNLB_F64 && tx == TNLB_F64 && ty == TNLB_F64)
      launch_short_xpby<double, double, double>(seg, cols, vals, x, y, num, den, st, skip);
   else if (tv == TNLB_F32 && tx == TNLB_F32 && ty == TNLB_F32)
      launch_short_xpby<float, float, float>(seg, cols, vals, x, y, num, den, st, skip);
   else if (tv == TNLB_F32 && tx == TNLB_F32 && ty == TNLB_F64)
      launch_short_xpby<float, float, double>(seg, cols, vals, x, y, num, den, st, skip);
   else {
      set_error("spmv_xpby: unsupported combination of value and vector types");
      return TNLB_ERR_INVALID_ARGUMENT;
   }
   TNLB_CHECK_LAUNCH();
   return TNLB_OK;
}

tnlb_status spmv_xpby(const tnlb_segments* seg, tnlb_real real, const int32_t* cols, const void* vals, const void* x,
                      void* y, const double* num, const double* den, cudaStream_t st, const int32_t* skip)
{
   return spmv_xpby_mixed(seg, real, real, real, cols, vals, x, y, num, den, st, skip);
}

tnlb_status spmv_csr(const tnlb_segments* seg, tnlb_real real, const int32_t* cols, const void* vals, const void* x,
                     void* y, double alpha, double beta, int32_t begin, int32_t end, tnlb_kernel kernel, int32_t tps,
                     cudaStream_t stream, int* launches, const int32_t* skip)
{
   if (real == TNLB_F64)
      return spmv_csr_t<double>(seg, cols, (const double*)vals, (const double*)x, (double*)y, alpha, beta, begin, end,
                                kernel, tps, stream, launches, skip);
   return spmv_csr_t<float>(seg, cols, (const float*)vals, (const float*)x, (float*)y, (float)alpha, (float)beta,
                            begin, end, kernel, tps, stream, launches, skip);
}

}  // namespace tnlb

// ------------------------------------------- CSR SpMV without allocation
//
// tnlb_spmv_csr_noalloc runs the tile kernel above on plain CSR arrays with
// no segments handle.  Its per-call scratch -- the tile plan and the carry
// of rows split between tiles -- lives in one statically sized device array
// of this file, so a call allocates no device memory.  Every call rewrites
// each scratch entry it reads (the plan kernel writes all tile coordinates
// and resets the carry rows; the tile kernel writes every tile's carry), so
// nothing has to start at zero.  Calls that overlap on one device share the
// array and race.

namespace {

constexpr int64_t kNoAllocMaxTiles = 262144;  // rows + nonzeros <= 67,108,864
constexpr size_t kNoAllocAlign = 256;
constexpr size_t round_up_256(size_t b) { return (b + kNoAllocAlign - 1) / kNoAllocAlign * kNoAllocAlign; }
constexpr size_t kNoAllocCarryValBytes = round_up_256(sizeof(double) * kNoAllocMaxTiles);
constexpr size_t kNoAllocPlanBytes = round_up_256(sizeof(int32_t) * (kNoAllocMaxTiles + 1));
constexpr size_t kNoAllocCarryRowBytes = round_up_256(sizeof(int32_t) * kNoAllocMaxTiles);
constexpr size_t kNoAllocBytes = kNoAllocCarryValBytes + 2 * kNoAllocPlanBytes + kNoAllocCarryRowBytes;

}  // namespace

// 5.2 MB: carry values (FP64 slots, FP32 uses the first half), tile rows,
// tile nonzero offsets, carry rows.
static __device__ __align__(256) unsigned char g_tile_scratch[kNoAllocBytes];

namespace {

// Address of g_tile_scratch in the current device's context.  It is looked
// up on every call (cheap once the module is loaded) rather than cached, so
// a device reset or another context on the same ordinal never leaves a
// stale address behind.
tnlb_status noalloc_scratch(unsigned char** base)
{
   void* p = nullptr;
   TNLB_CUDA_TRY(cudaGetSymbolAddress(&p, g_tile_scratch));
   *base = (unsigned char*)p;
   return TNLB_OK;
}

template <typename Real>
tnlb_status spmv_csr_noalloc_t(unsigned char* base, int32_t rows, int64_t nnz, int32_t tiles, const int32_t* rowptr,
                               const int32_t* cols, const Real* vals, const Real* x, Real* y, Real alpha, Real beta,
                               cudaStream_t st)
{
   Real* carry_val = (Real*)base;
   int32_t* tile_row = (int32_t*)(base + kNoAllocCarryValBytes);
   int32_t* tile_nnz = (int32_t*)(base + kNoAllocCarryValBytes + kNoAllocPlanBytes);
   int32_t* carry_row = (int32_t*)(base + kNoAllocCarryValBytes + 2 * kNoAllocPlanBytes);
   tnlb::k_tile_plan<<<tnlb::grid_for((int64_t)tiles + 1, 256), 256, 0, st>>>(rowptr, rows, nnz, tiles, tile_row,
                                                                               tile_nnz, carry_row);
   TNLB_CHECK_LAUNCH();
   tnlb::k_csr_tile<Real><<<tnlb::grid_for(tiles, tnlb::kTileThreads / 32), tnlb::kTileThreads, 0, st>>>(
      rowptr, cols, vals, x, y, tile_row, tile_nnz, tiles, rows, carry_row, carry_val, alpha, beta, nullptr);
   TNLB_CHECK_LAUNCH();
   tnlb::k_csr_tile_fixup<Real><<<tnlb::grid_for(tiles, 256), 256, 0, st>>>(carry_row, carry_val, tiles, y, alpha,
                                                                             nullptr);
   TNLB_CHECK_LAUNCH();
   return TNLB_OK;
}

}  // namespace

extern "C" tnlb_status tnlb_spmv_csr_noalloc(tnlb_real real, int32_t rows, int32_t columns, int64_t nnz,
                                             const int32_t* d_rowptr, const int32_t* d_cols, const void* d_values,
                                             const void* d_x, void* d_y, double alpha, double beta,
                                             tnlb_stream stream)
{
   using namespace tnlb;
   clear_error();
   TNLB_REQUIRE(real == TNLB_F32 || real == TNLB_F64, TNLB_ERR_INVALID_ARGUMENT, "unknown real type");
   TNLB_REQUIRE(rows >= 0 && columns >= 0 && nnz >= 0 && nnz <= INT32_MAX, TNLB_ERR_INVALID_ARGUMENT,
                "tnlb_spmv_csr_noalloc: negative size or more than 2^31-1 nonzeros");
   const int64_t tiles = ((int64_t)rows + nnz + kTileSize - 1) / kTileSize;
   TNLB_REQUIRE(tiles <= kNoAllocMaxTiles, TNLB_ERR_INVALID_ARGUMENT,
                "tnlb_spmv_csr_noalloc: rows + nonzeros exceeds the static scratch limit of 67108864 "
                "(262144 tiles of 256); use tnlb_spmv");
   if (rows == 0) return TNLB_OK;
   TNLB_REQUIRE(d_rowptr && d_y && (nnz == 0 || (d_cols && d_values && d_x)), TNLB_ERR_INVALID_ARGUMENT,
                "null array");
   unsigned char* base = nullptr;
   TNLB_TRY_STATUS(noalloc_scratch(&base));
   if (real == TNLB_F64)
      return spmv_csr_noalloc_t<double>(base, rows, nnz, (int32_t)tiles, d_rowptr, d_cols, (const double*)d_values,
                                        (const double*)d_x, (double*)d_y, alpha, beta, (cudaStream_t)stream);
   return spmv_csr_noalloc_t<float>(base, rows, nnz, (int32_t)tiles, d_rowptr, d_cols, (const float*)d_values,
                                    (const float*)d_x, (float*)d_y, (float)alpha, (float)beta, (cudaStream_t)stream);
}
