// spmv_ell.cu -- y = alpha*A*x + beta*y for Ellpack, SlicedEllpack,
// ChunkedEllpack and BiEllpack segments (both element organizations).
//
//  * Ellpack, column-major (the reference's GPU default): one thread per row
//    walking slots row + alignedSize*k -- consecutive rows give coalesced
//    loads (ReducingOperations_Ellpack.h:186-199).  Row-major: G lanes per
//    row (EllpackCudaReductionKernel, ReducingKernels_Ellpack.h:12-74).
//  * SlicedEllpack (slice 32), column-major: one warp per slice, lane = row,
//    slot k of the slice is 32 consecutive elements (256 B in FP64), loop
//    unrolled by 4 to keep loads in flight; G > 1 splits the slot range of a
//    slice over G warps of a block and combines them in shared memory
//    (reduceSegmentsSlicedEllpackKernel, ReducingKernels_SlicedEllpack.h:100-323).
//    Row-major: G lanes per row.
//  * ChunkedEllpack: one block per slice, one thread per chunk, per-chunk
//    partials in shared memory, then each row sums its chunks
//    (ChunkedEllpackReduceSegmentsKernel, ReducingKernels_ChunkedEllpack.h:13-98).
//  * BiEllpack: one warp per strip of 32 rows; lane = sorted position, groups
//    of halving height 32,16,8,4,2,1; the result is moved to the original
//    row through the permutation with one shuffle
//    (BiEllpackReduceSegmentsKernel, ReducingKernels_BiEllpack.h:70-217).
#include "internal.cuh"
#include "reduce.cuh"

namespace tnlb {
namespace {

template <typename Real>
__device__ __forceinline__ void keep_range(Real* y, int64_t row, Real v, Real alpha, Real beta, int32_t begin,
                                           int32_t end)
{
   if (row >= begin && row < end) keep(y, (int32_t)row, v, alpha, beta);
}

template <typename Real>
__device__ __forceinline__ Real fma_slot(const int32_t* cols, const Real* vals, const Real* x, int64_t g, Real acc)
{
   const int32_t c = ld_stream(cols + g);
   const Real v = ld_stream(vals + g);
   return c >= 0 ? acc + v * ld_gather(x + c) : acc;
}

// ------------------------------------------------------------- Ellpack

template <typename Real>
__global__ void k_ell_col(const int32_t* __restrict__ cols, const Real* __restrict__ vals, const Real* __restrict__ x,
                          Real* __restrict__ y, int32_t n, int32_t width, int32_t aligned, int32_t begin, int32_t end,
                          Real alpha, Real beta)
{
   const int64_t row = begin + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (row >= end) return;
   Real sum = 0;
   int32_t k = 0;
   if (width <= 8) {
      // narrow rows (stencils): every slot's load issued at once
      int32_t c[8];
      Real v[8];
#pragma unroll
      for (int u = 0; u < 8; u++) {
         c[u] = -1;
         v[u] = Real(0);
         if (u < width) {
            c[u] = ld_stream(cols + row + (int64_t)aligned * u);
            v[u] = ld_stream(vals + row + (int64_t)aligned * u);
         }
      }
#pragma unroll
      for (int u = 0; u < 8; u++)
         if (c[u] >= 0) sum += v[u] * ld_gather(x + c[u]);
      k = width;
   }
   for (; k + 4 <= width; k += 4) {
      int32_t c[4];
      Real v[4];
#pragma unroll
      for (int u = 0; u < 4; u++) {
         c[u] = ld_stream(cols + row + (int64_t)aligned * (k + u));
         v[u] = ld_stream(vals + row + (int64_t)aligned * (k + u));
      }
#pragma unroll
      for (int u = 0; u < 4; u++)
         if (c[u] >= 0) sum += v[u] * ld_gather(x + c[u]);
   }
   for (; k < width; k++) sum = fma_slot(cols, vals, x, row + (int64_t)aligned * k, sum);
   keep(y, (int32_t)row, sum, alpha, beta);
}

template <typename Real, int G>
__global__ void k_ell_row(const int32_t* __restrict__ cols, const Real* __restrict__ vals, const Real* __restrict__ x,
                          Real* __restrict__ y, int32_t width, int32_t begin, int32_t end, Real alpha, Real beta)
{
   const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   const int64_t row = begin + gid / G;
   const int lane = (int)(gid % G);
   Real sum = 0;
   if (row < end)
      for (int32_t k = lane; k < width; k += G) sum = fma_slot(cols, vals, x, row * width + k, sum);
   sum = group_sum<G>(sum);
   if (row < end && lane == 0) keep(y, (int32_t)row, sum, alpha, beta);
}

// ------------------------------------------------------- SlicedEllpack

// G warps per slice (G = 1, 2, 4, 8); the block holds 8/G slices.
template <typename Real, int G>
__global__ void __launch_bounds__(256) k_sell_col(const int32_t* __restrict__ cols, const Real* __restrict__ vals,
                                                  const Real* __restrict__ x, Real* __restrict__ y,
                                                  const int32_t* __restrict__ slice_off,
                                                  const int32_t* __restrict__ slice_w, int32_t slices, int32_t begin,
                                                  int32_t end, Real alpha, Real beta)
{
   __shared__ Real part[8][32];
   const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
   const int sub = wib % G;
   const int64_t slice = (int64_t)blockIdx.x * (8 / G) + wib / G;
   Real sum = 0;
   if (slice < slices) {
      const int64_t off = slice_off[slice] + lane;
      const int32_t w = slice_w[slice];
      int32_t k = sub;
      if (G == 1 && w <= 8) {
         // narrow slices (stencils): every slot's load issued at once
         int32_t c[8];
         Real v[8];
#pragma unroll
         for (int u = 0; u < 8; u++) {
            c[u] = -1;
            v[u] = Real(0);
            if (u < w) {
               c[u] = ld_stream(cols + off + (int64_t)kSellSlice * u);
               v[u] = ld_stream(vals + off + (int64_t)kSellSlice * u);
            }
         }
#pragma unroll
         for (int u = 0; u < 8; u++)
            if (c[u] >= 0) sum += v[u] * ld_gather(x + c[u]);
         k = w;
      }
      for (; k + 3 * G < w; k += 4 * G) {
         int32_t c[4];
         Real v[4];
#pragma unroll
         for (int u = 0; u < 4; u++) {
            c[u] = ld_stream(cols + off + (int64_t)kSellSlice * (k + u * G));
            v[u] = ld_stream(vals + off + (int64_t)kSellSlice * (k + u * G));
         }
#pragma unroll
         for (int u = 0; u < 4; u++)
            if (c[u] >= 0) sum += v[u] * ld_gather(x + c[u]);
      }
      for (; k < w; k += G) sum = fma_slot(cols, vals, x, off + (int64_t)kSellSlice * k, sum);
   }
   if (G == 1) {
      if (slice < slices) keep_range(y, slice * kSellSlice + lane, sum, alpha, beta, begin, end);
      return;
   }
   part[wib][lane] = sum;
   __syncthreads();
   if (sub == 0 && slice < slices) {
      Real s = 0;
#pragma unroll
      for (int q = 0; q < G; q++) s += part[wib + q][lane];
      keep_range(y, slice * kSellSlice + lane, s, alpha, beta, begin, end);
   }
}

// One warp per slice over a resident grid (G = 1): each warp walks the
// slices with the grid's warp count as stride and loads the next slice's
// offset and width before the current slice's entries, so the slice table
// is not a step of every slice's chain of dependent loads (on a 5-point
// operator the per-wave chain offset -> entries -> x made the full-grid
// launch 20% slower than Ellpack).
template <typename Real>
__global__ void __launch_bounds__(256) k_sell_walk(const int32_t* __restrict__ cols, const Real* __restrict__ vals,
                                                   const Real* __restrict__ x, Real* __restrict__ y,
                                                   const int32_t* __restrict__ slice_off,
                                                   const int32_t* __restrict__ slice_w, int32_t slices, int32_t begin,
                                                   int32_t end, Real alpha, Real beta)
{
   const int lane = threadIdx.x & 31;
   const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
   int64_t s = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
   int32_t o = 0, w = 0;
   if (s < slices) {
      o = slice_off[s];
      w = slice_w[s];
   }
   for (; s < slices; s += nw) {
      const int64_t off = (int64_t)o + lane;
      const int32_t wc = w;
      if (s + nw < slices) {
         o = slice_off[s + nw];
         w = slice_w[s + nw];
      }
      Real sum = 0;
      int32_t k = 0;
      if (wc <= 8) {
         int32_t c[8];
         Real v[8];
#pragma unroll
         for (int u = 0; u < 8; u++) {
            c[u] = -1;
            v[u] = Real(0);
            if (u < wc) {
               c[u] = ld_stream(cols + off + (int64_t)kSellSlice * u);
               v[u] = ld_stream(vals + off + (int64_t)kSellSlice * u);
            }
         }
#pragma unroll
         for (int u = 0; u < 8; u++)
            if (c[u] >= 0) sum += v[u] * ld_gather(x + c[u]);
         k = wc;
      }
      for (; k + 3 < wc; k += 4) {
         int32_t c[4];
         Real v[4];
#pragma unroll
         for (int u = 0; u < 4; u++) {
            c[u] = ld_stream(cols + off + (int64_t)kSellSlice * (k + u));
            v[u] = ld_stream(vals + off + (int64_t)kSellSlice * (k + u));
         }
#pragma unroll
         for (int u = 0; u < 4; u++)
            if (c[u] >= 0) sum += v[u] * ld_gather(x + c[u]);
      }
      for (; k < wc; k++) sum = fma_slot(cols, vals, x, off + (int64_t)kSellSlice * k, sum);
      keep_range(y, s * kSellSlice + lane, sum, alpha, beta, begin, end);
   }
}

template <typename Real, int G>
__global__ void k_sell_row(const int32_t* __restrict__ cols, const Real* __restrict__ vals, const Real* __restrict__ x,
                           Real* __restrict__ y, const int32_t* __restrict__ slice_off,
                           const int32_t* __restrict__ slice_w, int32_t begin, int32_t end, Real alpha, Real beta)
{
   const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   const int64_t row = begin + gid / G;
   const int lane = (int)(gid % G);
   Real sum = 0;
   if (row < end) {
      const int64_t s = row / kSellSlice;
      const int32_t w = slice_w[s];
      const int64_t base = slice_off[s] + (row % kSellSlice) * (int64_t)w;
      for (int32_t k = lane; k < w; k += G) sum = fma_slot(cols, vals, x, base + k, sum);
   }
   sum = group_sum<G>(sum);
   if (row < end && lane == 0) keep(y, (int32_t)row, sum, alpha, beta);
}

// ------------------------------------------------------ ChunkedEllpack

template <typename Real, bool ColMajor>
__global__ void __launch_bounds__(kChunksInSlice) k_chell(const int32_t* __restrict__ cols,
                                                          const Real* __restrict__ vals, const Real* __restrict__ x,
                                                          Real* __restrict__ y, const int32_t* __restrict__ sl_size,
                                                          const int32_t* __restrict__ sl_chunk,
                                                          const int32_t* __restrict__ sl_first,
                                                          const int32_t* __restrict__ sl_ptr,
                                                          const int32_t* __restrict__ seg_to_chunk, int32_t begin,
                                                          int32_t end, Real alpha, Real beta)
{
   __shared__ Real chunk_sum[kChunksInSlice];
   const int32_t s = blockIdx.x;
   const int c = threadIdx.x;
   const int64_t off = sl_ptr[s];
   const int32_t cs = sl_chunk[s];
   Real sum = 0;
   if (ColMajor) {
      for (int32_t k = 0; k < cs; k++) sum = fma_slot(cols, vals, x, off + c + (int64_t)kChunksInSlice * k, sum);
   }
   else {
      const int64_t b = off + (int64_t)c * cs;
      for (int32_t k = 0; k < cs; k++) sum = fma_slot(cols, vals, x, b + k, sum);
   }
   chunk_sum[c] = sum;
   __syncthreads();
   if (c < sl_size[s]) {
      const int32_t seg = sl_first[s] + c;
      int32_t ch = c == 0 ? 0 : seg_to_chunk[seg - 1];
      const int32_t last = seg_to_chunk[seg];
      Real r = 0;
      while (ch < last) r += chunk_sum[ch++];
      keep_range(y, seg, r, alpha, beta, begin, end);
   }
}

// ----------------------------------------------------------- BiEllpack

// Column-major strips: group g of a strip holds the h = 32 >> g widest rows
// (sorted positions 0..h-1) with w slots each, slot (k, r) at base + k h + r.
// All 32 lanes stride through the group's h w slots: lane l always meets
// row l & (h-1), so it keeps one partial sum, and the partials of a row are
// added across the lanes l, l + h, ... by log2(32/h) shuffles.  A strip with
// one dominant row (power-law matrices) thus spreads that row over the warp
// instead of leaving it to one lane.  Four slots per lane are loaded before
// any is used.
template <typename Real>
__global__ void k_biell_col(const int32_t* __restrict__ cols, const Real* __restrict__ vals,
                            const Real* __restrict__ x, Real* __restrict__ y, const int32_t* __restrict__ perm,
                            const int32_t* __restrict__ gp, int32_t n, int32_t strips, int32_t begin, int32_t end,
                            Real alpha, Real beta)
{
   const int64_t strip = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
   const int lane = threadIdx.x & 31;  // sorted position in the strip
   if (strip >= strips) return;
   const int32_t* g = gp + strip * kBiGroups;
   Real sum = 0;
   int h = 32;
   for (int grp = 0; grp < kBiGroups; grp++, h >>= 1) {
      const int64_t base = g[grp];
      const int32_t size = g[grp + 1] - g[grp];
      if (size == 0) continue;  // warp-uniform
      Real part = 0;
      int32_t s = lane;
      for (; s + 96 < size; s += 128) {
         int32_t c[4];
         Real v[4];
#pragma unroll
         for (int u = 0; u < 4; u++) {
            c[u] = ld_stream(cols + base + s + 32 * u);
            v[u] = ld_stream(vals + base + s + 32 * u);
         }
#pragma unroll
         for (int u = 0; u < 4; u++)
            if (c[u] >= 0) part += v[u] * ld_gather(x + c[u]);
      }
      for (; s < size; s += 32) part = fma_slot(cols, vals, x, base + s, part);
      for (int o = 16; o >= h; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
      if (lane < h) sum += part;
   }
   const int64_t row = strip * kBiStrip + lane;  // original row of this lane
   const int src = row < n ? perm[row] - (int32_t)(strip * kBiStrip) : 0;
   const Real mine = __shfl_sync(0xffffffffu, sum, src);
   if (row < n) keep_range(y, row, mine, alpha, beta, begin, end);
}

// Row-major strips: lane = sorted position walks its own w slots.
template <typename Real>
__global__ void k_biell_row(const int32_t* __restrict__ cols, const Real* __restrict__ vals,
                            const Real* __restrict__ x, Real* __restrict__ y, const int32_t* __restrict__ perm,
                            const int32_t* __restrict__ gp, int32_t n, int32_t strips, int32_t begin, int32_t end,
                            Real alpha, Real beta)
{
   const int64_t strip = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
   const int lane = threadIdx.x & 31;
   if (strip >= strips) return;
   const int32_t* g = gp + strip * kBiGroups;
   Real sum = 0;
   int h = 32;
   for (int grp = 0; grp < kBiGroups; grp++, h >>= 1) {
      const int64_t base = g[grp];
      const int32_t size = g[grp + 1] - g[grp];
      if (size == 0 || lane >= h) continue;
      const int32_t w = size / h;
      for (int32_t k = 0; k < w; k++) sum = fma_slot(cols, vals, x, base + (int64_t)lane * w + k, sum);
   }
   const int64_t row = strip * kBiStrip + lane;
   const int src = row < n ? perm[row] - (int32_t)(strip * kBiStrip) : 0;
   const Real mine = __shfl_sync(0xffffffffu, sum, src);
   if (row < n) keep_range(y, row, mine, alpha, beta, begin, end);
}

template <typename Real>
tnlb_status launch(const tnlb_segments* seg, const int32_t* cols, const Real* vals, const Real* x, Real* y, Real alpha,
                   Real beta, int32_t begin, int32_t end, tnlb_kernel kernel, int32_t tps, cudaStream_t st,
                   int* launches)
{
   const bool col = seg->organization == TNLB_COLUMN_MAJOR;
   *launches = 0;
   if (end <= begin) return TNLB_OK;
   switch (seg->format) {
      case TNLB_ELLPACK: {
         if (col) {
            k_ell_col<Real><<<grid_for((int64_t)end - begin, 256), 256, 0, st>>>(
               cols, vals, x, y, seg->n, seg->segment_size, seg->aligned_size, begin, end, alpha, beta);
         }
         else {
            int G = tps > 0 ? tps : 1;
            if (kernel == TNLB_KERNEL_DEFAULT && tps <= 0) G = seg->segment_size >= 32 ? 32 : (seg->segment_size >= 8 ? 8 : 1);
            const int64_t th = ((int64_t)end - begin) * G;
            switch (G) {
               case 1: k_ell_row<Real, 1><<<grid_for(th, 256), 256, 0, st>>>(cols, vals, x, y, seg->segment_size, begin, end, alpha, beta); break;
               case 2: k_ell_row<Real, 2><<<grid_for(th, 256), 256, 0, st>>>(cols, vals, x, y, seg->segment_size, begin, end, alpha, beta); break;
               case 4: k_ell_row<Real, 4><<<grid_for(th, 256), 256, 0, st>>>(cols, vals, x, y, seg->segment_size, begin, end, alpha, beta); break;
               case 8: k_ell_row<Real, 8><<<grid_for(th, 256), 256, 0, st>>>(cols, vals, x, y, seg->segment_size, begin, end, alpha, beta); break;
               case 16: k_ell_row<Real, 16><<<grid_for(th, 256), 256, 0, st>>>(cols, vals, x, y, seg->segment_size, begin, end, alpha, beta); break;
               case 32: k_ell_row<Real, 32><<<grid_for(th, 256), 256, 0, st>>>(cols, vals, x, y, seg->segment_size, begin, end, alpha, beta); break;
               default: set_error("threads per segment must be 1..32 for row-major Ellpack"); return TNLB_ERR_INVALID_ARGUMENT;
            }
         }
         break;
      }
      case TNLB_SLICED_ELLPACK: {
         if (seg->slices == 0) return TNLB_OK;
         if (col) {
            int G = tps > 0 ? tps : 1;
            if (kernel == TNLB_KERNEL_DEFAULT && tps <= 0) {
               const int64_t mean_w = seg->storage / ((int64_t)seg->slices * kSellSlice);
               G = mean_w >= 256 ? 8 : (mean_w >= 64 ? 4 : (mean_w >= 16 ? 2 : 1));
            }
            const int32_t* so = seg->slice_offsets.as<int32_t>();
            const int32_t* sw = seg->slice_segment_sizes.as<int32_t>();
            switch (G) {
               case 1:
                  // FP64: the slice walk (5-point 1024^2: 18.1 -> 15.7 us);
                  // FP32 entries are half the bytes per slice and the
                  // full-grid launch measured 0.6 us faster there
                  if (sizeof(Real) == 8) {
                     auto* k = k_sell_walk<Real>;
                     const unsigned g = resident_grid((const void*)k, 256, (int64_t)seg->slices * 32, 1);
                     k<<<g, 256, 0, st>>>(cols, vals, x, y, so, sw, seg->slices, begin, end, alpha, beta);
                  }
                  else
                     k_sell_col<Real, 1><<<grid_for(seg->slices, 8), 256, 0, st>>>(cols, vals, x, y, so, sw, seg->slices, begin, end, alpha, beta);
                  break;
               case 2: k_sell_col<Real, 2><<<grid_for(seg->slices, 4), 256, 0, st>>>(cols, vals, x, y, so, sw, seg->slices, begin, end, alpha, beta); break;
               case 4: k_sell_col<Real, 4><<<grid_for(seg->slices, 2), 256, 0, st>>>(cols, vals, x, y, so, sw, seg->slices, begin, end, alpha, beta); break;
               case 8: k_sell_col<Real, 8><<<grid_for(seg->slices, 1), 256, 0, st>>>(cols, vals, x, y, so, sw, seg->slices, begin, end, alpha, beta); break;
               default: set_error("threads per segment must be 1, 2, 4 or 8 for column-major SlicedEllpack"); return TNLB_ERR_INVALID_ARGUMENT;
            }
         }
         else {
            const int G = tps > 0 ? tps : 8;
            const int64_t th = ((int64_t)end - begin) * G;
            const int32_t* so = seg->slice_offsets.as<int32_t>();
            const int32_t* sw = seg->slice_segment_sizes.as<int32_t>();
            switch (G) {
               case 1: k_sell_row<Real, 1><<<grid_for(th, 256), 256, 0, st>>>(cols, vals, x, y, so, sw, begin, end, alpha, beta); break;
               case 2: k_sell_row<Real, 2><<<grid_for(th, 256), 256, 0, st>>>(cols, vals, x, y, so, sw, begin, end, alpha, beta); break;
               case 4: k_sell_row<Real, 4><<<grid_for(th, 256), 256, 0, st>>>(cols, vals, x, y, so, sw, begin, end, alpha, beta); break;
               case 8: k_sell_row<Real, 8><<<grid_for(th, 256), 256, 0, st>>>(cols, vals, x, y, so, sw, begin, end, alpha, beta); break;
               case 16: k_sell_row<Real, 16><<<grid_for(th, 256), 256, 0, st>>>(cols, vals, x, y, so, sw, begin, end, alpha, beta); break;
               case 32: k_sell_row<Real, 32><<<grid_for(th, 256), 256, 0, st>>>(cols, vals, x, y, so, sw, begin, end, alpha, beta); break;
               default: set_error("threads per segment must be 1..32 for row-major SlicedEllpack"); return TNLB_ERR_INVALID_ARGUMENT;
            }
         }
         break;
      }
      case TNLB_CHUNKED_ELLPACK: {
         if (seg->ch_slices == 0) return TNLB_OK;
         auto kern = col ? k_chell<Real, true> : k_chell<Real, false>;
         kern<<<seg->ch_slices, kChunksInSlice, 0, st>>>(
            cols, vals, x, y, seg->ch_slice_size.as<int32_t>(), seg->ch_slice_chunk_size.as<int32_t>(),
            seg->ch_slice_first.as<int32_t>(), seg->ch_slice_pointer.as<int32_t>(),
            seg->ch_segment_to_chunk.as<int32_t>(), begin, end, alpha, beta);
         break;
      }
      case TNLB_BIELLPACK: {
         if (seg->strips == 0) return TNLB_OK;
         auto kern = col ? k_biell_col<Real> : k_biell_row<Real>;
         kern<<<grid_for(seg->strips, 8), 256, 0, st>>>(cols, vals, x, y, seg->bi_perm.as<int32_t>(),
                                                         seg->bi_group_pointers.as<int32_t>(), seg->n, seg->strips,
                                                         begin, end, alpha, beta);
         break;
      }
      default: set_error("format has no Ellpack-family kernel"); return TNLB_ERR_INVALID_ARGUMENT;
   }
   TNLB_CHECK_LAUNCH();
   *launches = 1;
   return TNLB_OK;
}

}  // namespace

tnlb_status spmv_ell_family(const tnlb_segments* seg, tnlb_real real, const int32_t* cols, const void* vals,
                            const void* x, void* y, double alpha, double beta, int32_t begin, int32_t end,
                            tnlb_kernel kernel, int32_t tps, cudaStream_t stream, int* launches)
{
   if (real == TNLB_F64)
      return launch<double>(seg, cols, (const double*)vals, (const double*)x, (double*)y, alpha, beta, begin, end,
                            kernel, tps, stream, launches);
   return launch<float>(seg, cols, (const float*)vals, (const float*)x, (float*)y, (float)alpha, (float)beta, begin,
                        end, kernel, tps, stream, launches);
}

}  // namespace tnlb
