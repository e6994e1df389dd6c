// builders.cu -- GPU builders of the segment formats (Segments::setSegmentsSizes).
//
// The reference builds CSR, Ellpack and SlicedEllpack on the device but
// ChunkedEllpack, BiEllpack and AdaptiveCSR on the host only
// (ChunkedEllpack.hpp:203-214, BiEllpack.hpp:249-251, AdaptiveCSR.hpp:199-201).
// Here every builder runs on the GPU and produces metadata bit-identical to
// the reference's Host builders:
//
//  * CSR         -- exclusive scan of the sizes (CSR.hpp:87-103).
//  * Ellpack     -- max reduction; aligned size rounded to 32 for column-major;
//                   int32 overflow check (Ellpack.hpp:74-96).
//  * SlicedEllpack -- per-slice max (one warp per slice of 32) and an
//                   exclusive scan of max*32 (SlicedEllpack.hpp:116-150).
//  * BiEllpack   -- the reference's per-strip cocktail sort swaps only
//                   strictly smaller-before-larger neighbours, i.e. it is a
//                   stable descending sort; one warp per strip computes every
//                   segment's rank with 32 comparisons, then the 5 group
//                   widths (BiEllpack.hpp:247-342) and an exclusive scan.
//  * ChunkedEllpack -- the greedy slice partition (ChunkedEllpack.hpp:283-310)
//                   is a chain start -> end(start); every end(start) is found
//                   in parallel by binary search in the size prefix sums, and
//                   one block walks the chain through shared-memory windows.
//                   Chunk apportioning per slice (:315-380) runs one block per
//                   slice with IEEE round-to-nearest double division and
//                   multiplication (no FMA), truncated like the reference; the
//                   round-robin leftover loop is replaced by its closed form.
//  * AdaptiveCSR -- findLimit (AdaptiveCSR.hpp:167-192) for every start in
//                   parallel, the same chained walk, then descriptor emission
//                   (:197-230) for the 6 value sizes.
#include <vector>

#include "internal.cuh"

namespace tnlb {
namespace {

// --------------------------------------------------------------- helpers

__global__ void k_fill_i32(int32_t* p, int64_t n, int32_t v)
{
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
      p[i] = v;
}

// ------------------------------------------------------- SlicedEllpack

__global__ void k_sell_slice_max(const int32_t* __restrict__ sizes, int32_t n, int32_t slices,
                                 int32_t* __restrict__ slice_sizes, int32_t* __restrict__ slice_storage)
{
   const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
   const int lane = threadIdx.x & 31;
   if (warp >= slices) return;
   const int64_t g = warp * kSellSlice + lane;
   int32_t v = g < n ? sizes[g] : 0;
#pragma unroll
   for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
   if (lane == 0) {
      slice_sizes[warp] = v;
      slice_storage[warp] = v * kSellSlice;
   }
}

// ----------------------------------------------------------- BiEllpack

// One warp per strip of 32 segments.  perm[original] = strip*32 + rank where
// rank orders sizes descending and keeps the original order among equal
// sizes (the fixed point of the reference's cocktail sort).  Then the raw
// group sizes width*height of groups emptyGroups..4; slot 5 stays 0.
__global__ void k_biell_strips(const int32_t* __restrict__ sizes, int32_t n, int32_t strips, int32_t* __restrict__ perm,
                               int32_t* __restrict__ group_raw)
{
   __shared__ int32_t sorted[8][32];
   const int wib = threadIdx.x >> 5;
   const int64_t strip = (int64_t)blockIdx.x * (blockDim.x >> 5) + wib;
   const int lane = threadIdx.x & 31;
   if (strip >= strips) return;
   const int64_t b = strip * kBiStrip;
   const int cnt = (int)::tnlb::imin64(32, n - b);
   const bool valid = lane < cnt;
   const int32_t s = valid ? sizes[b + lane] : 0;
   int rank = 0;
   for (int j = 0; j < cnt; j++) {
      const int32_t sj = __shfl_sync(0xffffffffu, s, j);
      if (valid && (sj > s || (sj == s && j < lane))) rank++;
   }
   if (valid) {
      perm[b + lane] = (int32_t)(b + rank);
      sorted[wib][rank] = s;
   }
   __syncwarp();
   if (lane < kBiGroups) {
      int emptyGroups = 0;
      if (strip == strips - 1)
         while (cnt <= (1 << (4 - emptyGroups)) - 1) emptyGroups++;
      int32_t v = 0;
      const int g = lane;
      if (g >= emptyGroups && g < 5) {
         const int pos = (1 << (4 - g)) - 1;
         const int32_t allocated = (g == emptyGroups) ? 0 : sorted[wib][(1 << (5 - g)) - 1];
         const int32_t width = sorted[wib][pos] - allocated;
         v = width * (1 << (5 - g));
      }
      group_raw[strip * kBiGroups + g] = v;
   }
}

// ------------------------------------------------------ chained walks
// end[i] is the exclusive end of the greedy block that starts at i.  One
// block follows the chain 0 -> end[0] -> ... -> n, staging windows of end[]
// (and the block type, if any) in shared memory.  For each block it records
// the start and, for AdaptiveCSR, the index of its first descriptor (LONG
// blocks take 8 - count%8 descriptors, AdaptiveCSR.hpp:211-218).
constexpr int kWalkWindow = 6144;

__global__ void k_chain_walk(const int32_t* __restrict__ end, const uint8_t* __restrict__ type, int32_t n,
                             int32_t* __restrict__ starts, int64_t* __restrict__ desc_base,
                             int64_t* __restrict__ counts)
{
   __shared__ int32_t wend[kWalkWindow];
   __shared__ uint8_t wtype[kWalkWindow];
   __shared__ int32_t s_cur;
   __shared__ int64_t s_blocks, s_desc;
   if (threadIdx.x == 0) {
      s_cur = 0;
      s_blocks = 0;
      s_desc = 0;
   }
   __syncthreads();
   while (true) {
      const int32_t base = s_cur;
      if (base >= n) break;
      for (int k = threadIdx.x; k < kWalkWindow; k += blockDim.x) {
         const int64_t g = (int64_t)base + k;
         if (g < n) {
            wend[k] = end[g];
            if (type) wtype[k] = type[g];
         }
      }
      __syncthreads();
      if (threadIdx.x == 0) {
         int32_t cur = base;
         int64_t nb = s_blocks, nd = s_desc;
         while (cur < n && cur < base + kWalkWindow) {
            const int32_t e = wend[cur - base];
            starts[nb] = cur;
            if (desc_base) {
               desc_base[nb] = nd;
               nd += (type && wtype[cur - base] == 0) ? 8 - (nd & 7) : 1;
            }
            nb++;
            cur = e;
         }
         s_cur = cur;
         s_blocks = nb;
         s_desc = nd;
      }
      __syncthreads();
   }
   if (threadIdx.x == 0) {
      counts[0] = s_blocks;
      counts[1] = s_desc;
   }
}

// ------------------------------------------------------ ChunkedEllpack

// end of the slice starting at i: stop after segment j when the slice holds
// >= desired elements, or 256 segments, or the last segment
// (ChunkedEllpack.hpp:293-309).  P = exclusive prefix of sizes (n+1).
__global__ void k_chell_end(const int32_t* __restrict__ P, int32_t n, int32_t* __restrict__ end)
{
   const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (i >= n) return;
   const int64_t desired = (int64_t)kChunksInSlice * kDesiredChunkSize;
   const int64_t pi = P[i];
   int64_t lo = i, hi = ::tnlb::imin64(i + kChunksInSlice, n) - 1;  // candidate last segment
   // first j in [i, hi] with P[j+1] - P[i] >= desired, else hi
   int64_t ans = hi;
   while (lo <= hi) {
      const int64_t mid = (lo + hi) >> 1;
      if ((int64_t)P[mid + 1] - pi >= desired) {
         ans = mid;
         hi = mid - 1;
      }
      else
         lo = mid + 1;
   }
   end[i] = (int32_t)(ans + 1);
}

// One block (256 threads) per slice, one thread per segment (slices hold at
// most 256 segments).  setSlice (ChunkedEllpack.hpp:315-380).
__global__ void k_chell_slice(const int32_t* __restrict__ sizes, const int32_t* __restrict__ P,
                              const int32_t* __restrict__ starts, int32_t slices, int32_t n,
                              int32_t* __restrict__ slice_size, int32_t* __restrict__ slice_first,
                              int32_t* __restrict__ slice_chunk, int32_t* __restrict__ slice_storage,
                              int32_t* __restrict__ seg_to_chunk, int32_t* __restrict__ seg_to_slice,
                              int32_t* __restrict__ seg_ptr_raw)
{
   __shared__ int32_t s_max_len, s_added, s_max_count, s_max_chunk;
   __shared__ int32_t warp_tot[8];
   const int32_t s = blockIdx.x;
   const int32_t begin = starts[s];
   const int32_t end = (s + 1 < slices) ? starts[s + 1] : n;
   const int32_t ssz = end - begin;
   const int32_t allocated = P[end] - P[begin];
   const int t = threadIdx.x;
   const bool valid = t < ssz;
   const int32_t i = begin + t;
   const int32_t size = valid ? sizes[i] : 0;
   if (t == 0) {
      s_max_len = 0;
      s_added = 0;
      s_max_count = 0;
      s_max_chunk = 0;
   }
   __syncthreads();
   const int32_t freeChunks = kChunksInSlice - ssz;
   int32_t added = 0;
   if (valid) {
      double ratio = 0.0;
      if (allocated != 0) ratio = __ddiv_rn((double)size, (double)allocated);
      added = __double2int_rz(__dmul_rn((double)freeChunks, ratio));
      atomicMax(&s_max_len, size);
      atomicAdd(&s_added, added);
   }
   __syncthreads();
   const int32_t remaining = freeChunks - s_added;
   const bool is_max = valid && size == s_max_len;
   // rank among the maximal segments in index order (block prefix count)
   const unsigned ball = __ballot_sync(0xffffffffu, is_max);
   const int lane = t & 31, w = t >> 5;
   if (lane == 0) warp_tot[w] = __popc(ball);
   __syncthreads();
   int32_t before = 0, total_max = 0;
   for (int k = 0; k < 8; k++) {
      if (k < w) before += warp_tot[k];
      total_max += warp_tot[k];
   }
   before += __popc(ball & ((1u << lane) - 1u));
   int32_t chunks = 1 + added;
   if (is_max && total_max > 0)
      chunks += remaining / total_max + (before < remaining % total_max ? 1 : 0);
   if (valid) {
      const int32_t c = (size + chunks - 1) / chunks;
      atomicMax(&s_max_chunk, c);
   }
   __syncthreads();
   const int32_t maxChunk = s_max_chunk;
   // inclusive prefix of chunks within the slice
   int32_t v = valid ? chunks : 0;
   int32_t inc = v;
#pragma unroll
   for (int o = 1; o < 32; o <<= 1) {
      const int32_t x = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += x;
   }
   __syncthreads();
   if (lane == 31) warp_tot[w] = inc;
   __syncthreads();
   int32_t off = 0;
   for (int k = 0; k < w; k++) off += warp_tot[k];
   inc += off;
   if (valid) {
      seg_to_chunk[i] = inc;
      seg_to_slice[i] = s;
      seg_ptr_raw[i + 1] = maxChunk * chunks;
   }
   if (t == 0) {
      slice_size[s] = ssz;
      slice_first[s] = begin;
      slice_chunk[s] = maxChunk;
      slice_storage[s] = kChunksInSlice * maxChunk;
   }
}

__global__ void k_chell_chunks_to_segments(const int32_t* __restrict__ seg_to_chunk,
                                           const int32_t* __restrict__ seg_to_slice,
                                           const int32_t* __restrict__ slice_first, int32_t n,
                                           int32_t* __restrict__ c2s)
{
   const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (i >= n) return;
   const int32_t s = seg_to_slice[i];
   const int32_t first = (i == slice_first[s]) ? 0 : seg_to_chunk[i - 1];
   const int32_t last = seg_to_chunk[i];
   for (int32_t c = first; c < last; c++) c2s[(int64_t)s * kChunksInSlice + c] = (int32_t)i;
}

// ---------------------------------------------------------- AdaptiveCSR

// findLimit from every start (AdaptiveCSR.hpp:167-192): the first row `cur`
// at which the running element count exceeds `limit`; STREAM block
// [start, cur) if cur > start, else the single row as VECTOR (<= 1024
// elements) or LONG; STREAM to the end if the limit is never exceeded.
__global__ void k_acsr_end(const int32_t* __restrict__ off, int32_t n, int64_t limit, int32_t* __restrict__ end,
                           uint8_t* __restrict__ type)
{
   const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (i >= n) return;
   const int64_t oi = off[i];
   int64_t lo = i, hi = n - 1, cur = -1;
   while (lo <= hi) {
      const int64_t mid = (lo + hi) >> 1;
      if ((int64_t)off[mid + 1] - oi > limit) {
         cur = mid;
         hi = mid - 1;
      }
      else
         lo = mid + 1;
   }
   if (cur < 0) {
      end[i] = n;
      type[i] = 1;
   }
   else if (cur > i) {
      end[i] = (int32_t)cur;
      type[i] = 1;
   }
   else {
      end[i] = (int32_t)(i + 1);
      const int64_t len = (int64_t)off[i + 1] - oi;
      type[i] = len <= 2 * 512 ? 2 : 0;
   }
}

__global__ void k_acsr_emit(const int32_t* __restrict__ off, const int32_t* __restrict__ starts,
                            const int64_t* __restrict__ desc_base, const int32_t* __restrict__ end,
                            const uint8_t* __restrict__ type, int64_t blocks, int64_t total, int32_t n,
                            tnlb_acsr_block* __restrict__ out)
{
   const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (b > blocks) return;
   if (b == blocks) {  // closing descriptor (AdaptiveCSR.hpp:228)
      tnlb_acsr_block d{};
      d.type = 2;
      d.first_segment = n;
      out[total] = d;
      return;
   }
   const int32_t st = starts[b];
   const uint8_t t = type[st];
   const int64_t base = desc_base[b];
   if (t == 0) {
      const int32_t wl = 8 - (int32_t)(base & 7);
      for (int32_t idx = 0; idx < wl; idx++) {
         tnlb_acsr_block d{};
         d.type = 0;
         d.first_segment = st;
         d.warp_idx = (uint8_t)idx;
         d.warps_count = (uint8_t)wl;
         out[base + idx] = d;
      }
   }
   else {
      const int32_t e = end[st];
      tnlb_acsr_block d{};
      d.type = t;
      d.first_segment = st;
      d.block_size = off[e] - off[st];
      d.segments_in_block = e - st;
      out[base] = d;
   }
}

tnlb_status build_csr(tnlb_segments* seg, const int32_t* d_sizes, cudaStream_t stream)
{
   TNLB_TRY_STATUS(seg->offsets.alloc(sizeof(int32_t) * ((size_t)seg->n + 1)));
   int64_t total = 0;
   TNLB_TRY_STATUS(exclusive_scan_i32(d_sizes, seg->offsets.as<int32_t>(), seg->n, &total, stream, true));
   seg->elements = total;
   seg->storage = total;
   return TNLB_OK;
}

tnlb_status build_acsr(tnlb_segments* seg, cudaStream_t stream)
{
   const int32_t n = seg->n;
   for (int k = 0; k < 6; k++) seg->acsr_count[k] = 0;
   if (n == 0 || seg->max_size == 0) return TNLB_OK;  // max(offsets) == 0: blocks reset
   DeviceBuffer end, type, starts, base, counts;
   TNLB_TRY_STATUS(end.alloc(sizeof(int32_t) * n));
   TNLB_TRY_STATUS(type.alloc(n));
   TNLB_TRY_STATUS(starts.alloc(sizeof(int32_t) * n));
   TNLB_TRY_STATUS(base.alloc(sizeof(int64_t) * n));
   TNLB_TRY_STATUS(counts.alloc(sizeof(int64_t) * 2));
   for (int k = 0; k < 6; k++) {
      const int64_t sizeOfValue = 1 << k;
      const int64_t limit = (24576 / sizeOfValue) / 8;
      k_acsr_end<<<grid_for(n, 256), 256, 0, stream>>>(seg->offsets.as<int32_t>(), n, limit, end.as<int32_t>(),
                                                        type.as<uint8_t>());
      TNLB_CHECK_LAUNCH();
      k_chain_walk<<<1, 1024, 0, stream>>>(end.as<int32_t>(), type.as<uint8_t>(), n, starts.as<int32_t>(),
                                           base.as<int64_t>(), counts.as<int64_t>());
      TNLB_CHECK_LAUNCH();
      int64_t h[2];
      TNLB_CUDA_TRY(cudaMemcpyAsync(h, counts.ptr, sizeof(h), cudaMemcpyDeviceToHost, stream));
      TNLB_CUDA_TRY(cudaStreamSynchronize(stream));
      const int64_t blocks = h[0], total = h[1];
      TNLB_TRY_STATUS(seg->acsr_blocks[k].alloc(sizeof(tnlb_acsr_block) * (total + 1)));
      k_acsr_emit<<<grid_for(blocks + 1, 256), 256, 0, stream>>>(
         seg->offsets.as<int32_t>(), starts.as<int32_t>(), base.as<int64_t>(), end.as<int32_t>(), type.as<uint8_t>(),
         blocks, total, n, seg->acsr_blocks[k].as<tnlb_acsr_block>());
      TNLB_CHECK_LAUNCH();
      seg->acsr_count[k] = total + 1;
   }
   TNLB_CUDA_TRY(cudaStreamSynchronize(stream));
   return TNLB_OK;
}

tnlb_status build_chell(tnlb_segments* seg, const int32_t* d_sizes, cudaStream_t stream)
{
   const int32_t n = seg->n;
   seg->ch_slices = 0;
   TNLB_TRY_STATUS(seg->ch_segment_pointers.alloc(sizeof(int32_t) * ((size_t)n + 1)));
   TNLB_TRY_STATUS(seg->ch_segment_to_chunk.alloc(sizeof(int32_t) * (size_t)n));
   TNLB_TRY_STATUS(seg->ch_segment_to_slice.alloc(sizeof(int32_t) * (size_t)n));
   TNLB_CUDA_TRY(cudaMemsetAsync(seg->ch_segment_pointers.ptr, 0, sizeof(int32_t), stream));
   if (n == 0) {
      seg->storage = 0;
      for (auto* b : {&seg->ch_slice_size, &seg->ch_slice_chunk_size, &seg->ch_slice_first, &seg->ch_slice_pointer,
                      &seg->ch_chunks_to_segments})
         TNLB_TRY_STATUS(b->alloc(16));
      TNLB_CUDA_TRY(cudaStreamSynchronize(stream));
      return TNLB_OK;
   }
   DeviceBuffer P, end, starts, counts, storage_raw;
   TNLB_TRY_STATUS(P.alloc(sizeof(int32_t) * ((size_t)n + 1)));
   TNLB_TRY_STATUS(exclusive_scan_i32(d_sizes, P.as<int32_t>(), n, nullptr, stream, true));
   TNLB_TRY_STATUS(end.alloc(sizeof(int32_t) * n));
   TNLB_TRY_STATUS(starts.alloc(sizeof(int32_t) * n));
   TNLB_TRY_STATUS(counts.alloc(sizeof(int64_t) * 2));
   k_chell_end<<<grid_for(n, 256), 256, 0, stream>>>(P.as<int32_t>(), n, end.as<int32_t>());
   TNLB_CHECK_LAUNCH();
   k_chain_walk<<<1, 1024, 0, stream>>>(end.as<int32_t>(), nullptr, n, starts.as<int32_t>(), nullptr,
                                        counts.as<int64_t>());
   TNLB_CHECK_LAUNCH();
   int64_t h[2];
   TNLB_CUDA_TRY(cudaMemcpyAsync(h, counts.ptr, sizeof(h), cudaMemcpyDeviceToHost, stream));
   TNLB_CUDA_TRY(cudaStreamSynchronize(stream));
   const int32_t slices = (int32_t)h[0];
   seg->ch_slices = slices;
   TNLB_TRY_STATUS(seg->ch_slice_size.alloc(sizeof(int32_t) * slices));
   TNLB_TRY_STATUS(seg->ch_slice_chunk_size.alloc(sizeof(int32_t) * slices));
   TNLB_TRY_STATUS(seg->ch_slice_first.alloc(sizeof(int32_t) * slices));
   TNLB_TRY_STATUS(seg->ch_slice_pointer.alloc(sizeof(int32_t) * ((size_t)slices + 1)));
   TNLB_TRY_STATUS(storage_raw.alloc(sizeof(int32_t) * slices));
   k_chell_slice<<<slices, kChunksInSlice, 0, stream>>>(
      d_sizes, P.as<int32_t>(), starts.as<int32_t>(), slices, n, seg->ch_slice_size.as<int32_t>(),
      seg->ch_slice_first.as<int32_t>(), seg->ch_slice_chunk_size.as<int32_t>(), storage_raw.as<int32_t>(),
      seg->ch_segment_to_chunk.as<int32_t>(), seg->ch_segment_to_slice.as<int32_t>(),
      seg->ch_segment_pointers.as<int32_t>());
   TNLB_CHECK_LAUNCH();
   int64_t total = 0;
   TNLB_TRY_STATUS(exclusive_scan_i32(storage_raw.as<int32_t>(), seg->ch_slice_pointer.as<int32_t>(), slices, &total,
                                      stream, false));
   TNLB_REQUIRE(total <= INT32_MAX, TNLB_ERR_OVERFLOW, "ChunkedEllpack storage exceeds the int32 index range");
   seg->storage = total;
   TNLB_TRY_STATUS(inclusive_scan_i32_inplace(seg->ch_segment_pointers.as<int32_t>(), (int64_t)n + 1, stream));
   TNLB_TRY_STATUS(seg->ch_chunks_to_segments.alloc(sizeof(int32_t) * (size_t)slices * kChunksInSlice));
   k_chell_chunks_to_segments<<<grid_for(n, 256), 256, 0, stream>>>(
      seg->ch_segment_to_chunk.as<int32_t>(), seg->ch_segment_to_slice.as<int32_t>(),
      seg->ch_slice_first.as<int32_t>(), n, seg->ch_chunks_to_segments.as<int32_t>());
   TNLB_CHECK_LAUNCH();
   TNLB_CUDA_TRY(cudaStreamSynchronize(stream));
   return TNLB_OK;
}

}  // namespace

tnlb_status build_segments(tnlb_segments* seg, const int32_t* d_sizes, cudaStream_t stream)
{
   const int32_t n = seg->n;
   int32_t mx = 0;
   TNLB_TRY_STATUS(reduce_max_i32(d_sizes, n, &mx, stream));
   seg->max_size = mx;
   {
      int64_t sum = 0;
      if (seg->format == TNLB_CSR || seg->format == TNLB_ADAPTIVE_CSR) {
         TNLB_TRY_STATUS(build_csr(seg, d_sizes, stream));
         sum = seg->elements;
      }
      else {
         TNLB_TRY_STATUS(reduce_sum_i64(d_sizes, n, &sum, stream));
      }
      seg->elements = sum;
   }
   switch (seg->format) {
      case TNLB_CSR: {
         TNLB_TRY_STATUS(build_csr_tile_plan(seg, stream));
         return TNLB_OK;
      }
      case TNLB_ADAPTIVE_CSR: {
         TNLB_TRY_STATUS(build_acsr(seg, stream));
         TNLB_TRY_STATUS(build_csr_tile_plan(seg, stream));
         return TNLB_OK;
      }
      case TNLB_ELLPACK: {
         const int64_t aligned =
            seg->organization == TNLB_ROW_MAJOR ? (int64_t)n : ((int64_t)n + kEllAlignment - 1) / kEllAlignment * kEllAlignment;
         // max() over zero segments is the identity of Max, the lowest int
         // (Ellpack.hpp:77); the storage stays 0 since alignedSize is 0.
         seg->segment_size = n > 0 ? mx : INT32_MIN;
         seg->aligned_size = (int32_t)aligned;
         TNLB_REQUIRE(aligned <= INT32_MAX && aligned * (int64_t)mx <= INT32_MAX, TNLB_ERR_OVERFLOW,
                      "Ellpack: multiplication overflow - the storage size required for the segments is larger than "
                      "the maximal value of used index type.");
         seg->storage = n > 0 ? aligned * mx : 0;
         return TNLB_OK;
      }
      case TNLB_SLICED_ELLPACK: {
         const int32_t slices = (n + kSellSlice - 1) / kSellSlice;
         seg->slices = slices;
         TNLB_REQUIRE((int64_t)mx * kSellSlice <= INT32_MAX, TNLB_ERR_OVERFLOW,
                      "SlicedEllpack storage exceeds the int32 index range");
         TNLB_TRY_STATUS(seg->slice_offsets.alloc(sizeof(int32_t) * ((size_t)slices + 1)));
         TNLB_TRY_STATUS(seg->slice_segment_sizes.alloc(sizeof(int32_t) * (size_t)slices));
         DeviceBuffer raw;
         TNLB_TRY_STATUS(raw.alloc(sizeof(int32_t) * (size_t)slices));
         if (slices > 0) {
            k_sell_slice_max<<<grid_for((int64_t)slices * 32, 256), 256, 0, stream>>>(
               d_sizes, n, slices, seg->slice_segment_sizes.as<int32_t>(), raw.as<int32_t>());
            TNLB_CHECK_LAUNCH();
         }
         int64_t total = 0;
         TNLB_TRY_STATUS(
            exclusive_scan_i32(raw.as<int32_t>(), seg->slice_offsets.as<int32_t>(), slices, &total, stream, true));
         seg->storage = total;
         return TNLB_OK;
      }
      case TNLB_BIELLPACK: {
         const int32_t strips = (n + kBiStrip - 1) / kBiStrip;
         seg->strips = strips;
         TNLB_TRY_STATUS(seg->bi_perm.alloc(sizeof(int32_t) * (size_t)n));
         TNLB_TRY_STATUS(seg->bi_group_pointers.alloc(sizeof(int32_t) * ((size_t)strips * kBiGroups + 1)));
         DeviceBuffer raw;
         TNLB_TRY_STATUS(raw.alloc(sizeof(int32_t) * ((size_t)strips * kBiGroups)));
         if (strips > 0) {
            k_biell_strips<<<grid_for(strips, 8), 256, 0, stream>>>(d_sizes, n, strips, seg->bi_perm.as<int32_t>(),
                                                                     raw.as<int32_t>());
            TNLB_CHECK_LAUNCH();
         }
         int64_t total = 0;
         TNLB_TRY_STATUS(exclusive_scan_i32(raw.as<int32_t>(), seg->bi_group_pointers.as<int32_t>(),
                                            (int64_t)strips * kBiGroups, &total, stream, true));
         seg->storage = total;
         return TNLB_OK;
      }
      case TNLB_CHUNKED_ELLPACK: return build_chell(seg, d_sizes, stream);
   }
   set_error("unknown segments format");
   return TNLB_ERR_INVALID_ARGUMENT;
}

}  // namespace tnlb
