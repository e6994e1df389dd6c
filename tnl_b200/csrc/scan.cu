// scan.cu -- prefix sums and reductions of int32 arrays for the format
// builders: the row-pointer exclusive scan of CSR::setSegmentsSizes
// (Algorithms/Segments/CSR.hpp:87-103), slice offsets (SlicedEllpack.hpp:143),
// group pointers (BiEllpack.hpp:190) and the max/sum reductions
// (Ellpack.hpp:77, SlicedEllpack.hpp:147).
//
// Three passes: per-block totals (int64), a scan of the totals (recursive
// when there are many blocks), and a per-block scan that adds the block's
// offset.  Totals are int64 so that overflow of the int32 result is detected
// on the host instead of wrapping.
#include "internal.cuh"

namespace tnlb {
namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

template <typename T>
__device__ __forceinline__ int64_t block_sum_i64(int64_t v)
{
   __shared__ int64_t s[kScanThreads / 32];
   v = warp_sum(v);
   const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
   if (lane == 0) s[w] = v;
   __syncthreads();
   if (w == 0) {
      v = lane < kScanThreads / 32 ? s[lane] : 0;
      v = warp_sum(v);
   }
   return v;
}

// Exclusive scan of per-thread totals across the block; returns this
// thread's exclusive prefix and writes the block total.
__device__ __forceinline__ int64_t block_exclusive_i64(int64_t v, int64_t* total)
{
   __shared__ int64_t s[kScanThreads / 32];
   const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
   int64_t inc = v;
#pragma unroll
   for (int o = 1; o < 32; o <<= 1) {
      int64_t t = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += t;
   }
   if (lane == 31) s[w] = inc;
   __syncthreads();
   if (w == 0) {
      int64_t x = lane < kScanThreads / 32 ? s[lane] : 0;
      int64_t xi = x;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
         int64_t t = __shfl_up_sync(0xffffffffu, xi, o);
         if (lane >= o) xi += t;
      }
      if (lane < kScanThreads / 32) s[lane] = xi - x;  // exclusive warp offsets
      if (lane == kScanThreads / 32 - 1) *total = xi;
   }
   __syncthreads();
   return s[w] + inc - v;
}

template <typename In>
__global__ void k_block_totals(const In* __restrict__ in, int64_t n, int64_t* __restrict__ totals)
{
   const int64_t base = (int64_t)blockIdx.x * kScanTile;
   int64_t acc = 0;
#pragma unroll
   for (int i = 0; i < kScanItems; i++) {
      const int64_t g = base + (int64_t)i * kScanThreads + threadIdx.x;
      if (g < n) acc += (int64_t)in[g];
   }
   acc = block_sum_i64<int64_t>(acc);
   if (threadIdx.x == 0) totals[blockIdx.x] = acc;
}

// Per-block scan; `offsets` (may be null) holds the exclusive prefix of the
// block totals.  Out may alias In.
template <typename In, typename Out>
__global__ void k_block_scan(const In* in, int64_t n, const int64_t* __restrict__ offsets, Out* out, bool inclusive,
                             int64_t* __restrict__ grand_total)
{
   __shared__ int64_t tile[kScanTile];
   __shared__ int64_t total;
   const int64_t base = (int64_t)blockIdx.x * kScanTile;
#pragma unroll
   for (int i = 0; i < kScanItems; i++) {
      const int64_t g = base + (int64_t)i * kScanThreads + threadIdx.x;
      tile[i * kScanThreads + threadIdx.x] = g < n ? (int64_t)in[g] : 0;
   }
   __syncthreads();
   int64_t local[kScanItems];
   int64_t sum = 0;
#pragma unroll
   for (int i = 0; i < kScanItems; i++) {
      local[i] = tile[threadIdx.x * kScanItems + i];
      sum += local[i];
   }
   int64_t pre = block_exclusive_i64(sum, &total);
   if (offsets) pre += offsets[blockIdx.x];
#pragma unroll
   for (int i = 0; i < kScanItems; i++) {
      const int64_t v = local[i];
      tile[threadIdx.x * kScanItems + i] = inclusive ? pre + v : pre;
      pre += v;
   }
   __syncthreads();
#pragma unroll
   for (int i = 0; i < kScanItems; i++) {
      const int64_t g = base + (int64_t)i * kScanThreads + threadIdx.x;
      if (g < n) out[g] = (Out)tile[i * kScanThreads + threadIdx.x];
   }
   if (grand_total && blockIdx.x == gridDim.x - 1 && threadIdx.x == 0)
      *grand_total = (offsets ? offsets[blockIdx.x] : 0) + total;
}

__global__ void k_block_max(const int32_t* __restrict__ in, int64_t n, int32_t* __restrict__ out)
{
   __shared__ int32_t s[kScanThreads / 32];
   int32_t m = 0;
   for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < n; g += (int64_t)gridDim.x * blockDim.x)
      m = max(m, in[g]);
#pragma unroll
   for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
   if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = m;
   __syncthreads();
   if (threadIdx.x < 32) {
      m = threadIdx.x < kScanThreads / 32 ? s[threadIdx.x] : 0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
      if (threadIdx.x == 0) atomicMax(out, m);
   }
}

// Exclusive scan of int64 block totals in place (recursive).
tnlb_status scan_totals(int64_t* d, int64_t n, cudaStream_t stream)
{
   const int64_t blocks = (n + kScanTile - 1) / kScanTile;
   if (blocks <= 1) {
      k_block_scan<int64_t, int64_t><<<1, kScanThreads, 0, stream>>>(d, n, nullptr, d, false, nullptr);
      TNLB_CHECK_LAUNCH();
      return TNLB_OK;
   }
   DeviceBuffer t;
   TNLB_TRY_STATUS(t.alloc(sizeof(int64_t) * blocks));
   k_block_totals<int64_t><<<(unsigned)blocks, kScanThreads, 0, stream>>>(d, n, t.as<int64_t>());
   TNLB_CHECK_LAUNCH();
   TNLB_TRY_STATUS(scan_totals(t.as<int64_t>(), blocks, stream));
   k_block_scan<int64_t, int64_t><<<(unsigned)blocks, kScanThreads, 0, stream>>>(d, n, t.as<int64_t>(), d, false,
                                                                                   nullptr);
   TNLB_CHECK_LAUNCH();
   TNLB_CUDA_TRY(cudaStreamSynchronize(stream));
   return TNLB_OK;
}

template <bool Inclusive>
tnlb_status scan_i32(const int32_t* d_in, int32_t* d_out, int64_t n, int64_t* h_total, cudaStream_t stream,
                     bool append_total)
{
   const int64_t blocks = (n + kScanTile - 1) / kScanTile;
   DeviceBuffer totals, grand;
   TNLB_TRY_STATUS(grand.alloc(sizeof(int64_t)));
   TNLB_CUDA_TRY(cudaMemsetAsync(grand.ptr, 0, sizeof(int64_t), stream));
   if (n > 0) {
      TNLB_TRY_STATUS(totals.alloc(sizeof(int64_t) * blocks));
      k_block_totals<int32_t><<<(unsigned)blocks, kScanThreads, 0, stream>>>(d_in, n, totals.as<int64_t>());
      TNLB_CHECK_LAUNCH();
      TNLB_TRY_STATUS(scan_totals(totals.as<int64_t>(), blocks, stream));
      k_block_scan<int32_t, int32_t><<<(unsigned)blocks, kScanThreads, 0, stream>>>(
         d_in, n, totals.as<int64_t>(), d_out, Inclusive, grand.as<int64_t>());
      TNLB_CHECK_LAUNCH();
   }
   int64_t total = 0;
   TNLB_CUDA_TRY(cudaMemcpyAsync(&total, grand.ptr, sizeof(int64_t), cudaMemcpyDeviceToHost, stream));
   TNLB_CUDA_TRY(cudaStreamSynchronize(stream));
   if (h_total) *h_total = total;
   if (append_total) {
      TNLB_REQUIRE(total <= INT32_MAX, TNLB_ERR_OVERFLOW,
                   "prefix sum exceeds the int32 index range (" + std::to_string(total) + ")");
      const int32_t t32 = (int32_t)total;
      TNLB_CUDA_TRY(cudaMemcpyAsync(d_out + n, &t32, sizeof(int32_t), cudaMemcpyHostToDevice, stream));
      TNLB_CUDA_TRY(cudaStreamSynchronize(stream));
   }
   return TNLB_OK;
}

}  // namespace

tnlb_status exclusive_scan_i32(const int32_t* d_in, int32_t* d_out, int64_t n, int64_t* h_total, cudaStream_t stream,
                               bool append_total)
{
   return scan_i32<false>(d_in, d_out, n, h_total, stream, append_total);
}

tnlb_status inclusive_scan_i32_inplace(int32_t* d_data, int64_t n, cudaStream_t stream)
{
   return scan_i32<true>(d_data, d_data, n, nullptr, stream, false);
}

tnlb_status reduce_max_i32(const int32_t* d_in, int64_t n, int32_t* h_max, cudaStream_t stream)
{
   DeviceBuffer m;
   TNLB_TRY_STATUS(m.alloc(sizeof(int32_t)));
   TNLB_CUDA_TRY(cudaMemsetAsync(m.ptr, 0, sizeof(int32_t), stream));
   if (n > 0) {
      unsigned g = grid_for(n, kScanThreads * 8);
      if (g > 4096) g = 4096;
      k_block_max<<<g, kScanThreads, 0, stream>>>(d_in, n, m.as<int32_t>());
      TNLB_CHECK_LAUNCH();
   }
   TNLB_CUDA_TRY(cudaMemcpyAsync(h_max, m.ptr, sizeof(int32_t), cudaMemcpyDeviceToHost, stream));
   TNLB_CUDA_TRY(cudaStreamSynchronize(stream));
   return TNLB_OK;
}

tnlb_status reduce_sum_i64(const int32_t* d_in, int64_t n, int64_t* h_sum, cudaStream_t stream)
{
   DeviceBuffer tmp;
   TNLB_TRY_STATUS(tmp.alloc(sizeof(int32_t) * (n + 1)));
   return exclusive_scan_i32(d_in, tmp.as<int32_t>(), n, h_sum, stream, false);
}

}  // namespace tnlb
