// reduce.cuh -- deterministic grid reductions for the solver kernels.
//
// Each block writes its partial sums; the last block to arrive (atomic
// ticket after a memory fence) adds all partials in index order, so the
// result does not depend on which block finishes last.  The ticket counter
// is reset by that block, ready for the next launch on the same stream.
// Scalars stay in device memory: no host round trip per dot product (the
// reference copies every dot and norm to the host,
// Algorithms/detail/Reduction.hpp:273-320).
#pragma once

#include <mutex>
#include <unordered_map>

#include "internal.cuh"

namespace tnlb {

constexpr int kRedThreads = 256;
constexpr int kRedMaxBlocks = 148 * 8;  // grid-stride vector kernels use <= this many blocks

struct RedWork {
   double* partials;   // [kRedMaxBlocks * kRedSlots]
   unsigned* counter;  // ticket
};
constexpr int kRedSlots = 4;  // up to 4 simultaneous sums per kernel

inline unsigned vec_grid(int64_t n)
{
   int64_t g = (n + kRedThreads * 4 - 1) / (kRedThreads * 4);
   if (g < 1) g = 1;
   if (g > kRedMaxBlocks) g = kRedMaxBlocks;
   return (unsigned)g;
}

// Grid of a grid-stride kernel: the blocks of `threads` threads that
// `kernel` keeps resident at once on the whole device (its occupancy times
// the SM count, queried once per kernel), at most kRedMaxBlocks and at most
// one block per threads * per_thread items -- so no partial last wave.
inline unsigned resident_grid(const void* kernel, int threads, int64_t n, int64_t per_thread)
{
   static std::mutex mu;
   static std::unordered_map<const void*, int> occupancy;
   static int sms = 0;
   int occ = 0;
   {
      std::lock_guard<std::mutex> lock(mu);
      if (sms == 0) {
         int dev = 0, v = 0;
         if (cudaGetDevice(&dev) == cudaSuccess &&
             cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && v > 0)
            sms = v;
         else
            sms = 148;
      }
      auto it = occupancy.find(kernel);
      if (it == occupancy.end()) {
         int v = 0;
         if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, kernel, threads, 0) != cudaSuccess || v < 1) {
            cudaGetLastError();
            v = 1;
         }
         occupancy.emplace(kernel, v);
         occ = v;
      }
      else
         occ = it->second;
   }
   int64_t g = (n + (int64_t)threads * per_thread - 1) / ((int64_t)threads * per_thread);
   const int64_t cap = (int64_t)occ * sms;
   if (g > cap) g = cap;
   if (g > kRedMaxBlocks) g = kRedMaxBlocks;
   if (g < 1) g = 1;
   return (unsigned)g;
}

// Block sum; the result is valid in thread 0.
__device__ __forceinline__ double block_sum(double v)
{
   __shared__ double s_ws[kRedThreads / 32];
   const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
   v = warp_sum(v);
   __syncthreads();
   if (lane == 0) s_ws[w] = v;
   __syncthreads();
   if (w == 0) {
      v = lane < kRedThreads / 32 ? s_ws[lane] : 0.0;
      v = warp_sum(v);
   }
   return v;
}

// Writes K block partials and returns true in every thread of the last block.
template <int K>
__device__ __forceinline__ bool publish_and_arrive(const double (&v)[K], RedWork w)
{
   __shared__ bool s_last;
   double r[K];
#pragma unroll
   for (int k = 0; k < K; k++) r[k] = block_sum(v[k]);
   if (threadIdx.x == 0) {
#pragma unroll
      for (int k = 0; k < K; k++) w.partials[(size_t)k * kRedMaxBlocks + blockIdx.x] = r[k];
      __threadfence();
      const unsigned t = atomicAdd(w.counter, 1u);
      s_last = (t == gridDim.x - 1);
   }
   __syncthreads();
   return s_last;
}

// In the last block: totals of the K partial arrays (valid in thread 0),
// summed in block-index order.  Resets the ticket.
template <int K>
__device__ __forceinline__ void gather_totals(double (&out)[K], RedWork w)
{
#pragma unroll
   for (int k = 0; k < K; k++) {
      double v = 0.0;
      for (unsigned i = threadIdx.x; i < gridDim.x; i += kRedThreads) v += __ldcg(w.partials + (size_t)k * kRedMaxBlocks + i);
      out[k] = block_sum(v);
   }
   if (threadIdx.x == 0) *w.counter = 0;
}

}  // namespace tnlb
