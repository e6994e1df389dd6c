// fill.cu -- Segments::getGlobalIndex on the device and the cross-format
// matrix fill (copySparseToSparseMatrix, Matrices/SparseOperations.hpp:106-186).
#include "internal.cuh"
#include "segview.cuh"

namespace tnlb {
namespace {

__global__ void k_global_index(SegView v, const int32_t* __restrict__ segs, const int32_t* __restrict__ locals,
                               int64_t count, int64_t* __restrict__ out)
{
   const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (i < count) out[i] = (segs[i] >= 0 && segs[i] < v.n) ? global_index_of(v, segs[i], locals[i]) : -1;
}

__global__ void k_set_i32(int32_t* p, int64_t n, int32_t value)
{
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
      p[i] = value;
}

// One warp per source row; kept elements (value != 0, column != -1) are
// packed with a ballot prefix count into local slots 0, 1, 2, ...
template <typename Real>
__global__ void k_fill(SegView v, const int32_t* __restrict__ rowptr, const int32_t* __restrict__ src_cols,
                       const Real* __restrict__ src_vals, int32_t* __restrict__ cols, Real* __restrict__ vals,
                       int32_t* __restrict__ error)
{
   const int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
   const int lane = threadIdx.x & 31;
   if (row >= v.n) return;
   const int32_t b = rowptr[row], e = rowptr[row + 1];
   int32_t slot = 0;
   for (int32_t j0 = b; j0 < e; j0 += 32) {
      const int32_t j = j0 + lane;
      int32_t c = -1;
      Real val = 0;
      if (j < e) {
         c = src_cols[j];
         val = src_vals[j];
      }
      const bool kept = j < e && val != Real(0) && c != -1;
      const unsigned m = __ballot_sync(0xffffffffu, kept);
      if (kept) {
         const int32_t local = slot + __popc(m & ((1u << lane) - 1u));
         const int64_t g = global_index_of(v, (int32_t)row, local);
         if (g < 0)
            atomicExch(error, 1);
         else {
            cols[g] = c;
            vals[g] = val;
         }
      }
      slot += __popc(m);
   }
}

// Gather a matrix stored in any format into CSR (rows keep their slot order,
// padding dropped): count pass then copy pass.
__global__ void k_count_row(SegView v, const int32_t* __restrict__ cols, int32_t* __restrict__ cnt)
{
   const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (i >= v.n) return;
   int32_t c = 0;
   for (int32_t k = 0;; k++) {
      const int64_t g = global_index_of(v, (int32_t)i, k);
      if (g < 0) break;
      if (cols[g] >= 0) c++;
   }
   cnt[i] = c;
}

template <typename Real>
__global__ void k_gather_row(SegView v, const int32_t* __restrict__ cols, const Real* __restrict__ vals,
                             const int32_t* __restrict__ rp, int32_t* __restrict__ oc, Real* __restrict__ ov)
{
   const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (i >= v.n) return;
   int32_t o = rp[i];
   for (int32_t k = 0;; k++) {
      const int64_t g = global_index_of(v, (int32_t)i, k);
      if (g < 0) break;
      if (cols[g] >= 0) {
         oc[o] = cols[g];
         ov[o] = vals[g];
         o++;
      }
   }
}

}  // namespace

// CSR copy of a matrix stored in any format: rows keep their slot order
// (ascending columns, as the fill packs them), padding slots are dropped.
tnlb_status gather_csr(const SegView& v, tnlb_real real, const int32_t* cols, const void* vals, DeviceBuffer& rp,
                       DeviceBuffer& oc, DeviceBuffer& ov, cudaStream_t st)
{
   const int32_t n = v.n;
   DeviceBuffer cnt;
   TNLB_TRY_STATUS(cnt.alloc(sizeof(int32_t) * (n > 0 ? n : 1)));
   if (n > 0) {
      k_count_row<<<grid_for(n, 256), 256, 0, st>>>(v, cols, cnt.as<int32_t>());
      TNLB_CHECK_LAUNCH();
   }
   TNLB_TRY_STATUS(rp.alloc(sizeof(int32_t) * ((size_t)n + 1)));
   int64_t nnz = 0;
   TNLB_TRY_STATUS(exclusive_scan_i32(cnt.as<int32_t>(), rp.as<int32_t>(), n, &nnz, st, true));
   const size_t rs = real == TNLB_F64 ? 8 : 4;
   TNLB_TRY_STATUS(oc.alloc(sizeof(int32_t) * (size_t)(nnz > 0 ? nnz : 1)));
   TNLB_TRY_STATUS(ov.alloc(rs * (size_t)(nnz > 0 ? nnz : 1)));
   if (n > 0) {
      if (real == TNLB_F64)
         k_gather_row<double><<<grid_for(n, 256), 256, 0, st>>>(v, cols, (const double*)vals, rp.as<int32_t>(),
                                                                oc.as<int32_t>(), ov.as<double>());
      else
         k_gather_row<float><<<grid_for(n, 256), 256, 0, st>>>(v, cols, (const float*)vals, rp.as<int32_t>(),
                                                               oc.as<int32_t>(), ov.as<float>());
      TNLB_CHECK_LAUNCH();
   }
   return TNLB_OK;
}

tnlb_status global_index(const tnlb_segments* seg, const int32_t* segs, const int32_t* locals, int64_t count,
                         int64_t* out, cudaStream_t stream)
{
   if (count <= 0) return TNLB_OK;
   k_global_index<<<grid_for(count, 256), 256, 0, stream>>>(view_of(seg), segs, locals, count, out);
   TNLB_CHECK_LAUNCH();
   return TNLB_OK;
}

tnlb_status fill_from_csr(const tnlb_segments* seg, tnlb_real real, const int32_t* rowptr, const int32_t* src_cols,
                          const void* src_vals, int32_t* cols, void* vals, cudaStream_t stream)
{
   const size_t rs = real == TNLB_F64 ? 8 : 4;
   if (seg->storage > 0) {
      unsigned g = grid_for(seg->storage, 256);
      if (g > 65536) g = 65536;
      k_set_i32<<<g, 256, 0, stream>>>(cols, seg->storage, -1);
      TNLB_CHECK_LAUNCH();
      TNLB_CUDA_TRY(cudaMemsetAsync(vals, 0, rs * (size_t)seg->storage, stream));
   }
   if (seg->n == 0) return TNLB_OK;
   DeviceBuffer err;
   TNLB_TRY_STATUS(err.alloc(sizeof(int32_t)));
   TNLB_CUDA_TRY(cudaMemsetAsync(err.ptr, 0, sizeof(int32_t), stream));
   const SegView v = view_of(seg);
   if (real == TNLB_F64)
      k_fill<double><<<grid_for((int64_t)seg->n * 32, 256), 256, 0, stream>>>(
         v, rowptr, src_cols, (const double*)src_vals, cols, (double*)vals, err.as<int32_t>());
   else
      k_fill<float><<<grid_for((int64_t)seg->n * 32, 256), 256, 0, stream>>>(
         v, rowptr, src_cols, (const float*)src_vals, cols, (float*)vals, err.as<int32_t>());
   TNLB_CHECK_LAUNCH();
   int32_t h = 0;
   TNLB_CUDA_TRY(cudaMemcpyAsync(&h, err.ptr, sizeof(int32_t), cudaMemcpyDeviceToHost, stream));
   TNLB_CUDA_TRY(cudaStreamSynchronize(stream));
   TNLB_REQUIRE(h == 0, TNLB_ERR_INVALID_ARGUMENT,
                "matrix fill: a row holds more elements than its segment capacity");
   return TNLB_OK;
}

}  // namespace tnlb
