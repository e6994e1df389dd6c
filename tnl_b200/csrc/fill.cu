// fill.cu -- Segments::getGlobalIndex on the device and the cross-format
// matrix fill (copySparseToSparseMatrix, Matrices/SparseOperations.hpp:106-186).
#include "internal.cuh"

namespace tnlb {
namespace {

// Device view of the metadata needed by getGlobalIndex.
struct SegView {
   int32_t format, colmajor, n;
   const int32_t* offsets;
   int32_t segment_size, aligned_size;
   const int32_t *slice_off, *slice_w;
   const int32_t *seg_to_chunk, *seg_to_slice, *sl_chunk, *sl_first, *sl_ptr;
   const int32_t *perm, *gp;
};

SegView view_of(const tnlb_segments* s)
{
   SegView v;
   v.format = s->format;
   v.colmajor = s->organization == TNLB_COLUMN_MAJOR;
   v.n = s->n;
   v.offsets = s->offsets.as<int32_t>();
   v.segment_size = s->segment_size;
   v.aligned_size = s->aligned_size;
   v.slice_off = s->slice_offsets.as<int32_t>();
   v.slice_w = s->slice_segment_sizes.as<int32_t>();
   v.seg_to_chunk = s->ch_segment_to_chunk.as<int32_t>();
   v.seg_to_slice = s->ch_segment_to_slice.as<int32_t>();
   v.sl_chunk = s->ch_slice_chunk_size.as<int32_t>();
   v.sl_first = s->ch_slice_first.as<int32_t>();
   v.sl_ptr = s->ch_slice_pointer.as<int32_t>();
   v.perm = s->bi_perm.as<int32_t>();
   v.gp = s->bi_group_pointers.as<int32_t>();
   return v;
}

// getGlobalIndex: EllpackBase.hpp:110-117, SlicedEllpackBase.hpp:121-145,
// detail/ChunkedEllpack.h:86-113, detail/BiEllpack.h:134-163.  -1 when the
// local index is beyond the segment's capacity.
__device__ int64_t global_index_of(const SegView& v, int32_t seg, int32_t local)
{
   switch (v.format) {
      case TNLB_CSR:
      case TNLB_ADAPTIVE_CSR: {
         const int32_t b = v.offsets[seg];
         return local < v.offsets[seg + 1] - b ? (int64_t)b + local : -1;
      }
      case TNLB_ELLPACK:
         if (local >= v.segment_size) return -1;
         return v.colmajor ? (int64_t)seg + (int64_t)v.aligned_size * local : (int64_t)seg * v.segment_size + local;
      case TNLB_SLICED_ELLPACK: {
         const int32_t sl = seg / kSellSlice, in = seg % kSellSlice;
         const int32_t w = v.slice_w[sl];
         if (local >= w) return -1;
         const int64_t off = v.slice_off[sl];
         return v.colmajor ? off + in + (int64_t)kSellSlice * local : off + (int64_t)in * w + local;
      }
      case TNLB_CHUNKED_ELLPACK: {
         const int32_t sl = v.seg_to_slice[seg];
         const int32_t first = seg == v.sl_first[sl] ? 0 : v.seg_to_chunk[seg - 1];
         const int32_t cs = v.sl_chunk[sl];
         if (local >= (v.seg_to_chunk[seg] - first) * cs) return -1;
         const int64_t off = v.sl_ptr[sl];
         if (!v.colmajor) return off + (int64_t)first * cs + local;
         return off + (int64_t)(local % cs) * kChunksInSlice + first + local / cs;
      }
      case TNLB_BIELLPACK: {
         const int32_t strip = seg / kBiStrip;
         const int32_t p = v.perm[seg] - strip * kBiStrip;
         int groups = 0;
         for (int i = 0, bis = 1; i < kBiGroups; i++, bis *= 2)
            if (p < bis) {
               groups = kBiGroups - i;
               break;
            }
         const int32_t* g = v.gp + (int64_t)strip * kBiGroups;
         int64_t base = g[0];
         int h = 32;
         for (int grp = 0; grp < groups; grp++, h >>= 1) {
            const int32_t gs = g[grp + 1] - g[grp];
            if (gs == 0) continue;
            const int32_t w = gs / h;
            if (local >= w) {
               local -= w;
               base += gs;
            }
            else
               return v.colmajor ? base + p + (int64_t)local * h : base + (int64_t)p * w + local;
         }
         return -1;
      }
   }
   return -1;
}

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

}  // namespace

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
