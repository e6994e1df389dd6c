// segview.cuh -- device view of segment metadata and Segments::getGlobalIndex.
#pragma once

#include "internal.cuh"

namespace tnlb {

// Device view of the metadata needed by getGlobalIndex.
struct SegView {
   int32_t format, colmajor, n;
   const int32_t* offsets;
   int32_t segment_size, aligned_size;
   const int32_t *slice_off, *slice_w;
   const int32_t *seg_to_chunk, *seg_to_slice, *sl_chunk, *sl_first, *sl_ptr;
   const int32_t *perm, *gp;
};

inline SegView view_of(const tnlb_segments* s)
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
__device__ inline int64_t global_index_of(const SegView& v, int32_t seg, int32_t local)
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


// CSR copy of a matrix in any format (fill.cu).
tnlb_status gather_csr(const SegView& v, tnlb_real real, const int32_t* cols, const void* vals, DeviceBuffer& rp,
                       DeviceBuffer& oc, DeviceBuffer& ov, cudaStream_t st);

}  // namespace tnlb
