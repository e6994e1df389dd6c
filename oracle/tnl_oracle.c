/*
 * tnl_oracle.c -- CPU restatement of TNL's sparse formats, SpMV and Krylov
 * solvers, used ONLY as the checker.
 *
 * TEST INFRASTRUCTURE.  Nothing in the product (libtnlb200.so, the tnl_b200
 * package, the C++ drop-in headers) links, loads or calls this file.  Only
 * tests/, __graft_entry__.smoke() and the cpu_baseline leg of bench.py may
 * load the library built from it, and only to check or to time the CPU path.
 *
 * Every function restates the algorithm of the reference (TNL 0.4.0,
 * src/TNL/...) in plain C; the file:line each follows is cited beside it.
 * The restatement is pinned in tests/test_oracle.py against
 *   (1) the known-answer vectors of the reference's own unit tests
 *       (src/UnitTests/Matrices/SparseMatrixVectorProductTest.hpp), and
 *   (2) the reference itself, compiled from its headers into oracle/_ref
 *       (oracle/ref_tnl.cpp), on the same seeded inputs -- metadata is
 *       compared with ==, SpMV bit-for-bit where the summation order is the
 *       same, solver iteration counts and residuals to rounding.
 *
 * Index type is int32 (the configurations use int32 indices); sizes that can
 * exceed int32 (Ellpack storage) are checked the way the reference checks.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_OK 0
#define ORC_ERR_INVALID 1
#define ORC_ERR_OVERFLOW 2
#define ORC_ERR_BREAKDOWN 3

enum { ORC_CSR = 0, ORC_ELLPACK = 1, ORC_SLICED_ELLPACK = 2, ORC_CHUNKED_ELLPACK = 3, ORC_BIELLPACK = 4 };

/* ------------------------------------------------------------------------ */
/* Builders                                                                 */
/* ------------------------------------------------------------------------ */

/* CSR::setSegmentsSizes -- offsets = exclusiveScan([sizes..., 0])
 * (Algorithms/Segments/CSR.hpp:87-103). */
void orc_csr_build(const int32_t* sizes, int32_t n, int32_t* offsets)
{
   int32_t acc = 0;
   for (int32_t i = 0; i < n; i++) {
      offsets[i] = acc;
      acc += sizes[i];
   }
   offsets[n] = acc;
}

/* Ellpack::setSegmentsSizes -- segmentSize = max(sizes); alignedSize = n
 * (row-major) or roundUp(n, Alignment=32) (column-major); overflow of
 * alignedSize*segmentSize in Index throws std::overflow_error
 * (Algorithms/Segments/Ellpack.hpp:74-96, Ellpack.h:40). */
int orc_ellpack_build(const int32_t* sizes, int32_t n, int colmajor, int32_t* segmentSize, int32_t* alignedSize)
{
   /* max() of an empty vector is the identity of Max, the lowest int */
   int32_t mx = n > 0 ? 0 : INT32_MIN;
   for (int32_t i = 0; i < n; i++)
      if (sizes[i] > mx) mx = sizes[i];
   int64_t aligned = colmajor ? ((int64_t)(n + 31) / 32) * 32 : n;
   *segmentSize = mx;
   *alignedSize = (int32_t)aligned;
   if (aligned > INT32_MAX || aligned * (int64_t)mx > INT32_MAX || aligned * (int64_t)mx < INT32_MIN) return ORC_ERR_OVERFLOW;
   return ORC_OK;
}

/* SlicedEllpack::setSegmentsSizes -- per slice of 32 segments the max size
 * (virtual segments past n count as 0), sliceOffsets = exclusiveScan(max*32)
 * (Algorithms/Segments/SlicedEllpack.hpp:116-150).  Returns the storage
 * size (sliceOffsets[slices]) or -1 on int32 overflow. */
int64_t orc_sell_build(const int32_t* sizes, int32_t n, int32_t* sliceOffsets, int32_t* sliceSegmentSizes)
{
   const int32_t slices = (n + 31) / 32;
   int64_t acc = 0;
   for (int32_t s = 0; s < slices; s++) {
      int32_t mx = 0;
      for (int32_t k = 0; k < 32; k++) {
         int64_t g = (int64_t)s * 32 + k;
         int32_t v = g < n ? sizes[g] : 0;
         if (v > mx) mx = v;
      }
      sliceSegmentSizes[s] = mx;
      sliceOffsets[s] = (int32_t)acc;
      acc += (int64_t)mx * 32;
      if (acc > INT32_MAX) return -1;
   }
   sliceOffsets[slices] = (int32_t)acc;
   return acc;
}

/* ChunkedEllpack::resolveSliceSizes -- greedy slices: add segments until
 * the slice holds >= chunksInSlice*desiredChunkSize elements or
 * chunksInSlice segments (Algorithms/Segments/ChunkedEllpack.hpp:283-310).
 * Returns the number of slices; fills size/firstSegment/pointer(temp). */
int32_t orc_chell_slices(const int32_t* sizes, int32_t n, int32_t chunksInSlice, int32_t desiredChunkSize,
                         int32_t* sliceSize, int32_t* sliceFirst, int32_t* sliceAlloc)
{
   const int32_t desired = chunksInSlice * desiredChunkSize;
   int32_t seg = 0, ssize = 0, alloc = 0, ns = 0;
   while (seg < n) {
      alloc += sizes[seg];
      ssize++;
      seg++;
      if (alloc < desired)
         if (seg < n && ssize < chunksInSlice) continue;
      if (sliceSize) {
         sliceSize[ns] = ssize;
         sliceFirst[ns] = seg - ssize;
         sliceAlloc[ns] = alloc;
      }
      ssize = 0;
      ns++;
      alloc = 0;
   }
   return ns;
}

/* ChunkedEllpack::setSegmentsSizes + setSlice (ChunkedEllpack.hpp:158-215,
 * 315-380).  Chunk apportioning uses the reference's IEEE double ratio
 * (double)size/(double)allocated, times freeChunks, truncated toward zero;
 * leftover chunks go round-robin to the segments of maximal size.
 * segmentToChunk[i] = (exclusive) end chunk of segment i within its slice;
 * segmentPointers = inclusive scan of chunkSize*chunks;
 * chunksToSegments has numberOfSlices*chunksInSlice entries.
 * Returns 0, or ORC_ERR_OVERFLOW if the storage exceeds int32. */
int orc_chell_build(const int32_t* sizes, int32_t n, int32_t chunksInSlice, int32_t desiredChunkSize, int32_t numberOfSlices,
                    int32_t* sliceSize, int32_t* sliceChunkSize, int32_t* sliceFirst, int32_t* slicePointer,
                    int32_t* segmentToChunk, int32_t* segmentToSlice, int32_t* segmentPointers, int32_t* chunksToSegments,
                    int32_t* storageSize)
{
   int32_t* sliceAlloc = (int32_t*)malloc(sizeof(int32_t) * (size_t)(numberOfSlices > 0 ? numberOfSlices : 1));
   int32_t ns = orc_chell_slices(sizes, n, chunksInSlice, desiredChunkSize, sliceSize, sliceFirst, sliceAlloc);
   if (ns != numberOfSlices) {
      free(sliceAlloc);
      return ORC_ERR_INVALID;
   }
   int64_t elementsToAllocation = 0;
   if (n >= 0) segmentPointers[0] = 0;
   for (int32_t s = 0; s < ns; s++) {
      const int32_t ssz = sliceSize[s], begin = sliceFirst[s], end = begin + ssz;
      const int32_t allocated = sliceAlloc[s];
      int32_t freeChunks = chunksInSlice - ssz;
      for (int32_t i = begin; i < end; i++) segmentToChunk[i] = 1;
      int32_t totalAdded = 0;
      int32_t maxLen = sizes[begin];
      for (int32_t i = begin; i < end; i++) {
         double ratio = 0.0;
         if (allocated != 0) ratio = (double)sizes[i] / (double)allocated;
         const int32_t added = (int32_t)((double)freeChunks * ratio);
         totalAdded += added;
         segmentToChunk[i] += added;
         if (maxLen < sizes[i]) maxLen = sizes[i];
      }
      freeChunks -= totalAdded;
      while (freeChunks)
         for (int32_t i = begin; i < end && freeChunks; i++)
            if (sizes[i] == maxLen) {
               segmentToChunk[i]++;
               freeChunks--;
            }
      int32_t maxChunk = 0;
      for (int32_t i = begin; i < end; i++) {
         int32_t c = (sizes[i] + segmentToChunk[i] - 1) / segmentToChunk[i];
         if (c > maxChunk) maxChunk = c;
      }
      sliceChunkSize[s] = maxChunk;
      slicePointer[s] = (int32_t)elementsToAllocation;
      elementsToAllocation += (int64_t)chunksInSlice * maxChunk;
      if (elementsToAllocation > INT32_MAX) {
         free(sliceAlloc);
         return ORC_ERR_OVERFLOW;
      }
      for (int32_t i = begin; i < end; i++) segmentToSlice[i] = s;
      for (int32_t i = begin; i < end; i++) segmentPointers[i + 1] = maxChunk * segmentToChunk[i];
      for (int32_t j = begin + 1; j < end; j++) segmentToChunk[j] += segmentToChunk[j - 1];
   }
   /* inplaceInclusiveScan( segmentPointers ) */
   for (int32_t i = 1; i <= n; i++) segmentPointers[i] += segmentPointers[i - 1];
   /* chunksToSegmentsMapping (ChunkedEllpack.hpp:174-186) */
   int64_t chunkIdx = 0;
   for (int32_t seg = 0; seg < n; seg++) {
      const int32_t s = segmentToSlice[seg];
      int32_t first = 0;
      if (seg != sliceFirst[s]) first = segmentToChunk[seg - 1];
      const int32_t cnt = segmentToChunk[seg] - first;
      for (int32_t i = 0; i < cnt; i++) chunksToSegments[chunkIdx++] = seg;
   }
   *storageSize = (int32_t)elementsToAllocation;
   free(sliceAlloc);
   return ORC_OK;
}

/* BiEllpack::initSegmentsPermutation (Algorithms/Segments/BiEllpack.hpp:247-301):
 * per strip of 32 segments a cocktail-shaker sort by descending size that
 * swaps only strictly smaller-before-larger neighbours, i.e. a STABLE
 * descending sort; perm[original] = sorted position.  Restated here as the
 * equivalent rank: #(larger) + #(equal and earlier).
 * BiEllpack::initGroupPointers (BiEllpack.hpp:306-342): per strip 6 slots;
 * group g in [emptyGroups,5) has height 32>>g and width
 * size(sorted pos (16>>g)-1) - columns already allocated; slot 5 stays 0;
 * then an exclusive scan.  Returns the storage size or -1 on overflow. */
int64_t orc_biell_build(const int32_t* sizes, int32_t n, int32_t* perm, int32_t* groupPointers)
{
   const int32_t strips = (n + 31) / 32;
   const int32_t G = 6; /* log2(32) + 1 */
   for (int32_t st = 0; st < strips; st++) {
      const int32_t b = st * 32;
      const int32_t e = (b + 32 < n) ? b + 32 : n;
      int32_t bySorted[32];
      for (int32_t i = b; i < e; i++) {
         int32_t rank = 0;
         for (int32_t j = b; j < e; j++)
            if (sizes[j] > sizes[i] || (sizes[j] == sizes[i] && j < i)) rank++;
         perm[i] = b + rank;
         bySorted[rank] = sizes[i];
      }
      const int32_t cnt = e - b;
      int32_t emptyGroups = 0;
      if (st == strips - 1)
         while (cnt <= (1 << (4 - emptyGroups)) - 1) emptyGroups++;
      for (int32_t g = 0; g < G; g++) groupPointers[st * G + g] = 0;
      int32_t allocated = 0;
      for (int32_t g = emptyGroups; g < 5; g++) {
         const int32_t pos = (1 << (4 - g)) - 1;
         const int32_t width = bySorted[pos] - allocated;
         const int32_t height = 1 << (5 - g);
         groupPointers[st * G + g] = width * height;
         allocated = bySorted[pos];
      }
   }
   int64_t acc = 0;
   const int64_t total = (int64_t)strips * G;
   for (int64_t i = 0; i < total; i++) {
      int32_t v = groupPointers[i];
      groupPointers[i] = (int32_t)acc;
      acc += v;
      if (acc > INT32_MAX) return -1;
   }
   groupPointers[total] = (int32_t)acc;
   return acc;
}

/* AdaptiveCSR block descriptors for one value size (AdaptiveCSR.hpp:167-230,
 * findLimit :167-192; parameters detail/CSRAdaptiveKernelParameters.h:12-109:
 * StreamedSharedElementsPerWarp = 24576/SizeOfValue/8, MaxAdaptiveElements
 * PerWarp = 512, 8 warps per 256-thread block).  Descriptor fields follow
 * the non-union layout (detail/CSRAdaptiveKernelBlockDescriptor.h:134-199):
 * type (LONG=0, STREAM=1, VECTOR=2), firstSegment, blockSize, segmentsInBlock,
 * warpIdx, warpsCount.  LONG and the closing descriptor leave blockSize and
 * segmentsInBlock unset in the reference; here they are written as 0.
 * With out arrays NULL only the descriptor count is returned. */
int64_t orc_acsr_blocks(const int32_t* offsets, int32_t n, int32_t sizeOfValue, uint8_t* type, int32_t* first,
                        int32_t* blockSize, int32_t* segsInBlock, uint8_t* warpIdx, uint8_t* warpsCount)
{
   int32_t mx = 0;
   for (int32_t i = 0; i <= n; i++)
      if (offsets[i] > mx) mx = offsets[i];
   if (mx == 0) return 0; /* all blocks arrays are reset */
   const uint64_t streamPerWarp = (uint64_t)(24576 / sizeOfValue) / 8;
   const uint64_t maxAdaptive = 512;
   const int32_t rows = n + 1;
   int32_t start = 0, nextStart = 0;
   int64_t cnt = 0;
#define EMIT(T, F, BS, SIB, WI, WC)           \
   do {                                       \
      if (type) {                             \
         type[cnt] = (uint8_t)(T);            \
         first[cnt] = (F);                    \
         blockSize[cnt] = (BS);               \
         segsInBlock[cnt] = (SIB);            \
         warpIdx[cnt] = (uint8_t)(WI);        \
         warpsCount[cnt] = (uint8_t)(WC);     \
      }                                       \
      cnt++;                                  \
   } while (0)
   while (nextStart != rows - 1) {
      /* findLimit */
      int t = 1; /* STREAM */
      uint64_t sum = 0;
      int32_t limit = rows - 1;
      for (int32_t cur = start; cur < rows - 1; cur++) {
         sum += (uint64_t)(offsets[cur + 1] - offsets[cur]);
         if (sum > streamPerWarp) {
            if (cur - start > 0) {
               t = 1;
               limit = cur;
            }
            else {
               t = (sum <= 2 * maxAdaptive) ? 2 : 0;
               limit = cur + 1;
            }
            goto found;
         }
      }
      t = 1;
      limit = rows - 1;
   found:
      nextStart = limit;
      if (t == 0) {
         const int64_t warpsPerBlock = 8;
         int64_t warpsLeft = ((cnt + warpsPerBlock - 1) / warpsPerBlock) * warpsPerBlock - cnt;
         if (warpsLeft == 0) warpsLeft = warpsPerBlock;
         for (int64_t idx = 0; idx < warpsLeft; idx++) EMIT(0, start, 0, 0, idx, warpsLeft);
      }
      else {
         EMIT(t, start, offsets[nextStart] - offsets[start], nextStart - start, 0, 0);
      }
      start = nextStart;
   }
   EMIT(2, nextStart, 0, 0, 0, 0);
#undef EMIT
   return cnt;
}

/* ------------------------------------------------------------------------ */
/* Index maps                                                               */
/* ------------------------------------------------------------------------ */

typedef struct {
   int32_t kind;
   int32_t colmajor;
   int32_t n;
   int32_t storage;
   /* CSR */
   const int32_t* offsets;
   /* Ellpack */
   int32_t segmentSize;
   int32_t alignedSize;
   /* SlicedEllpack (slice size 32) */
   const int32_t* sliceOffsets;
   const int32_t* sliceSegmentSizes;
   /* ChunkedEllpack */
   int32_t chunksInSlice;
   const int32_t* segmentToChunk;
   const int32_t* segmentToSlice;
   const int32_t* sliceChunkSize;
   const int32_t* sliceFirst;
   const int32_t* slicePointer;
   /* BiEllpack */
   const int32_t* perm;
   const int32_t* groupPointers;
} orc_segments;

/* Number of BiEllpack groups a segment takes part in: sorted position p in
 * its strip -> 6 - (number of halvings until p < 2^k)
 * (detail/BiEllpack.h:45-59). */
static int32_t biell_active_groups(int32_t p)
{
   int32_t bis = 1;
   for (int32_t i = 0; i < 6; i++) {
      if (p < bis) return 6 - i;
      bis *= 2;
   }
   return -1;
}

/* Capacity (slots) of one segment in its format. */
int32_t orc_segment_capacity(const orc_segments* s, int32_t seg)
{
   switch (s->kind) {
      case ORC_CSR: return s->offsets[seg + 1] - s->offsets[seg];
      case ORC_ELLPACK: return s->segmentSize;
      case ORC_SLICED_ELLPACK: return s->sliceSegmentSizes[seg / 32];
      case ORC_CHUNKED_ELLPACK: {
         /* detail/ChunkedEllpack.h:50-64 */
         const int32_t sl = s->segmentToSlice[seg];
         int32_t first = 0;
         if (seg != s->sliceFirst[sl]) first = s->segmentToChunk[seg - 1];
         return (s->segmentToChunk[seg] - first) * s->sliceChunkSize[sl];
      }
      case ORC_BIELLPACK: {
         /* detail/BiEllpack.h:93-110 */
         const int32_t strip = seg / 32;
         const int32_t groups = biell_active_groups(s->perm[seg] - strip * 32);
         int32_t h = 32, size = 0;
         for (int32_t g = 0; g < groups; g++) {
            const int32_t gs = s->groupPointers[strip * 6 + g + 1] - s->groupPointers[strip * 6 + g];
            size += gs / h;
            h /= 2;
         }
         return size;
      }
   }
   return 0;
}

/* getGlobalIndex(segment, local) for each format:
 * Ellpack EllpackBase.hpp:110-117; SlicedEllpack SlicedEllpackBase.hpp:121-145;
 * ChunkedEllpack detail/ChunkedEllpack.h:86-113; BiEllpack detail/BiEllpack.h:134-163. */
int64_t orc_global_index(const orc_segments* s, int32_t seg, int32_t local)
{
   switch (s->kind) {
      case ORC_CSR: return (int64_t)s->offsets[seg] + local;
      case ORC_ELLPACK:
         if (!s->colmajor) return (int64_t)seg * s->segmentSize + local;
         return (int64_t)seg + (int64_t)s->alignedSize * local;
      case ORC_SLICED_ELLPACK: {
         const int32_t sl = seg / 32, in = seg % 32;
         const int64_t off = s->sliceOffsets[sl];
         if (!s->colmajor) return off + (int64_t)in * s->sliceSegmentSizes[sl] + local;
         return off + in + 32 * (int64_t)local;
      }
      case ORC_CHUNKED_ELLPACK: {
         const int32_t sl = s->segmentToSlice[seg];
         int32_t first = 0;
         if (seg != s->sliceFirst[sl]) first = s->segmentToChunk[seg - 1];
         const int64_t off = s->slicePointer[sl];
         const int32_t cs = s->sliceChunkSize[sl];
         if (!s->colmajor) return off + (int64_t)first * cs + local;
         return off + (int64_t)(local % cs) * s->chunksInSlice + first + local / cs;
      }
      case ORC_BIELLPACK: {
         const int32_t strip = seg / 32;
         const int32_t p = s->perm[seg] - strip * 32;
         const int32_t groups = biell_active_groups(p);
         int64_t g0 = s->groupPointers[strip * 6];
         int32_t h = 32;
         for (int32_t g = 0; g < groups; g++) {
            const int32_t gs = s->groupPointers[strip * 6 + g + 1] - s->groupPointers[strip * 6 + g];
            if (gs) {
               const int32_t w = gs / h;
               if (local >= w) {
                  local -= w;
                  g0 += gs;
               }
               else {
                  if (!s->colmajor) return g0 + (int64_t)p * w + local;
                  return g0 + p + (int64_t)local * h;
               }
            }
            h /= 2;
         }
         return -1;
      }
   }
   return -1;
}

/* copySparseToSparseMatrix for a CSR source (Matrices/SparseOperations.hpp:106-186,
 * SparseMatrix::setRowCapacities SparseMatrix.hpp:303-325): target columns
 * start as paddingIndex -1 and values as 0; each source element with value
 * != 0 and column != -1 goes to getGlobalIndex(row, k++). */
#define ORC_FILL(NAME, T)                                                                                            \
   void NAME(const orc_segments* s, const int32_t* rowptr, const int32_t* cols, const T* vals, int32_t* out_cols,    \
             T* out_vals)                                                                                            \
   {                                                                                                                 \
      for (int64_t g = 0; g < s->storage; g++) {                                                                     \
         out_cols[g] = -1;                                                                                           \
         out_vals[g] = 0;                                                                                            \
      }                                                                                                              \
      for (int32_t r = 0; r < s->n; r++) {                                                                           \
         int32_t k = 0;                                                                                              \
         for (int32_t j = rowptr[r]; j < rowptr[r + 1]; j++) {                                                       \
            if (vals[j] != 0.0 && cols[j] != -1) {                                                                   \
               int64_t g = orc_global_index(s, r, k++);                                                              \
               out_cols[g] = cols[j];                                                                                \
               out_vals[g] = vals[j];                                                                                \
            }                                                                                                        \
         }                                                                                                           \
      }                                                                                                              \
   }
ORC_FILL(orc_fill_f64, double)
ORC_FILL(orc_fill_f32, float)

/* SparseMatrixBase::vectorProduct (Matrices/SparseMatrixBase.hpp:270-393):
 * fetch = values[g]*x[col] (0 for padding -1), summed over the segment in
 * local-index order (the Host reduction is sequential per row,
 * detail/ReducingOperations_CSR.h:46-61), then one of four keep variants:
 * beta==0 does not read y.  Rows [begin,end); end==0 means all rows. */
#define ORC_SPMV(NAME, T)                                                                                            \
   void NAME(const orc_segments* s, const int32_t* cols, const T* vals, const T* x, T* y, double alpha, double beta,  \
             int32_t begin, int32_t end)                                                                             \
   {                                                                                                                 \
      if (end == 0) end = s->n;                                                                                      \
      const T a = (T)alpha, b = (T)beta;                                                                             \
      for (int32_t r = begin; r < end; r++) {                                                                        \
         const int32_t cap = orc_segment_capacity(s, r);                                                             \
         T acc = 0;                                                                                                  \
         for (int32_t k = 0; k < cap; k++) {                                                                         \
            const int64_t g = orc_global_index(s, r, k);                                                             \
            const int32_t c = cols[g];                                                                               \
            if (c == -1) continue;                                                                                   \
            acc += vals[g] * x[c];                                                                                   \
         }                                                                                                           \
         if (b == 0) {                                                                                               \
            if (a == 1) y[r] = acc;                                                                                  \
            else y[r] = a * acc;                                                                                     \
         }                                                                                                           \
         else {                                                                                                      \
            if (a == 1) y[r] = b * y[r] + acc;                                                                       \
            else y[r] = b * y[r] + a * acc;                                                                          \
         }                                                                                                           \
      }                                                                                                              \
   }
ORC_SPMV(orc_spmv_f64, double)
ORC_SPMV(orc_spmv_f32, float)

/* vectorProduct of a symmetric matrix (SparseMatrixBase.hpp:296-330): only
 * one triangle is stored; y *= beta unless beta == 1 (y is read even when
 * beta == 0, as the reference's `outVector *= outVectorMultiplicator`);
 * then, for each row r in [begin,end), y[r] += alpha * sum_k a_k x[c_k] and,
 * for every stored c < r, y[c] += alpha * a * x[r] (the reference adds these
 * with atomics, so its order of additions is not fixed; here rows go in
 * order, elements in local-index order). */
#define ORC_SPMV_SYM(NAME, T)                                                                          \
   void NAME(const orc_segments* s, const int32_t* cols, const T* vals, const T* x, T* y, double alpha, \
             double beta, int32_t begin, int32_t end)                                                  \
   {                                                                                                   \
      if (end == 0) end = s->n;                                                                        \
      const T a = (T)alpha, b = (T)beta;                                                               \
      if (b != 1)                                                                                      \
         for (int32_t i = 0; i < s->n; i++) y[i] = y[i] * b;                                           \
      for (int32_t r = begin; r < end; r++) {                                                          \
         const int32_t cap = orc_segment_capacity(s, r);                                               \
         T acc = 0;                                                                                    \
         for (int32_t k = 0; k < cap; k++) {                                                           \
            const int64_t g = orc_global_index(s, r, k);                                               \
            const int32_t c = cols[g];                                                                 \
            if (c == -1) continue;                                                                     \
            if (c < r) y[c] += a * vals[g] * x[r];                                                     \
            acc += vals[g] * x[c];                                                                     \
         }                                                                                             \
         y[r] += a * acc;                                                                              \
      }                                                                                                \
   }
ORC_SPMV_SYM(orc_spmv_symmetric_f64, double)
ORC_SPMV_SYM(orc_spmv_symmetric_f32, float)

/* transposedVectorProduct (SparseMatrixBase.hpp:542-588): y (length
 * `columns`) *= beta unless beta == 1, then y[c] += alpha * x[r] * a for
 * every stored element (r, c, a) with c in [begin,end); end == 0 means all
 * columns.  Rows in order, elements in local-index order (the reference's
 * atomics leave the order open). */
#define ORC_SPMV_T(NAME, T)                                                                                 \
   void NAME(const orc_segments* s, const int32_t* cols, const T* vals, int32_t columns, const T* x, T* y,  \
             double alpha, double beta, int32_t begin, int32_t end)                                         \
   {                                                                                                        \
      if (end == 0) end = columns;                                                                          \
      const T a = (T)alpha, b = (T)beta;                                                                    \
      if (b != 1)                                                                                           \
         for (int32_t i = 0; i < columns; i++) y[i] = y[i] * b;                                             \
      for (int32_t r = 0; r < s->n; r++) {                                                                  \
         const int32_t cap = orc_segment_capacity(s, r);                                                    \
         for (int32_t k = 0; k < cap; k++) {                                                                \
            const int64_t g = orc_global_index(s, r, k);                                                    \
            const int32_t c = cols[g];                                                                      \
            if (c >= begin && c < end && c != -1) y[c] += a * x[r] * vals[g];                               \
         }                                                                                                  \
      }                                                                                                     \
   }
ORC_SPMV_T(orc_spmv_transposed_f64, double)
ORC_SPMV_T(orc_spmv_transposed_f32, float)

/* ------------------------------------------------------------------------ */
/* Krylov solvers on a CSR matrix (double)                                  */
/* ------------------------------------------------------------------------ */

typedef struct {
   int32_t n;
   const int32_t* rowptr;
   const int32_t* cols;
   const double* vals;
} orc_csr;

static void csr_mv(const orc_csr* A, const double* x, double* y)
{
   for (int32_t r = 0; r < A->n; r++) {
      double acc = 0;
      for (int32_t j = A->rowptr[r]; j < A->rowptr[r + 1]; j++) {
         if (A->cols[j] == -1) continue;
         acc += A->vals[j] * x[A->cols[j]];
      }
      y[r] = acc;
   }
}

static double dot(const double* a, const double* b, int32_t n)
{
   double s = 0;
   for (int32_t i = 0; i < n; i++) s += a[i] * b[i];
   return s;
}

/* Preconditioner: 0 none, 1 Jacobi (Diagonal.hpp:15-43: d_i = A_ii via
 * getElement, x = b / d), 2 ILU(0) (ILU0.hpp:15-140). */
typedef struct {
   int kind;
   int32_t n;
   double* diag;
   /* ILU(0): L in CSR without diagonal (unit implied), U with rows stored
    * reversed (row N-1-i holds row i, diagonal first). */
   int32_t *Lp, *Lc, *Up, *Uc;
   double *Lv, *Uv;
} orc_prec;

/* getElement(i, j) of a row with sorted columns; 0 if absent
 * (CSR getElement: linear search of the row). */
static double row_get(const int32_t* p, const int32_t* c, const double* v, int32_t row, int32_t col)
{
   for (int32_t j = p[row]; j < p[row + 1]; j++)
      if (c[j] == col) return v[j];
   return 0.0;
}

static int prec_setup(orc_prec* P, const orc_csr* A, int kind)
{
   memset(P, 0, sizeof(*P));
   P->kind = kind;
   P->n = A->n;
   const int32_t N = A->n;
   if (kind == 1) {
      P->diag = (double*)malloc(sizeof(double) * (size_t)N);
      for (int32_t i = 0; i < N; i++) P->diag[i] = row_get(A->rowptr, A->cols, A->vals, i, i);
   }
   else if (kind == 2) {
      /* ILU0.hpp:31-56 -- L holds columns < i, U columns >= i. */
      P->Lp = (int32_t*)calloc((size_t)N + 1, sizeof(int32_t));
      P->Up = (int32_t*)calloc((size_t)N + 1, sizeof(int32_t));
      for (int32_t i = 0; i < N; i++) {
         int32_t le = 0, ue = 0;
         for (int32_t j = A->rowptr[i]; j < A->rowptr[i + 1]; j++) {
            const int32_t c = A->cols[j];
            if (c < 0) continue;
            if (c < i) le++;
            else if (c < N) ue++;
            else break;
         }
         P->Lp[i + 1] = le;
         P->Up[N - 1 - i + 1] = ue;
      }
      for (int32_t i = 0; i < N; i++) {
         P->Lp[i + 1] += P->Lp[i];
         P->Up[i + 1] += P->Up[i];
      }
      P->Lc = (int32_t*)malloc(sizeof(int32_t) * (size_t)(P->Lp[N] + 1));
      P->Lv = (double*)malloc(sizeof(double) * (size_t)(P->Lp[N] + 1));
      P->Uc = (int32_t*)malloc(sizeof(int32_t) * (size_t)(P->Up[N] + 1));
      P->Uv = (double*)malloc(sizeof(double) * (size_t)(P->Up[N] + 1));
      /* ILU0.hpp:59-118 -- IKJ elimination, row by row. */
      for (int32_t i = 0; i < N; i++) {
         const int32_t le = P->Lp[i + 1] - P->Lp[i];
         const int32_t ui = N - 1 - i;
         const int32_t ue = P->Up[ui + 1] - P->Up[ui];
         int32_t j0 = A->rowptr[i];
         while (j0 < A->rowptr[i + 1] && A->cols[j0] < 0) j0++;
         for (int32_t c = 0; c < ue; c++) {
            P->Uc[P->Up[ui] + c] = A->cols[j0 + le + c];
            P->Uv[P->Up[ui] + c] = A->vals[j0 + le + c];
         }
         if (le > 0) {
            int32_t* Lc = P->Lc + P->Lp[i];
            double* Lv = P->Lv + P->Lp[i];
            for (int32_t c = 0; c < le; c++) {
               Lc[c] = A->cols[j0 + c];
               Lv[c] = A->vals[j0 + c];
            }
            for (int32_t ck = 0; ck < le; ck++) {
               const int32_t k = Lc[ck];
               const int32_t uk = N - 1 - k;
               const double Lik = Lv[ck] / row_get(P->Up, P->Uc, P->Uv, uk, k);
               Lv[ck] = Lik;
               for (int32_t cj = ck + 1; cj < le; cj++) {
                  const int32_t j = Lc[cj];
                  Lv[cj] = Lv[cj] - Lik * row_get(P->Up, P->Uc, P->Uv, uk, j);
               }
               for (int32_t cj = 0; cj < ue; cj++) {
                  const int32_t j = P->Uc[P->Up[ui] + cj];
                  P->Uv[P->Up[ui] + cj] = P->Uv[P->Up[ui] + cj] - Lik * row_get(P->Up, P->Uc, P->Uv, uk, j);
               }
            }
         }
      }
   }
   return ORC_OK;
}

/* Preconditioner::solve: Jacobi x = b/d; ILU(0) triangularSolveLower then
 * triangularSolveUpper<reversedRows> (Utils/TriangularSolve.h:20-103). */
static void prec_apply(const orc_prec* P, const double* b, double* x)
{
   const int32_t N = P->n;
   if (P->kind == 0) {
      memcpy(x, b, sizeof(double) * (size_t)N);
   }
   else if (P->kind == 1) {
      for (int32_t i = 0; i < N; i++) x[i] = b[i] / P->diag[i];
   }
   else {
      for (int32_t i = 0; i < N; i++) {
         double xi = b[i];
         for (int32_t j = P->Lp[i]; j < P->Lp[i + 1]; j++) xi -= P->Lv[j] * x[P->Lc[j]];
         x[i] = xi;
      }
      for (int32_t k = 0; k < N; k++) {
         const int32_t i = N - 1 - k;
         double xi = x[i];
         const int32_t p0 = P->Up[k], p1 = P->Up[k + 1];
         const double uii = P->Uv[p0];
         for (int32_t j = p0 + 1; j < p1; j++) xi -= P->Uv[j] * x[P->Uc[j]];
         x[i] = xi / uii;
      }
   }
}

static void prec_free(orc_prec* P)
{
   free(P->diag);
   free(P->Lp);
   free(P->Lc);
   free(P->Lv);
   free(P->Up);
   free(P->Uc);
   free(P->Uv);
}

/* ILU(0) factors, exported so the GPU factorisation can be compared
 * with them element by element.  Outputs are sized by the caller:
 * Lp/Up n+1, Lc/Lv/Uc/Uv nnz. */
int orc_ilu0_factor(int32_t n, const int32_t* rowptr, const int32_t* cols, const double* vals, int32_t* Lp, int32_t* Lc,
                    double* Lv, int32_t* Up, int32_t* Uc, double* Uv)
{
   orc_csr A = {n, rowptr, cols, vals};
   orc_prec P;
   prec_setup(&P, &A, 2);
   memcpy(Lp, P.Lp, sizeof(int32_t) * ((size_t)n + 1));
   memcpy(Up, P.Up, sizeof(int32_t) * ((size_t)n + 1));
   memcpy(Lc, P.Lc, sizeof(int32_t) * (size_t)P.Lp[n]);
   memcpy(Lv, P.Lv, sizeof(double) * (size_t)P.Lp[n]);
   memcpy(Uc, P.Uc, sizeof(int32_t) * (size_t)P.Up[n]);
   memcpy(Uv, P.Uv, sizeof(double) * (size_t)P.Up[n]);
   prec_free(&P);
   return ORC_OK;
}

int orc_prec_apply(int32_t n, const int32_t* rowptr, const int32_t* cols, const double* vals, int kind, const double* b,
                   double* x)
{
   orc_csr A = {n, rowptr, cols, vals};
   orc_prec P;
   prec_setup(&P, &A, kind);
   prec_apply(&P, b, x);
   prec_free(&P);
   return ORC_OK;
}

/* Stopping rules (Solvers/IterativeSolver.hpp:98-143); defaults maxIterations
 * 1e9, minIterations 0, divergence DBL_MAX (IterativeSolver.h:226-236). */
typedef struct {
   int32_t maxIterations;
   int32_t minIterations;
   double convergenceResidue;
   double divergenceResidue;
   int32_t iterations;
   double residue;
   double* history; /* optional: residue after each setResidue, indexed by iteration */
   int32_t historyCap;
} orc_solver_state;

static int check_next(const orc_solver_state* S)
{
   return !(isnan(S->residue) || S->iterations > S->maxIterations ||
            (S->residue > S->divergenceResidue && S->iterations >= S->minIterations) ||
            (S->residue < S->convergenceResidue && S->iterations >= S->minIterations));
}

static int next_iteration(orc_solver_state* S)
{
   int r = check_next(S);
   S->iterations++;
   return r;
}

static void set_residue(orc_solver_state* S, double r)
{
   S->residue = r;
   if (S->history && S->iterations < S->historyCap) S->history[S->iterations] = r;
}

static int check_convergence(const orc_solver_state* S)
{
   if (isnan(S->residue)) return 0;
   if (S->residue > S->divergenceResidue && S->iterations > S->minIterations) return 0;
   if (S->iterations >= S->maxIterations) return 0;
   if (S->residue > S->convergenceResidue) return 0;
   return 1;
}

static double l2(const double* a, int32_t n) { return sqrt(dot(a, a, n)); }

/* CG::solve (Solvers/Linear/CG.hpp:12-109). Returns 1 on convergence. */
int orc_cg(int32_t n, const int32_t* rowptr, const int32_t* cols, const double* vals, int precond, const double* b,
           double* x, orc_solver_state* S)
{
   orc_csr A = {n, rowptr, cols, vals};
   orc_prec P;
   prec_setup(&P, &A, precond);
   double* r = (double*)malloc(sizeof(double) * (size_t)n);
   double* p = (double*)malloc(sizeof(double) * (size_t)n);
   double* Ap = (double*)malloc(sizeof(double) * (size_t)n);
   double* z = (double*)malloc(sizeof(double) * (size_t)n);
   S->iterations = 0;
   double normb;
   if (precond) {
      prec_apply(&P, b, r);
      normb = l2(r, n);
   }
   else
      normb = l2(b, n);
   int ok = 1;
   if (normb == 0) {
      for (int32_t i = 0; i < n; i++) x[i] = 0;
      goto done;
   }
   csr_mv(&A, x, r);
   for (int32_t i = 0; i < n; i++) r[i] = b[i] - r[i];
   double s1, s2;
   if (precond) {
      prec_apply(&P, r, z);
      memcpy(p, z, sizeof(double) * (size_t)n);
      s1 = dot(r, z, n);
   }
   else {
      memcpy(p, r, sizeof(double) * (size_t)n);
      s1 = dot(r, r, n);
   }
   set_residue(S, sqrt(s1) / normb);
   while (next_iteration(S)) {
      csr_mv(&A, p, Ap);
      s2 = dot(Ap, p, n);
      if (s2 == 0.0) {
         set_residue(S, 0.0);
         break;
      }
      const double alpha = s1 / s2;
      for (int32_t i = 0; i < n; i++) x[i] += alpha * p[i];
      for (int32_t i = 0; i < n; i++) r[i] -= alpha * Ap[i];
      if (precond) {
         prec_apply(&P, r, z);
         s2 = s1;
         s1 = dot(r, z, n);
      }
      else {
         s2 = s1;
         s1 = dot(r, r, n);
      }
      const double beta = (s2 == 0.0) ? 0.0 : s1 / s2;
      const double* zz = precond ? z : r;
      for (int32_t i = 0; i < n; i++) p[i] = zz[i] + beta * p[i];
      set_residue(S, sqrt(s1) / normb);
   }
   ok = check_convergence(S);
done:
   free(r);
   free(p);
   free(Ap);
   free(z);
   prec_free(&P);
   return ok;
}

/* BICGStab::solve (Solvers/Linear/BICGStab.hpp:34-122), left preconditioning
 * in compute_residue/preconditioned_matvec (:125-151). */
int orc_bicgstab(int32_t n, const int32_t* rowptr, const int32_t* cols, const double* vals, int precond,
                 int exact_residue, const double* b, double* x, orc_solver_state* S)
{
   orc_csr A = {n, rowptr, cols, vals};
   orc_prec P;
   prec_setup(&P, &A, precond);
   const size_t nb = sizeof(double) * (size_t)n;
   double *r = malloc(nb), *r_ast = malloc(nb), *p = malloc(nb), *s = malloc(nb), *Ap = malloc(nb), *As = malloc(nb),
          *M_tmp = malloc(nb);
   int ok = 1;
   double b_norm;
   S->iterations = 0;
   if (precond) {
      prec_apply(&P, b, M_tmp);
      b_norm = l2(M_tmp, n);
   }
   else
      b_norm = l2(b, n);
   if (b_norm == 0) {
      for (int32_t i = 0; i < n; i++) x[i] = 0;
      goto done;
   }
#define RESIDUE(R)                                                      \
   do {                                                                 \
      csr_mv(&A, x, M_tmp);                                             \
      for (int32_t i = 0; i < n; i++) M_tmp[i] = b[i] - M_tmp[i];       \
      prec_apply(&P, M_tmp, (R));                                       \
   } while (0)
#define PMATVEC(SRC, DST)                                               \
   do {                                                                 \
      csr_mv(&A, (SRC), M_tmp);                                         \
      prec_apply(&P, M_tmp, (DST));                                     \
   } while (0)
   RESIDUE(r);
   memcpy(r_ast, r, nb);
   memcpy(p, r, nb);
   memset(s, 0, nb);
   double rho = dot(r, r_ast, n);
   double r_ast_sqnorm = rho;
   const double eps2 = 2.220446049250313e-16 * 2.220446049250313e-16;
   S->iterations = 0;
   set_residue(S, sqrt(rho) / b_norm);
   while (next_iteration(S)) {
      PMATVEC(p, Ap);
      const double alpha = rho / dot(Ap, r_ast, n);
      for (int32_t i = 0; i < n; i++) s[i] = r[i] - alpha * Ap[i];
      PMATVEC(s, As);
      const double omega = dot(As, s, n) / dot(As, As, n);
      for (int32_t i = 0; i < n; i++) x[i] += alpha * p[i] + omega * s[i];
      for (int32_t i = 0; i < n; i++) r[i] = s[i] - omega * As[i];
      const double rho_old = rho;
      rho = dot(r, r_ast, n);
      if (fabs(rho) < eps2 * r_ast_sqnorm) {
         RESIDUE(r);
         memcpy(r_ast, r, nb);
         r_ast_sqnorm = rho = dot(r, r_ast, n);
      }
      const double beta = (rho / rho_old) * (alpha / omega);
      for (int32_t i = 0; i < n; i++) p[i] = r[i] + beta * p[i] - (beta * omega) * Ap[i];
      if (exact_residue) {
         RESIDUE(s);
         set_residue(S, l2(s, n) / b_norm);
      }
      else
         set_residue(S, l2(r, n) / b_norm);
   }
#undef RESIDUE
#undef PMATVEC
   ok = check_convergence(S);
done:
   free(r);
   free(r_ast);
   free(p);
   free(s);
   free(Ap);
   free(As);
   free(M_tmp);
   prec_free(&P);
   return ok;
}

/* GMRES::solve with the MGS / MGSR orthogonalisation
 * (Solvers/Linear/GMRES.hpp:73-180, orthogonalize_MGS :280-347,
 * update :648-684, Givens :731-770).  restarting_min == restarting_max
 * (no adaptivity: the reference's defaults are equal).  reorth = 1 (MGS)
 * or 2 (MGSR).  Returns 1 on convergence, 0 otherwise, -1 on a zero
 * Hessenberg diagonal (the reference throws there). */
int orc_gmres(int32_t n, const int32_t* rowptr, const int32_t* cols, const double* vals, int precond, int32_t m,
              int reorth, const double* b, double* x, orc_solver_state* S)
{
   orc_csr A = {n, rowptr, cols, vals};
   orc_prec P;
   prec_setup(&P, &A, precond);
   const size_t nb = sizeof(double) * (size_t)n;
   double *r = malloc(nb), *w = malloc(nb), *M_tmp = malloc(nb);
   double* V = (double*)malloc(nb * (size_t)(m + 1));
   double* H = (double*)calloc((size_t)(m + 1) * m, sizeof(double));
   double* s = (double*)calloc((size_t)m + 1, sizeof(double));
   double* cs = (double*)calloc((size_t)m + 1, sizeof(double));
   double* sn = (double*)calloc((size_t)m + 1, sizeof(double));
   double* y = (double*)calloc((size_t)m + 1, sizeof(double));
   int ok = 1;
   double normb;
   S->iterations = 0;
   if (precond) {
      prec_apply(&P, b, M_tmp);
      normb = l2(M_tmp, n);
   }
   else
      normb = l2(b, n);
   if (normb == 0) {
      for (int32_t i = 0; i < n; i++) x[i] = 0;
      goto done;
   }
#define RESIDUE(R)                                                      \
   do {                                                                 \
      csr_mv(&A, x, M_tmp);                                             \
      for (int32_t i = 0; i < n; i++) M_tmp[i] = b[i] - M_tmp[i];       \
      prec_apply(&P, M_tmp, (R));                                       \
   } while (0)
   RESIDUE(r);
   double beta = l2(r, n);
   S->iterations = 0;
   set_residue(S, beta / normb);
   while (check_next(S)) {
      /* orthogonalize_MGS */
      int o_steps = m;
      for (int32_t i = 0; i < n; i++) V[i] = (1.0 / beta) * r[i];
      for (int32_t i = 0; i < (m + 1) * m; i++) H[i] = 0.0;
      for (int32_t i = 0; i <= m; i++) s[i] = 0.0;
      s[0] = beta;
      for (int i = 0; i < m && next_iteration(S); i++) {
         double* vi = V + (size_t)i * n;
         csr_mv(&A, vi, M_tmp);
         prec_apply(&P, M_tmp, w);
         for (int k = 0; k <= i; k++) H[k + i * (m + 1)] = 0.0;
         for (int l = 0; l < reorth; l++)
            for (int k = 0; k <= i; k++) {
               const double* vk = V + (size_t)k * n;
               const double hki = dot(w, vk, n);
               H[k + i * (m + 1)] += hki;
               for (int32_t t = 0; t < n; t++) w[t] = w[t] - hki * vk[t];
            }
         const double normw = l2(w, n);
         H[i + 1 + i * (m + 1)] = normw;
         double* vn = V + (size_t)(i + 1) * n;
         for (int32_t t = 0; t < n; t++) vn[t] = (1.0 / normw) * w[t];
         /* apply_givens_rotations */
         for (int k = 0; k < i; k++) {
            double* dx = &H[k + i * (m + 1)];
            double* dy = &H[k + 1 + i * (m + 1)];
            const double tmp = cs[k] * *dx + sn[k] * *dy;
            *dy = cs[k] * *dy - sn[k] * *dx;
            *dx = tmp;
         }
         if (H[i + 1 + i * (m + 1)] != 0.0) {
            double dx = H[i + i * (m + 1)], dy = H[i + 1 + i * (m + 1)];
            if (dy == 0.0) {
               cs[i] = 1.0;
               sn[i] = 0.0;
            }
            else if (fabs(dy) > fabs(dx)) {
               const double t = dx / dy;
               sn[i] = 1.0 / sqrt(1.0 + t * t);
               cs[i] = t * sn[i];
            }
            else {
               const double t = dy / dx;
               cs[i] = 1.0 / sqrt(1.0 + t * t);
               sn[i] = t * cs[i];
            }
            double* hx = &H[i + i * (m + 1)];
            double* hy = &H[i + 1 + i * (m + 1)];
            double tmp = cs[i] * *hx + sn[i] * *hy;
            *hy = cs[i] * *hy - sn[i] * *hx;
            *hx = tmp;
            tmp = cs[i] * s[i] + sn[i] * s[i + 1];
            s[i + 1] = cs[i] * s[i + 1] - sn[i] * s[i];
            s[i] = tmp;
         }
         set_residue(S, fabs(s[i + 1]) / normb);
         if (!check_next(S)) {
            o_steps = i;
            break;
         }
      }
      const int k_upd = (o_steps < m) ? o_steps : m - 1;
      /* update(k, m, H, s, V, x) */
      for (int i = 0; i <= m; i++) y[i] = s[i];
      for (int i = k_upd; i >= 0; i--) {
         if (H[i + i * (m + 1)] == 0) {
            ok = -1;
            goto done;
         }
         y[i] /= H[i + i * (m + 1)];
         for (int j = i - 1; j >= 0; j--) y[j] -= H[j + i * (m + 1)] * y[i];
      }
      for (int32_t t = 0; t < n; t++) {
         double acc = 0;
         for (int j = 0; j <= k_upd; j++) acc += V[(size_t)j * n + t] * y[j];
         x[t] = acc + x[t];
      }
      if (o_steps < m) {
         ok = check_convergence(S);
         goto done;
      }
      RESIDUE(r);
      beta = l2(r, n);
      set_residue(S, beta / normb);
   }
#undef RESIDUE
   ok = check_convergence(S);
done:
   free(r);
   free(w);
   free(M_tmp);
   free(V);
   free(H);
   free(s);
   free(cs);
   free(sn);
   free(y);
   prec_free(&P);
   return ok;
}

/* GMRES::apply_givens_rotations (Solvers/Linear/GMRES.hpp:731-770) on
 * column i of H (leading dimension m + 1) and on s. */
static void givens_column(int i, int m, double* H, double* s, double* cs, double* sn)
{
   for (int k = 0; k < i; k++) {
      double* dx = &H[k + i * (m + 1)];
      double* dy = &H[k + 1 + i * (m + 1)];
      const double tmp = cs[k] * *dx + sn[k] * *dy;
      *dy = cs[k] * *dy - sn[k] * *dx;
      *dx = tmp;
   }
   if (H[i + 1 + i * (m + 1)] != 0.0) {
      double dx = H[i + i * (m + 1)], dy = H[i + 1 + i * (m + 1)];
      if (dy == 0.0) {
         cs[i] = 1.0;
         sn[i] = 0.0;
      }
      else if (fabs(dy) > fabs(dx)) {
         const double t = dx / dy;
         sn[i] = 1.0 / sqrt(1.0 + t * t);
         cs[i] = t * sn[i];
      }
      else {
         const double t = dy / dx;
         cs[i] = 1.0 / sqrt(1.0 + t * t);
         sn[i] = t * cs[i];
      }
      double* hx = &H[i + i * (m + 1)];
      double* hy = &H[i + 1 + i * (m + 1)];
      double tmp = cs[i] * *hx + sn[i] * *hy;
      *hy = cs[i] * *hy - sn[i] * *hx;
      *hx = tmp;
      tmp = cs[i] * s[i] + sn[i] * s[i + 1];
      s[i + 1] = cs[i] * s[i + 1] - sn[i] * s[i];
      s[i] = tmp;
   }
}

/* GMRES::solve with the CWY orthogonalisation: Householder reflections
 * P_i = I - t_i y_i y_i^T accumulated in compact WY form I - Y T Y^T
 * (orthogonalize_CWY, Solvers/Linear/GMRES.hpp:350-423; hauseholder_generate
 * :468-537; hauseholder_apply_trunc :539-570; hauseholder_cwy :572-604;
 * hauseholder_cwy_transposed :606-643; the CWY branch of update :685-720).
 * The basis vectors are not stored: v_i = (I - Y T Y^T) e_i is rebuilt when
 * needed.  Y is n x (m+1) (column j zero above row j); YL holds its upper
 * (m+1) x (m+1) block; T is upper triangular with leading dimension m+1.
 * Each orthogonalisation cycle counts m+1 iterations (i = 0..m) and makes m
 * products.  Requires n >= m + 1.  Returns as orc_gmres. */
int orc_gmres_cwy(int32_t n, const int32_t* rowptr, const int32_t* cols, const double* vals, int precond, int32_t m,
                  const double* b, double* x, orc_solver_state* S)
{
   orc_csr A = {n, rowptr, cols, vals};
   orc_prec P;
   prec_setup(&P, &A, precond);
   const int L = m + 1;  /* restarting_max + 1 */
   const size_t nb = sizeof(double) * (size_t)n;
   double *r = malloc(nb), *w = malloc(nb), *z = malloc(nb), *v = malloc(nb), *M_tmp = malloc(nb);
   double* Y = (double*)calloc((size_t)n * L, sizeof(double));
   double* YL = (double*)calloc((size_t)L * L, sizeof(double));
   double* T = (double*)calloc((size_t)L * L, sizeof(double));
   double* H = (double*)calloc((size_t)(m + 1) * m, sizeof(double));
   double* s = (double*)calloc((size_t)m + 1, sizeof(double));
   double* cs = (double*)calloc((size_t)m + 1, sizeof(double));
   double* sn = (double*)calloc((size_t)m + 1, sizeof(double));
   double* y = (double*)calloc((size_t)m + 1, sizeof(double));
   double* aux = (double*)calloc((size_t)L, sizeof(double));
   int ok = 1;
   double normb;
   S->iterations = 0;
   if (n < L) {
      ok = 0;
      goto done;
   }
   if (precond) {
      prec_apply(&P, b, M_tmp);
      normb = l2(M_tmp, n);
   }
   else
      normb = l2(b, n);
   if (normb == 0) {
      for (int32_t i = 0; i < n; i++) x[i] = 0;
      goto done;
   }
#define RESIDUE(R)                                                      \
   do {                                                                 \
      csr_mv(&A, x, M_tmp);                                             \
      for (int32_t i = 0; i < n; i++) M_tmp[i] = b[i] - M_tmp[i];       \
      prec_apply(&P, M_tmp, (R));                                       \
   } while (0)
   RESIDUE(r);
   double beta = l2(r, n);
   S->iterations = 0;
   set_residue(S, beta / normb);
   while (check_next(S)) {
      int o_steps = m;
      for (int32_t t = 0; t < n; t++) z[t] = r[t];
      for (int32_t t = 0; t < (m + 1) * m; t++) H[t] = 0.0;
      for (int32_t t = 0; t <= m; t++) s[t] = 0.0;
      for (int32_t t = 0; t < L * L; t++) T[t] = 0.0;
      for (int i = 0; i <= m && next_iteration(S); i++) {
         double* yi = Y + (size_t)i * n;
         /* hauseholder_generate: y_i = z truncated above row i, reflected */
         for (int32_t j = 0; j < n; j++) yi[j] = j < i ? 0.0 : z[j];
         const double normz = l2(yi, n);
         const double y_ii = yi[i];
         yi[i] = y_ii > 0.0 ? y_ii + normz : y_ii - normz;
         const double norm_yi_squared = 2 * (normz * normz + fabs(y_ii) * normz);
         const double t_i = 2.0 / norm_yi_squared;
         T[i + i * L] = t_i;
         if (i > 0) {
            for (int k = 0; k < i; k++) aux[k] = dot(Y + (size_t)k * n, yi, n);
            for (int k = 0; k < i; k++) {
               T[k + i * L] = 0.0;
               for (int j = k; j < i; j++) T[k + i * L] -= T[k + j * L] * (t_i * aux[j]);
            }
         }
         /* hauseholder_apply_trunc: out = z[0..i] - y_i[0..i] (t_i (y_i, z) = 1) */
         double* YLi = YL + (size_t)i * L;
         for (int k = 0; k < L; k++) YLi[k] = yi[k];
         double* out = i == 0 ? s : H + (size_t)(i - 1) * (m + 1);
         for (int k = 0; k <= i; k++) out[k] = z[k] - YLi[k] * 1.0;
         /* hauseholder_cwy: v = e_i - Y_i T_i Y_i^T e_i */
         for (int k = 0; k <= i; k++) aux[k] = YL[i + k * L];
         for (int k = 0; k <= i; k++) {
            double a2 = 0.0;
            for (int j = k; j <= i; j++) a2 += T[k + j * L] * aux[j];
            aux[k] = a2;
         }
         for (int32_t t = 0; t < n; t++) {
            double acc = 0;
            for (int k = 0; k <= i; k++) acc += Y[(size_t)k * n + t] * aux[k];
            v[t] = -1.0 * acc;
         }
         v[i] = 1.0 + v[i];
         if (i < m) {
            /* w = M^-1 A v_i; z = (I - Y_i T_i^T Y_i^T) w */
            csr_mv(&A, v, M_tmp);
            prec_apply(&P, M_tmp, w);
            for (int k = 0; k <= i; k++) aux[k] = dot(Y + (size_t)k * n, w, n);
            for (int k = i; k >= 0; k--) {
               double a2 = 0.0;
               for (int j = 0; j <= k; j++) a2 += T[j + k * L] * aux[j];
               aux[k] = a2;
            }
            for (int32_t t = 0; t < n; t++) {
               double acc = 0;
               for (int k = 0; k <= i; k++) acc += Y[(size_t)k * n + t] * aux[k];
               z[t] = -1.0 * acc + w[t];
            }
         }
         if (i > 0) givens_column(i - 1, m, H, s, cs, sn);
         set_residue(S, fabs(s[i]) / normb);
         if (i > 0 && !check_next(S)) {
            o_steps = i - 1;
            break;
         }
      }
      const int k_upd = (o_steps < m) ? o_steps : m - 1;
      /* update(k, m, H, s, V, x), CWY branch */
      for (int i = 0; i <= m; i++) y[i] = s[i];
      for (int i = k_upd; i >= 0; i--) {
         if (H[i + i * (m + 1)] == 0) {
            ok = -1;
            goto done;
         }
         y[i] /= H[i + i * (m + 1)];
         for (int j = i - 1; j >= 0; j--) y[j] -= H[j + i * (m + 1)] * y[i];
      }
      for (int j = 0; j <= k_upd; j++) aux[j] = 0;
      for (int j = 0; j <= k_upd; j++)
         for (int i = 0; i <= j; i++) aux[i] += y[j] * YL[j + i * L];
      for (int i = 0; i <= k_upd; i++) {
         double a2 = 0.0;
         for (int j = i; j <= k_upd; j++) a2 += T[i + j * L] * aux[j];
         aux[i] = a2;
      }
      for (int32_t t = 0; t < n; t++) {
         double acc = 0;
         for (int k = 0; k <= k_upd; k++) acc += Y[(size_t)k * n + t] * aux[k];
         x[t] = -1.0 * acc + x[t];
      }
      for (int j = 0; j <= k_upd; j++) x[j] = x[j] + y[j];  /* x += sum_j y_j e_j */
      if (o_steps < m) {
         ok = check_convergence(S);
         goto done;
      }
      RESIDUE(r);
      beta = l2(r, n);
      set_residue(S, beta / normb);
   }
#undef RESIDUE
   ok = check_convergence(S);
done:
   free(r);
   free(w);
   free(z);
   free(v);
   free(M_tmp);
   free(Y);
   free(YL);
   free(T);
   free(H);
   free(s);
   free(cs);
   free(sn);
   free(y);
   free(aux);
   prec_free(&P);
   return ok;
}

/* FGMRES: the GMRES below with right, flexible preconditioning -- no
 * counterpart in the reference; z_i = M^-1 v_i is kept, w = A z_i, x += Z y,
 * residues unpreconditioned (normb = ||b||).  Derived from GMRES::solve with the MGS / MGSR orthogonalisation
 * (Solvers/Linear/GMRES.hpp:73-180, orthogonalize_MGS :280-347,
 * update :648-684, Givens :731-770).  restarting_min == restarting_max
 * (no adaptivity: the reference's defaults are equal).  reorth = 1 (MGS)
 * or 2 (MGSR).  Returns 1 on convergence, 0 otherwise, -1 on a zero
 * Hessenberg diagonal (the reference throws there). */
int orc_fgmres(int32_t n, const int32_t* rowptr, const int32_t* cols, const double* vals, int precond, int32_t m,
              int reorth, const double* b, double* x, orc_solver_state* S)
{
   orc_csr A = {n, rowptr, cols, vals};
   orc_prec P;
   prec_setup(&P, &A, precond);
   const size_t nb = sizeof(double) * (size_t)n;
   double *r = malloc(nb), *w = malloc(nb), *M_tmp = malloc(nb);
   double* V = (double*)malloc(nb * (size_t)(m + 1));
   double* Zb = (double*)malloc(nb * (size_t)(m + 1));
   double* H = (double*)calloc((size_t)(m + 1) * m, sizeof(double));
   double* s = (double*)calloc((size_t)m + 1, sizeof(double));
   double* cs = (double*)calloc((size_t)m + 1, sizeof(double));
   double* sn = (double*)calloc((size_t)m + 1, sizeof(double));
   double* y = (double*)calloc((size_t)m + 1, sizeof(double));
   int ok = 1;
   double normb;
   S->iterations = 0;
   normb = l2(b, n);
   if (normb == 0) {
      for (int32_t i = 0; i < n; i++) x[i] = 0;
      goto done;
   }
#define RESIDUE(R)                                                      \
   do {                                                                 \
      csr_mv(&A, x, (R));                                               \
      for (int32_t i = 0; i < n; i++) (R)[i] = b[i] - (R)[i];           \
   } while (0)
   RESIDUE(r);
   double beta = l2(r, n);
   S->iterations = 0;
   set_residue(S, beta / normb);
   while (check_next(S)) {
      /* orthogonalize_MGS */
      int o_steps = m;
      for (int32_t i = 0; i < n; i++) V[i] = (1.0 / beta) * r[i];
      for (int32_t i = 0; i < (m + 1) * m; i++) H[i] = 0.0;
      for (int32_t i = 0; i <= m; i++) s[i] = 0.0;
      s[0] = beta;
      for (int i = 0; i < m && next_iteration(S); i++) {
         double* vi = V + (size_t)i * n;
         double* zi = Zb + (size_t)i * n;
         prec_apply(&P, vi, zi);
         csr_mv(&A, zi, w);
         for (int k = 0; k <= i; k++) H[k + i * (m + 1)] = 0.0;
         for (int l = 0; l < reorth; l++)
            for (int k = 0; k <= i; k++) {
               const double* vk = V + (size_t)k * n;
               const double hki = dot(w, vk, n);
               H[k + i * (m + 1)] += hki;
               for (int32_t t = 0; t < n; t++) w[t] = w[t] - hki * vk[t];
            }
         const double normw = l2(w, n);
         H[i + 1 + i * (m + 1)] = normw;
         double* vn = V + (size_t)(i + 1) * n;
         for (int32_t t = 0; t < n; t++) vn[t] = (1.0 / normw) * w[t];
         /* apply_givens_rotations */
         for (int k = 0; k < i; k++) {
            double* dx = &H[k + i * (m + 1)];
            double* dy = &H[k + 1 + i * (m + 1)];
            const double tmp = cs[k] * *dx + sn[k] * *dy;
            *dy = cs[k] * *dy - sn[k] * *dx;
            *dx = tmp;
         }
         if (H[i + 1 + i * (m + 1)] != 0.0) {
            double dx = H[i + i * (m + 1)], dy = H[i + 1 + i * (m + 1)];
            if (dy == 0.0) {
               cs[i] = 1.0;
               sn[i] = 0.0;
            }
            else if (fabs(dy) > fabs(dx)) {
               const double t = dx / dy;
               sn[i] = 1.0 / sqrt(1.0 + t * t);
               cs[i] = t * sn[i];
            }
            else {
               const double t = dy / dx;
               cs[i] = 1.0 / sqrt(1.0 + t * t);
               sn[i] = t * cs[i];
            }
            double* hx = &H[i + i * (m + 1)];
            double* hy = &H[i + 1 + i * (m + 1)];
            double tmp = cs[i] * *hx + sn[i] * *hy;
            *hy = cs[i] * *hy - sn[i] * *hx;
            *hx = tmp;
            tmp = cs[i] * s[i] + sn[i] * s[i + 1];
            s[i + 1] = cs[i] * s[i + 1] - sn[i] * s[i];
            s[i] = tmp;
         }
         set_residue(S, fabs(s[i + 1]) / normb);
         if (!check_next(S)) {
            o_steps = i;
            break;
         }
      }
      const int k_upd = (o_steps < m) ? o_steps : m - 1;
      /* update(k, m, H, s, V, x) */
      for (int i = 0; i <= m; i++) y[i] = s[i];
      for (int i = k_upd; i >= 0; i--) {
         if (H[i + i * (m + 1)] == 0) {
            ok = -1;
            goto done;
         }
         y[i] /= H[i + i * (m + 1)];
         for (int j = i - 1; j >= 0; j--) y[j] -= H[j + i * (m + 1)] * y[i];
      }
      for (int32_t t = 0; t < n; t++) {
         double acc = 0;
         for (int j = 0; j <= k_upd; j++) acc += Zb[(size_t)j * n + t] * y[j];
         x[t] = acc + x[t];
      }
      if (o_steps < m) {
         ok = check_convergence(S);
         goto done;
      }
      RESIDUE(r);
      beta = l2(r, n);
      set_residue(S, beta / normb);
   }
#undef RESIDUE
   ok = check_convergence(S);
done:
   free(r);
   free(w);
   free(M_tmp);
   free(V);
   free(Zb);
   free(H);
   free(s);
   free(cs);
   free(sn);
   free(y);
   prec_free(&P);
   return ok;
}

/* True residual ||b - A x|| / ||b|| (Solvers/Linear/Utils/LinearResidueGetter.hpp:11-23). */
double orc_true_residual(int32_t n, const int32_t* rowptr, const int32_t* cols, const double* vals, const double* b,
                         const double* x)
{
   orc_csr A = {n, rowptr, cols, vals};
   double* t = (double*)malloc(sizeof(double) * (size_t)n);
   csr_mv(&A, x, t);
   double num = 0, den = 0;
   for (int32_t i = 0; i < n; i++) {
      const double d = b[i] - t[i];
      num += d * d;
      den += b[i] * b[i];
   }
   free(t);
   return sqrt(num) / sqrt(den);
}

/* ------------------------------------------------------------------------
 * The other Krylov solvers of the reference's linear-solver benchmark.
 * ---------------------------------------------------------------------- */

static void prec_apply_any(const orc_prec* P, const double* b, double* x)
{
   if (P->kind == 0) {
      if (x != b) memmove(x, b, sizeof(double) * (size_t)P->n);
   }
   else
      prec_apply(P, b, x);
}

/* TFQMR::solve (Solvers/Linear/TFQMR.hpp:12-113), left-preconditioned;
 * the residue is the quasi-residual bound tau*sqrt(iter+1)/||M^-1 b||.
 * Returns 1 on convergence, 0 otherwise. */
int orc_tfqmr(int32_t n, const int32_t* rowptr, const int32_t* cols, const double* vals, int precond,
              const double* b, double* x, orc_solver_state* S)
{
   orc_csr A = {n, rowptr, cols, vals};
   orc_prec P;
   prec_setup(&P, &A, precond);
   const size_t nb = sizeof(double) * (size_t)n;
   double *d = calloc(n, sizeof(double)), *r = malloc(nb), *w = malloc(nb), *u = malloc(nb), *v = malloc(nb);
   double *r_ast = malloc(nb), *Au = malloc(nb), *M_tmp = malloc(nb);
   int ok = 1;
   double b_norm;
   S->iterations = 0;
   if (precond) {
      prec_apply(&P, b, M_tmp);
      b_norm = l2(M_tmp, n);
      csr_mv(&A, x, M_tmp);
      for (int32_t i = 0; i < n; i++) M_tmp[i] = b[i] - M_tmp[i];
      prec_apply(&P, M_tmp, r);
   }
   else {
      b_norm = l2(b, n);
      csr_mv(&A, x, r);
      for (int32_t i = 0; i < n; i++) r[i] = b[i] - r[i];
   }
   if (b_norm == 0) {
      for (int32_t i = 0; i < n; i++) x[i] = 0;
      goto done;
   }
#define PMV(SRC, DST)                     \
   do {                                   \
      if (precond) {                      \
         csr_mv(&A, (SRC), M_tmp);        \
         prec_apply(&P, M_tmp, (DST));    \
      }                                   \
      else                                \
         csr_mv(&A, (SRC), (DST));        \
   } while (0)
   memcpy(w, r, nb);
   memcpy(u, r, nb);
   PMV(u, Au);
   memcpy(v, Au, nb);
   double tau = l2(r, n), theta = 0.0, eta = 0.0;
   memcpy(r_ast, r, nb);
   double rho = dot(r_ast, r, n), alpha = 0.0;
   S->iterations = 0;
   set_residue(S, tau / b_norm);
   while (next_iteration(S)) {
      const int32_t iter = S->iterations;
      if (iter % 2 == 1)
         alpha = rho / dot(v, r_ast, n);
      else
         PMV(u, Au);
      for (int32_t i = 0; i < n; i++) w[i] = w[i] - alpha * Au[i];
      const double dc = theta * theta * eta / alpha;
      for (int32_t i = 0; i < n; i++) d[i] = u[i] + dc * d[i];
      const double w_norm = l2(w, n);
      theta = w_norm / tau;
      const double c = 1.0 / sqrt(1.0 + theta * theta);
      tau = tau * theta * c;
      eta = c * c * alpha;
      for (int32_t i = 0; i < n; i++) x[i] = x[i] + eta * d[i];
      set_residue(S, tau * sqrt((double)(iter + 1)) / b_norm);
      if (iter > S->minIterations && S->residue < S->convergenceResidue) break;
      if (iter % 2 == 0) {
         const double rho_new = dot(w, r_ast, n);
         const double beta = rho_new / rho;
         rho = rho_new;
         for (int32_t i = 0; i < n; i++) u[i] = w[i] + beta * u[i];
         for (int32_t i = 0; i < n; i++) v[i] = beta * Au[i] + (beta * beta) * v[i];
         PMV(u, Au);
         for (int32_t i = 0; i < n; i++) v[i] = v[i] + Au[i];
      }
      else
         for (int32_t i = 0; i < n; i++) u[i] = u[i] - alpha * v[i];
   }
   ok = check_convergence(S);
done:
   free(d);
   free(r);
   free(w);
   free(u);
   free(v);
   free(r_ast);
   free(Au);
   free(M_tmp);
   prec_free(&P);
   return ok;
}

/* BICGStabL::solve (Solvers/Linear/BICGStabL.hpp:36-242): BiCGStab(ell),
 * left-preconditioned; R and U hold ell+1 columns of length n; T, sigma and
 * the g vectors live on the host.  Note sigma[j] = (r_j, r_j) for j >= 1 but
 * sigma[0] = ||r_0|| (as in the reference).  `exact` selects the exact
 * preconditioned residue for stopping.  Returns 1 on convergence, 0
 * otherwise, -2 on a NaN initial residue (the reference throws). */
int orc_bicgstabl(int32_t n, const int32_t* rowptr, const int32_t* cols, const double* vals, int precond, int ell,
                  int exact, const double* b, double* x, orc_solver_state* S)
{
   orc_csr A = {n, rowptr, cols, vals};
   orc_prec P;
   prec_setup(&P, &A, precond);
   const size_t nb = sizeof(double) * (size_t)n;
   double* R = calloc((size_t)n * (ell + 1), sizeof(double));
   double* U = calloc((size_t)n * (ell + 1), sizeof(double));
   double *r_ast = malloc(nb), *M_tmp = malloc(nb), *res_tmp = malloc(nb);
   double* T = calloc((size_t)ell * ell, sizeof(double));
   double *sigma = calloc(ell + 1, sizeof(double)), *g0 = calloc(ell + 1, sizeof(double));
   double *g1 = calloc(ell + 1, sizeof(double)), *g2 = calloc(ell + 1, sizeof(double));
   int ok = 1;
   double b_norm;
   S->iterations = 0;
   if (precond) {
      prec_apply(&P, b, M_tmp);
      b_norm = l2(M_tmp, n);
   }
   else
      b_norm = l2(b, n);
   if (b_norm == 0) {
      for (int32_t i = 0; i < n; i++) x[i] = 0;
      goto done;
   }
#define RESID(RV)                                                       \
   do {                                                                 \
      if (precond) {                                                    \
         csr_mv(&A, x, M_tmp);                                          \
         for (int32_t i = 0; i < n; i++) M_tmp[i] = b[i] - M_tmp[i];    \
         prec_apply(&P, M_tmp, (RV));                                   \
      }                                                                 \
      else {                                                            \
         csr_mv(&A, x, (RV));                                           \
         for (int32_t i = 0; i < n; i++) (RV)[i] = b[i] - (RV)[i];      \
      }                                                                 \
   } while (0)
   double* r0 = R;
   double* u0 = U;
   RESID(r0);
   sigma[0] = l2(r0, n);
   if (isnan(sigma[0])) {
      ok = -2;
      goto done;
   }
   for (int32_t i = 0; i < n; i++) r_ast[i] = r0[i];
   for (int32_t i = 0; i < n; i++) r_ast[i] = r_ast[i] / sigma[0];
   double rho_0 = 1.0, rho_1, alpha = 0.0, beta, gamma, omega = 1.0;
   S->iterations = 0;
   set_residue(S, sigma[0] / b_norm);
   while (check_next(S)) {
      rho_0 = -omega * rho_0;
      for (int j = 0; j < ell; j++) {
         next_iteration(S);
         double* rj = R + (size_t)j * n;
         rho_1 = dot(r_ast, rj, n);
         beta = alpha * rho_1 / rho_0;
         rho_0 = rho_1;
         for (int c = 0; c <= j; c++)
            for (int32_t i = 0; i < n; i++)
               U[(size_t)c * n + i] = 1.0 * R[(size_t)c * n + i] + (-beta) * U[(size_t)c * n + i];
         PMV(U + (size_t)j * n, U + (size_t)(j + 1) * n);
         gamma = dot(r_ast, U + (size_t)(j + 1) * n, n);
         alpha = rho_0 / gamma;
         for (int c = 0; c <= j; c++)
            for (int32_t i = 0; i < n; i++)
               R[(size_t)c * n + i] = 1.0 * R[(size_t)c * n + i] + (-alpha) * U[(size_t)(c + 1) * n + i];
         PMV(R + (size_t)j * n, R + (size_t)(j + 1) * n);
         for (int32_t i = 0; i < n; i++) x[i] = x[i] + alpha * u0[i];
      }
      for (int j = 1; j <= ell; j++) {
         double* rj = R + (size_t)j * n;
         for (int i = 1; i < j; i++) {
            const double* ri = R + (size_t)i * n;
            const int ij = (i - 1) + (j - 1) * ell;
            T[ij] = dot(ri, rj, n) / sigma[i];
            for (int32_t t = 0; t < n; t++) rj[t] = rj[t] - T[ij] * ri[t];
         }
         sigma[j] = dot(rj, rj, n);
         g1[j] = dot(r0, rj, n) / sigma[j];
      }
      omega = g1[ell];
      for (int j = ell; j >= 1; j--) {
         g0[j] = g1[j];
         for (int i = j + 1; i <= ell; i++) g0[j] -= T[(j - 1) + (i - 1) * ell] * g0[i];
      }
      for (int j = 1; j < ell; j++) {
         g2[j] = g0[j + 1];
         for (int i = j + 1; i < ell; i++) g2[j] += T[(j - 1) + (i - 1) * ell] * g0[i + 1];
      }
      g2[0] = g0[1];
      for (int32_t t = 0; t < n; t++) {
         double acc = 0;
         for (int c = 0; c < ell; c++) acc += R[(size_t)c * n + t] * g2[c];
         x[t] = acc + x[t];
      }
      for (int32_t t = 0; t < n; t++) {
         double acc = 0;
         for (int c = 0; c < ell; c++) acc += R[(size_t)(c + 1) * n + t] * g1[c + 1];
         r0[t] = -1.0 * acc + r0[t];
      }
      for (int32_t t = 0; t < n; t++) {
         double acc = 0;
         for (int c = 0; c < ell; c++) acc += U[(size_t)(c + 1) * n + t] * g0[c + 1];
         u0[t] = -1.0 * acc + u0[t];
      }
      if (exact) {
         RESID(res_tmp);
         sigma[0] = l2(res_tmp, n);
      }
      else
         sigma[0] = l2(r0, n);
      set_residue(S, sigma[0] / b_norm);
   }
   ok = check_convergence(S);
#undef RESID
done:
   free(R);
   free(U);
   free(r_ast);
   free(M_tmp);
   free(res_tmp);
   free(T);
   free(sigma);
   free(g0);
   free(g1);
   free(g2);
   prec_free(&P);
   return ok;
}

/* LU_sequential_factorize / LU_sequential_solve
 * (Matrices/Factorization/LUsequential.h:14-72): no pivoting; A is m x m,
 * row-major with leading dimension ld. */
static void lu_solve_small(double* A, int m, int ld, const double* bvec, double* xvec)
{
   for (int k = 0; k < m; k++) {
      const double pivot = A[k * ld + k];
      for (int j = k + 1; j < m; j++) {
         const double factor = A[j * ld + k] / pivot;
         A[j * ld + k] = factor;
         for (int i = k + 1; i < m; i++) A[j * ld + i] = A[j * ld + i] - factor * A[k * ld + i];
      }
   }
   for (int k = 0; k < m; k++) xvec[k] = bvec[k];
   for (int k = 1; k < m; k++)
      for (int j = 0; j < k; j++) xvec[k] -= A[k * ld + j] * xvec[j];
   for (int k = m - 1; k >= 0; k--) {
      for (int j = m - 1; j > k; j--) xvec[k] -= A[k * ld + j] * xvec[j];
      xvec[k] /= A[k * ld + k];
   }
}

/* IDRs::solve (Solvers/Linear/IDRs.hpp:50-250): IDR(s) with the shadow
 * space P (n x s, column-major) drawn by the caller as IDRs::setSize does
 * (:270-300; orc_idrs_shadow); the preconditioner is applied on the right
 * of the update directions (psolve), residues are unpreconditioned.
 * `smoothing` enables residual smoothing.  Returns 1 on convergence, 0
 * otherwise (including the reference's early `return false` on a zero
 * M(k,k) or omega), -2 on a NaN initial residue (the reference throws). */
int orc_idrs(int32_t n, const int32_t* rowptr, const int32_t* cols, const double* vals, int precond, int s,
             int smoothing, const double* Pm, const double* b, double* x, orc_solver_state* S)
{
   orc_csr A = {n, rowptr, cols, vals};
   orc_prec Pc;
   prec_setup(&Pc, &A, precond);
   const size_t nb = sizeof(double) * (size_t)n;
   double* G = calloc((size_t)n * s, sizeof(double));
   double* U = calloc((size_t)n * s, sizeof(double));
   double *r = malloc(nb), *v = malloc(nb), *t = malloc(nb), *x_s = malloc(nb), *r_s = malloc(nb);
   double* M = calloc((size_t)s * s, sizeof(double));
   double *f = calloc(s, sizeof(double)), *c = calloc(s, sizeof(double)), *Msub = calloc((size_t)s * s, sizeof(double));
   int ok = 1;
   S->iterations = 0;
   const double b_norm = l2(b, n);
   if (b_norm == 0) {
      for (int32_t i = 0; i < n; i++) x[i] = 0;
      goto done;
   }
   csr_mv(&A, x, r);
   for (int32_t i = 0; i < n; i++) r[i] = b[i] - r[i];
   double r_norm = l2(r, n);
   if (isnan(r_norm)) {
      ok = -2;
      goto done;
   }
   const double angle = 0.7;
   double omega = 1.0;
   for (int i = 0; i < s; i++) M[i * s + i] = 1;
   if (smoothing) {
      memcpy(x_s, x, nb);
      memcpy(r_s, r, nb);
   }
#define SMOOTH()                                                                  \
   do {                                                                           \
      if (smoothing) {                                                            \
         for (int32_t q = 0; q < n; q++) t[q] = r_s[q] - r[q];                    \
         const double gam = dot(t, r_s, n) / dot(t, t, n);                        \
         for (int32_t q = 0; q < n; q++) r_s[q] = r_s[q] - gam * t[q];            \
         for (int32_t q = 0; q < n; q++) x_s[q] = x_s[q] - gam * (x_s[q] - x[q]); \
         r_norm = l2(r_s, n);                                                     \
      }                                                                           \
   } while (0)
   S->iterations = 0;
   set_residue(S, r_norm / b_norm);
   while (check_next(S)) {
      for (int i = 0; i < s; i++) f[i] = dot(Pm + (size_t)i * n, r, n);
      for (int k = 0; k < s; k++) {
         double* Uk = U + (size_t)k * n;
         double* Gk = G + (size_t)k * n;
         const int m = s - k;
         for (int i = k; i < s; i++)
            for (int j = k; j < s; j++) Msub[(i - k) * s + (j - k)] = M[i * s + j];
         lu_solve_small(Msub, m, s, f + k, c);
         for (int32_t q = 0; q < n; q++) {
            double acc = 0;
            for (int i = 0; i < m; i++) acc += G[(size_t)(k + i) * n + q] * c[i];
            v[q] = -1.0 * acc + r[q];
         }
         prec_apply_any(&Pc, v, v);
         for (int32_t q = 0; q < n; q++) {
            double acc = 0;
            for (int i = 0; i < m; i++) acc += U[(size_t)(k + i) * n + q] * c[i];
            Uk[q] = acc;
         }
         for (int32_t q = 0; q < n; q++) Uk[q] = Uk[q] + omega * v[q];
         csr_mv(&A, Uk, Gk);
         for (int i = 0; i < k; i++) {
            const double* Pi = Pm + (size_t)i * n;
            const double* Ui = U + (size_t)i * n;
            const double* Gi = G + (size_t)i * n;
            const double alpha = dot(Pi, Gk, n) / M[i * s + i];
            for (int32_t q = 0; q < n; q++) Uk[q] = Uk[q] - alpha * Ui[q];
            for (int32_t q = 0; q < n; q++) Gk[q] = Gk[q] - alpha * Gi[q];
         }
         for (int i = k; i < s; i++) M[i * s + k] = dot(Pm + (size_t)i * n, Gk, n);
         if (M[k * s + k] == 0) {
            ok = 0;
            goto done;
         }
         const double beta = f[k] / M[k * s + k];
         for (int32_t q = 0; q < n; q++) x[q] = x[q] + beta * Uk[q];
         for (int32_t q = 0; q < n; q++) r[q] = r[q] - beta * Gk[q];
         r_norm = l2(r, n);
         SMOOTH();
         set_residue(S, r_norm / b_norm);
         if (!next_iteration(S)) {
            if (smoothing) memcpy(x, x_s, nb);
            ok = check_convergence(S);
            goto done;
         }
         if (k < s - 1)
            for (int i = k + 1; i < s; i++) f[i] = f[i] - beta * M[i * s + k];
      }
      prec_apply_any(&Pc, r, v);
      csr_mv(&A, v, t);
      const double t_norm = l2(t, n);
      const double tr = dot(t, r, n);
      const double rho = fabs(tr / (t_norm * r_norm));
      omega = tr / (t_norm * t_norm);
      if (rho < angle) omega = omega * angle / rho;
      if (omega == 0) {
         ok = 0;
         goto done;
      }
      for (int32_t q = 0; q < n; q++) x[q] = x[q] + omega * v[q];
      for (int32_t q = 0; q < n; q++) r[q] = r[q] - omega * t[q];
      r_norm = l2(r, n);
      SMOOTH();
      set_residue(S, r_norm / b_norm);
      next_iteration(S);
   }
   if (smoothing) memcpy(x, x_s, nb);
   ok = check_convergence(S);
#undef SMOOTH
#undef PMV
done:
   free(G);
   free(U);
   free(r);
   free(v);
   free(t);
   free(x_s);
   free(r_s);
   free(M);
   free(f);
   free(c);
   free(Msub);
   prec_free(&Pc);
   return ok;
}

/* Mixed-precision PCG with reliable updates -- the library's own solver
 * (no counterpart in the reference), restated for its tests: CG on FP32
 * values with vectors of type VT (float or double; rows summed in VT, dot
 * products in FP64); the correction xc (FP64: the exact product of the VT
 * alpha and p added in FP64) is folded into the FP64 x and r
 * replaced by (VT)(b - A x) (FP64 product) whenever the recursive |r|^2
 * falls below max(delta |r_u|, tol |b|)^2, r_u the residual of the last
 * update; p is kept, beta = (r, z)_new / (r, z)_old.  precond: 0 none,
 * 1 Jacobi (diagonal of the FP32 values), 2 FSAI z = G^T (G r) from the
 * factor G and its transpose as the solver applies them (CSR, FP32 values;
 * rows summed in VT in entry order) with (r, z) = |G r|^2.  With `excess`
 * (when every row holds its diagonal entry) the FP32 product is the
 * library's row-excess form: the diagonal entry replaced by the row's FP64
 * sum rounded to FP32, rows summed as s_i p_i + sum_j a_ij (p_j - p_i) in
 * entry order.  Row sums and vector updates use fused multiply-adds
 * (fmaf / fma, correctly rounded in software where the CPU has none) where
 * the GPU kernels' a * b + c compile to one: on ill-conditioned matrices the
 * iteration counts follow that rounding.  An update is
 * also due 4096 iterations after the last one.  Returns 1 when the true
 * FP64 residual ||b - A x|| / ||b|| < tol, 2 when the iteration stalled
 * (the true residual at the updates not halved within the last
 * max(16384, iterations to the last halving) iterations, a breakdown, or
 * a non-finite residual; x is then the x of the lowest true residual, from
 * which the library finishes in FP64), else 0. */
typedef struct {
   const int32_t *grp, *gcols, *gtrp, *gtcols;
   const float *gvals, *gtvals;
} OrcFsaiFactors;
#define ORC_RELIABLE(NAME, VT, FMA)                                                                                   \
   static int NAME(int32_t n, const int32_t* rowptr, const int32_t* cols, const double* vals, int precond,         \
                   const OrcFsaiFactors* F, const double* b, double* x, double tol, double delta, int32_t maxit,  \
                   int excess, int32_t* iterations, int32_t* updates, double* resid)                              \
   {                                                                                                              \
      const int32_t nnz = rowptr[n];                                                                              \
      float* v32 = (float*)malloc(sizeof(float) * (size_t)(nnz > 0 ? nnz : 1));                                   \
      float* s32 = (float*)malloc(sizeof(float) * (size_t)(n > 0 ? n : 1));                                       \
      float* d = (float*)malloc(sizeof(float) * (size_t)n);                                                       \
      VT *r = (VT*)malloc(sizeof(VT) * (size_t)n), *z = (VT*)malloc(sizeof(VT) * (size_t)n);                      \
      VT *p = (VT*)calloc((size_t)n, sizeof(VT)), *Ap = (VT*)malloc(sizeof(VT) * (size_t)n);                      \
      double* xc = (double*)calloc((size_t)n, sizeof(double)); /* the correction is FP64 */                      \
      VT* t = (VT*)malloc(sizeof(VT) * (size_t)(n > 0 ? n : 1));                                                  \
      double* xbest = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));                                  \
      double lowest = HUGE_VAL;                                                                                   \
      for (int32_t k = 0; k < nnz; k++) v32[k] = (float)vals[k];                                                  \
      for (int32_t i = 0; i < n && excess; i++) { /* row excess: the FP64 row sum; off without a diagonal */      \
         double e = 0.0;                                                                                          \
         int has = 0;                                                                                             \
         for (int32_t k = rowptr[i]; k < rowptr[i + 1]; k++) {                                                    \
            e += vals[k];                                                                                         \
            has |= cols[k] == i;                                                                                  \
         }                                                                                                        \
         s32[i] = (float)e;                                                                                       \
         if (!has) excess = 0;                                                                                    \
      }                                                                                                           \
      for (int32_t i = 0; i < n; i++) {                                                                           \
         float di = 0.0f;                                                                                         \
         for (int32_t k = rowptr[i]; k < rowptr[i + 1]; k++)                                                      \
            if (cols[k] == i) di = v32[k];                                                                        \
         d[i] = di;                                                                                               \
      }                                                                                                           \
      double rz = 1.0, rz_cur = 0.0, res = 0.0, best = HUGE_VAL;                                                  \
      int32_t it = 0, upd = 0, halt = 1, ok = 0, force_at = 0, it_best = 0;                                       \
      for (;;) {                                                                                                  \
         for (int32_t i = 0; i < n; i++) {                                                                        \
            x[i] += xc[i];                                                                                        \
            xc[i] = 0.0;                                                                                          \
         }                                                                                                        \
         double rn2 = 0.0, bn2 = 0.0;                                                                             \
         for (int32_t i = 0; i < n; i++) {                                                                        \
            double acc = 0.0;                                                                                     \
            for (int32_t k = rowptr[i]; k < rowptr[i + 1]; k++)                                                   \
               if (cols[k] >= 0) acc += vals[k] * x[cols[k]];                                                     \
            const double di = b[i] - acc;                                                                         \
            r[i] = (VT)di;                                                                                        \
            rn2 += di * di;                                                                                       \
            bn2 += b[i] * b[i];                                                                                   \
         }                                                                                                        \
         const double rn = sqrt(rn2), bn = sqrt(bn2);                                                             \
         res = bn > 0 ? rn / bn : 0.0;                                                                            \
         if (bn == 0 || res < tol) {                                                                              \
            ok = 1;                                                                                               \
            break;                                                                                                \
         }                                                                                                        \
         if (!isfinite(res)) {                                                                                    \
            ok = 2;                                                                                               \
            break;                                                                                                \
         }                                                                                                        \
         if (res < lowest) {                                                                                      \
            lowest = res;                                                                                         \
            memcpy(xbest, x, sizeof(double) * (size_t)n);                                                         \
         }                                                                                                        \
         if (halt == 2) {                                                                                         \
            ok = 2;                                                                                               \
            break;                                                                                                \
         }                                                                                                        \
         if (it >= maxit) break;                                                                                  \
         if (res < 0.5 * best) {                                                                                  \
            best = res;                                                                                           \
            it_best = it;                                                                                         \
         }                                                                                                        \
         else if (it - it_best > (it_best > 16384 ? it_best : 16384)) {                                           \
            ok = 2;                                                                                               \
            break;                                                                                                \
         }                                                                                                        \
         if (it > 0) upd++;                                                                                       \
         force_at = it + 4096;                                                                                    \
         const double t1 = delta * rn, t2 = tol * bn;                                                             \
         const double trig2 = t1 > t2 ? t1 * t1 : t2 * t2;                                                        \
         halt = 0;                                                                                                \
         rz_cur = 0.0;                                                                                            \
         if (precond == 2)                                                                                        \
            rz_cur = NAME##_fsai(n, F, r, t, z);                                                                  \
         else                                                                                                     \
            for (int32_t i = 0; i < n; i++) {                                                                     \
               z[i] = precond == 1 ? r[i] / (VT)d[i] : r[i];                                                      \
               rz_cur += (double)r[i] * (double)z[i];                                                             \
            }                                                                                                     \
         {                                                                                                        \
            const VT beta = (VT)(rz_cur / rz);                                                                    \
            for (int32_t i = 0; i < n; i++) p[i] = FMA(beta, p[i], z[i]);                                         \
         }                                                                                                        \
         while (!halt) {                                                                                          \
            double pap = 0.0;                                                                                     \
            for (int32_t i = 0; i < n; i++) {                                                                     \
               VT s = (VT)0;                                                                                      \
               for (int32_t k = rowptr[i]; k < rowptr[i + 1]; k++)                                                \
                  if (cols[k] >= 0) {                                                                             \
                     if (!excess)                                                                                 \
                        s = FMA((VT)v32[k], p[cols[k]], s);                                                       \
                     else if (cols[k] == i)                                                                       \
                        s = FMA((VT)s32[i], p[i], s);                                                             \
                     else                                                                                         \
                        s = FMA((VT)v32[k], p[cols[k]] - p[i], s);                                                \
                  }                                                                                               \
               Ap[i] = s;                                                                                         \
               pap += (double)s * (double)p[i];                                                                   \
            }                                                                                                     \
            rz = rz_cur;                                                                                          \
            if (pap == 0.0 || !isfinite(pap)) {                                                                   \
               halt = 2;                                                                                          \
               break;                                                                                             \
            }                                                                                                     \
            const VT alpha = (VT)(rz / pap);                                                                      \
            double rr = 0.0, rzn = 0.0;                                                                           \
            for (int32_t i = 0; i < n; i++) {                                                                     \
               xc[i] += (double)alpha * (double)p[i];                                                             \
               r[i] = FMA(-alpha, Ap[i], r[i]);                                                                    \
               rr += (double)r[i] * (double)r[i];                                                                 \
               if (precond != 2) {                                                                                \
                  z[i] = precond == 1 ? r[i] / (VT)d[i] : r[i];                                                   \
                  rzn += (double)r[i] * (double)z[i];                                                             \
               }                                                                                                  \
            }                                                                                                     \
            if (precond == 2) rzn = NAME##_fsai(n, F, r, t, z);                                                   \
            it++;                                                                                                 \
            if (!isfinite(rr))                                                                                    \
               halt = 2;                                                                                          \
            else if (rr < trig2 || it >= force_at)                                                                \
               halt = 1;                                                                                          \
            else if (it >= maxit)                                                                                 \
               halt = 3;                                                                                          \
            if (halt) break;                                                                                      \
            rz_cur = rzn;                                                                                         \
            const VT beta = (VT)(rz_cur / rz);                                                                    \
            for (int32_t i = 0; i < n; i++) p[i] = FMA(beta, p[i], z[i]);                                         \
         }                                                                                                        \
      }                                                                                                           \
      if (ok == 2 && lowest < HUGE_VAL && !(res <= lowest)) { /* back to the lowest true residual */            \
         memcpy(x, xbest, sizeof(double) * (size_t)n);                                                            \
         res = lowest;                                                                                            \
      }                                                                                                           \
      *iterations = it;                                                                                           \
      *updates = upd;                                                                                             \
      *resid = res;                                                                                               \
      free(xbest);                                                                                                \
      free(v32);                                                                                                  \
      free(s32);                                                                                                  \
      free(d);                                                                                                    \
      free(r);                                                                                                    \
      free(z);                                                                                                    \
      free(p);                                                                                                    \
      free(Ap);                                                                                                   \
      free(xc);                                                                                                   \
      free(t);                                                                                                    \
      return ok;                                                                                                  \
   }

/* t = G r, z = G^T t, returns (t, t) = (r, z). */
#define ORC_FSAI_APPLY(NAME, VT, FMA)                                                                                 \
   static double NAME(int32_t n, const OrcFsaiFactors* F, const VT* r, VT* t, VT* z)                             \
   {                                                                                                              \
      double rz = 0.0;                                                                                            \
      for (int32_t i = 0; i < n; i++) {                                                                           \
         VT s = (VT)0;                                                                                            \
         for (int32_t k = F->grp[i]; k < F->grp[i + 1]; k++) s = FMA((VT)F->gvals[k], r[F->gcols[k]], s);         \
         t[i] = s;                                                                                                \
         rz += (double)s * (double)s;                                                                             \
      }                                                                                                           \
      for (int32_t i = 0; i < n; i++) {                                                                           \
         VT s = (VT)0;                                                                                            \
         for (int32_t k = F->gtrp[i]; k < F->gtrp[i + 1]; k++) s = FMA((VT)F->gtvals[k], t[F->gtcols[k]], s);    \
         z[i] = s;                                                                                                \
      }                                                                                                           \
      return rz;                                                                                                  \
   }
ORC_FSAI_APPLY(reliable_f32_fsai, float, fmaf)
ORC_FSAI_APPLY(reliable_f64_fsai, double, fma)
#undef ORC_FSAI_APPLY

ORC_RELIABLE(reliable_f32, float, fmaf)
ORC_RELIABLE(reliable_f64, double, fma)
#undef ORC_RELIABLE

int orc_pcg_reliable(int32_t n, const int32_t* rowptr, const int32_t* cols, const double* vals, int precond,
                     const double* b, double* x, double tol, double delta, int32_t maxit, int vec64, int excess,
                     int32_t* iterations, int32_t* updates, double* resid)
{
   if (precond == 2) return 0;
   if (vec64)
      return reliable_f64(n, rowptr, cols, vals, precond, NULL, b, x, tol, delta, maxit, excess, iterations, updates,
                          resid);
   return reliable_f32(n, rowptr, cols, vals, precond, NULL, b, x, tol, delta, maxit, excess, iterations, updates,
                       resid);
}

/* The same with an FSAI factor pair (precond 2). */
int orc_pcg_reliable_fsai(int32_t n, const int32_t* rowptr, const int32_t* cols, const double* vals,
                          const int32_t* grp, const int32_t* gcols, const float* gvals, const int32_t* gtrp,
                          const int32_t* gtcols, const float* gtvals, const double* b, double* x, double tol,
                          double delta, int32_t maxit, int vec64, int excess, int32_t* iterations,
                          int32_t* updates, double* resid)
{
   const OrcFsaiFactors F = {grp, gcols, gtrp, gtcols, gvals, gtvals};
   if (vec64)
      return reliable_f64(n, rowptr, cols, vals, 2, &F, b, x, tol, delta, maxit, excess, iterations, updates, resid);
   return reliable_f32(n, rowptr, cols, vals, 2, &F, b, x, tol, delta, maxit, excess, iterations, updates, resid);
}
