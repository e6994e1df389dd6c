// transpose.cu -- B = multiplicator * A^T as device CSR arrays
// (SparseMatrix::getTransposition, Matrices/SparseMatrix.hpp:495-551).
//
// The reference counts the entries of every column with atomic adds, sets
// those counts as the row capacities of B and writes each entry of A at an
// atomically claimed slot of its row of B.  With one thread the rows of B
// come out in ascending column order (the rows of A are walked in order);
// with several the order inside a row of B depends on the race.  Here the
// entries are sorted once by (column, row) -- a stable radix sort of 64-bit
// keys -- so the rows of B are always in ascending column order, the
// single-threaded reference's result.
#include <cub/device/device_radix_sort.cuh>

#include "internal.cuh"
#include "segview.cuh"

namespace tnlb {

namespace {

// Entries per column over all storage slots (padding slots hold column -1).
__global__ void k_count_cols(const int32_t* __restrict__ cols, int64_t slots, int32_t columns, int32_t* __restrict__ cnt,
                             int32_t* __restrict__ bad)
{
   for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < slots; q += (int64_t)gridDim.x * blockDim.x) {
      const int32_t c = cols[q];
      if (c >= 0 && c < columns)
         atomicAdd(cnt + c, 1);
      else if (c != -1)
         *bad = 1;
   }
}

// key = column << 32 | row, value = position in the CSR copy of A
__global__ void k_transpose_keys(const int32_t* __restrict__ rp, const int32_t* __restrict__ cols, int32_t n,
                                 uint64_t* __restrict__ keys, int32_t* __restrict__ src)
{
   const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (i >= n) return;
   for (int32_t q = rp[i]; q < rp[i + 1]; q++) {
      keys[q] = ((uint64_t)(uint32_t)cols[q] << 32) | (uint32_t)i;
      src[q] = q;
   }
}

template <typename Real>
__global__ void k_transpose_fill(const uint64_t* __restrict__ keys, const int32_t* __restrict__ src, int64_t nnz,
                                 const Real* __restrict__ vals, Real mult, int32_t* __restrict__ tcols,
                                 Real* __restrict__ tvals)
{
   for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < nnz; q += (int64_t)gridDim.x * blockDim.x) {
      tcols[q] = (int32_t)(uint32_t)(keys[q] & 0xffffffffu);
      tvals[q] = vals[src[q]] * mult;
   }
}

int bits_for(int64_t v)
{
   int b = 1;
   while (b < 32 && (int64_t(1) << b) <= v) b++;
   return b;
}

}  // namespace

// Row pointer of B (columns + 1 entries) and its number of entries.
tnlb_status transpose_rowptr(const tnlb_segments* seg, const int32_t* cols, int32_t columns, int32_t* trowptr,
                             int64_t* nnz_out, cudaStream_t st)
{
   const int64_t slots = seg->storage;
   DeviceBuffer cnt, bad;
   TNLB_TRY_STATUS(cnt.alloc(sizeof(int32_t) * (size_t)(columns > 0 ? columns : 1)));
   TNLB_TRY_STATUS(bad.alloc(sizeof(int32_t)));
   TNLB_CUDA_TRY(cudaMemsetAsync(cnt.ptr, 0, sizeof(int32_t) * (size_t)(columns > 0 ? columns : 1), st));
   TNLB_CUDA_TRY(cudaMemsetAsync(bad.ptr, 0, sizeof(int32_t), st));
   if (slots > 0) {
      k_count_cols<<<grid_for(slots, 256 * 4), 256, 0, st>>>(cols, slots, columns, cnt.as<int32_t>(),
                                                             bad.as<int32_t>());
      TNLB_CHECK_LAUNCH();
   }
   int32_t hbad = 0;
   TNLB_CUDA_TRY(cudaMemcpyAsync(&hbad, bad.ptr, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
   TNLB_CUDA_TRY(cudaStreamSynchronize(st));
   TNLB_REQUIRE(!hbad, TNLB_ERR_INVALID_ARGUMENT, "getTransposition: a column index lies outside [0, columns)");
   int64_t nnz = 0;
   TNLB_TRY_STATUS(exclusive_scan_i32(cnt.as<int32_t>(), trowptr, columns, &nnz, st, true));
   TNLB_CUDA_TRY(cudaStreamSynchronize(st));
   *nnz_out = nnz;
   return TNLB_OK;
}

// Columns and values of B (rows of B in ascending column order).
tnlb_status transpose_fill(const tnlb_segments* seg, tnlb_real real, const int32_t* cols, const void* vals,
                           int32_t columns, double mult, int32_t* tcols, void* tvals, cudaStream_t st)
{
   DeviceBuffer rp, oc, ov;
   TNLB_TRY_STATUS(gather_csr(view_of(seg), real, cols, vals, rp, oc, ov, st));
   int32_t nnz32 = 0;
   TNLB_CUDA_TRY(cudaMemcpyAsync(&nnz32, rp.as<int32_t>() + seg->n, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
   TNLB_CUDA_TRY(cudaStreamSynchronize(st));
   const int64_t nnz = nnz32;
   if (nnz == 0) return TNLB_OK;
   DeviceBuffer keys, keys2, src, src2, temp;
   TNLB_TRY_STATUS(keys.alloc(sizeof(uint64_t) * nnz));
   TNLB_TRY_STATUS(keys2.alloc(sizeof(uint64_t) * nnz));
   TNLB_TRY_STATUS(src.alloc(sizeof(int32_t) * nnz));
   TNLB_TRY_STATUS(src2.alloc(sizeof(int32_t) * nnz));
   k_transpose_keys<<<grid_for(seg->n, 256), 256, 0, st>>>(rp.as<int32_t>(), oc.as<int32_t>(), seg->n,
                                                           keys.as<uint64_t>(), src.as<int32_t>());
   TNLB_CHECK_LAUNCH();
   // sort on the row bits and the column bits only
   const int end_bit = 32 + bits_for(columns);
   size_t temp_bytes = 0;
   TNLB_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, temp_bytes, keys.as<uint64_t>(), keys2.as<uint64_t>(),
                                                 src.as<int32_t>(), src2.as<int32_t>(), (int)nnz, 0, end_bit, st));
   TNLB_TRY_STATUS(temp.alloc(temp_bytes > 0 ? temp_bytes : 1));
   TNLB_CUDA_TRY(cub::DeviceRadixSort::SortPairs(temp.ptr, temp_bytes, keys.as<uint64_t>(), keys2.as<uint64_t>(),
                                                 src.as<int32_t>(), src2.as<int32_t>(), (int)nnz, 0, end_bit, st));
   if (real == TNLB_F64)
      k_transpose_fill<double><<<grid_for(nnz, 256 * 4), 256, 0, st>>>(
         keys2.as<uint64_t>(), src2.as<int32_t>(), nnz, ov.as<double>(), mult, tcols, (double*)tvals);
   else
      k_transpose_fill<float><<<grid_for(nnz, 256 * 4), 256, 0, st>>>(
         keys2.as<uint64_t>(), src2.as<int32_t>(), nnz, ov.as<float>(), (float)mult, tcols, (float*)tvals);
   TNLB_CHECK_LAUNCH();
   TNLB_CUDA_TRY(cudaStreamSynchronize(st));
   return TNLB_OK;
}

}  // namespace tnlb

extern "C" tnlb_status tnlb_matrix_transpose_rowptr(const tnlb_segments* seg, const int32_t* d_cols, int32_t columns,
                                                    int32_t* d_trowptr, int64_t* h_nnz, tnlb_stream stream)
{
   using namespace tnlb;
   clear_error();
   TNLB_REQUIRE(seg && d_trowptr && h_nnz, TNLB_ERR_INVALID_ARGUMENT, "null argument");
   TNLB_REQUIRE(columns >= 0, TNLB_ERR_INVALID_ARGUMENT, "negative number of columns");
   return transpose_rowptr(seg, d_cols, columns, d_trowptr, h_nnz, (cudaStream_t)stream);
}

extern "C" tnlb_status tnlb_matrix_transpose_fill(const tnlb_segments* seg, tnlb_real real, const int32_t* d_cols,
                                                  const void* d_values, int32_t columns, double multiplicator,
                                                  int32_t* d_tcols, void* d_tvalues, tnlb_stream stream)
{
   using namespace tnlb;
   clear_error();
   TNLB_REQUIRE(seg, TNLB_ERR_INVALID_ARGUMENT, "null argument");
   TNLB_REQUIRE(real == TNLB_F32 || real == TNLB_F64, TNLB_ERR_INVALID_ARGUMENT, "unknown real type");
   TNLB_REQUIRE(columns >= 0, TNLB_ERR_INVALID_ARGUMENT, "negative number of columns");
   return transpose_fill(seg, real, d_cols, d_values, columns, multiplicator, d_tcols, d_tvalues,
                         (cudaStream_t)stream);
}
