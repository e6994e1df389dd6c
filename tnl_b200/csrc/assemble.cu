// assemble.cu -- device-side matrix assembly (SparseMatrixBase::forAllRows /
// forElements, Matrices/SparseMatrixBase.h:589, 858, with the lambda of the
// reference's sparse set-up benchmark, Documentation/UsersGuide/Matrices/
// SparseMatrixSetup_Benchmark.cpp): the 2D Laplace operator of a grid of
// side N written straight into a matrix's storage on the GPU, any segment
// format, one thread per row, through the segments' index map.  Boundary
// rows are identity rows (1 on the diagonal); interior rows hold
// 1, 1, -4, 1, 1 at columns i - N, i - 1, i, i + 1, i + N.  The row
// capacities must be at least 1 on the boundary and 5 inside (the
// benchmark sets 5 everywhere); the slots a row does not use keep the
// padding column -1 and value 0.
//
// A C++ caller with its own device lambda uses SparseMatrix::forElements
// of include/tnlb/tnlb.hpp instead, which runs the lambda on the CSR rows
// of tnlb_segments_offsets_view.
#include "internal.cuh"
#include "segview.cuh"

namespace tnlb {
namespace {

template <typename Real>
__global__ void k_laplace_2d(SegView v, int32_t N, int32_t* __restrict__ cols, Real* __restrict__ vals,
                             int32_t* __restrict__ err)
{
   const int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (row >= v.n) return;
   const int32_t i = (int32_t)(row % N), j = (int32_t)(row / N);
   const int32_t r = (int32_t)row;
   auto put = [&](int32_t local, int32_t c, Real a) {
      const int64_t g = global_index_of(v, r, local);
      if (g < 0) {
         atomicExch(err, 1);
         return;
      }
      cols[g] = c;
      vals[g] = a;
   };
   if (i == 0 || j == 0 || i == N - 1 || j == N - 1)
      put(0, r, Real(1));
   else {
      put(0, r - N, Real(1));
      put(1, r - 1, Real(1));
      put(2, r, Real(-4));
      put(3, r + 1, Real(1));
      put(4, r + N, Real(1));
   }
}

}  // namespace
}  // namespace tnlb

extern "C" tnlb_status tnlb_matrix_assemble_laplace_2d(const tnlb_segments* seg, tnlb_real real, int32_t grid_size,
                                                       int32_t* d_cols, void* d_values, tnlb_stream stream)
{
   using namespace tnlb;
   clear_error();
   TNLB_REQUIRE(seg && d_cols && d_values, TNLB_ERR_INVALID_ARGUMENT, "null argument");
   TNLB_REQUIRE(real == TNLB_F32 || real == TNLB_F64, TNLB_ERR_INVALID_ARGUMENT, "unknown real type");
   TNLB_REQUIRE(grid_size > 0 && (int64_t)grid_size * grid_size == seg->n, TNLB_ERR_INVALID_ARGUMENT,
                "assemble_laplace_2d: the segments must have grid_size^2 rows");
   cudaStream_t st = (cudaStream_t)stream;
   DeviceBuffer err;
   TNLB_TRY_STATUS(err.alloc(sizeof(int32_t)));
   TNLB_CUDA_TRY(cudaMemsetAsync(err.ptr, 0, sizeof(int32_t), st));
   const SegView v = view_of(seg);
   if (real == TNLB_F64)
      k_laplace_2d<double><<<grid_for(seg->n, 256), 256, 0, st>>>(v, grid_size, d_cols, (double*)d_values,
                                                                  err.as<int32_t>());
   else
      k_laplace_2d<float><<<grid_for(seg->n, 256), 256, 0, st>>>(v, grid_size, d_cols, (float*)d_values,
                                                                 err.as<int32_t>());
   TNLB_CHECK_LAUNCH();
   int32_t h = 0;
   TNLB_CUDA_TRY(cudaMemcpyAsync(&h, err.ptr, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
   TNLB_CUDA_TRY(cudaStreamSynchronize(st));
   TNLB_REQUIRE(h == 0, TNLB_ERR_INVALID_ARGUMENT,
                "assemble_laplace_2d: a row's capacity is smaller than the entries of its stencil");
   return TNLB_OK;
}

extern "C" tnlb_status tnlb_segments_offsets_view(const tnlb_segments* seg, const int32_t** d_offsets)
{
   using namespace tnlb;
   clear_error();
   TNLB_REQUIRE(seg && d_offsets, TNLB_ERR_INVALID_ARGUMENT, "null argument");
   TNLB_REQUIRE(seg->format == TNLB_CSR || seg->format == TNLB_ADAPTIVE_CSR, TNLB_ERR_INVALID_ARGUMENT,
                "segments_offsets_view: only the CSR formats store their rows contiguously");
   *d_offsets = seg->offsets.as<int32_t>();
   return TNLB_OK;
}
