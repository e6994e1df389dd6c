// api.cu -- the extern "C" entry points of libtnlb200.so declared in
// include/tnlb200.h.  No entry point throws; failures return a status and
// leave a message for tnlb_last_error().
#include <cfloat>
#include <new>

#include "fsai.cuh"
#include "internal.cuh"
#include "lfsai.cuh"

namespace tnlb {

namespace {
thread_local std::string g_last_error;
thread_local int32_t g_last_launches = 0;
}  // namespace

void set_error(const std::string& msg) { g_last_error = msg; }
void clear_error() { g_last_error.clear(); }

namespace {

// y = alpha x + beta y (beta == 0: y is not read)
template <typename Real>
__global__ void k_axpby(int64_t n, Real alpha, const Real* __restrict__ x, Real beta, Real* __restrict__ y)
{
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
      y[i] = beta == Real(0) ? alpha * x[i] : alpha * x[i] + beta * y[i];
}

template <typename T>
__global__ void k_dot(int64_t n, const T* __restrict__ a, const T* __restrict__ b, double* __restrict__ out)
{
   __shared__ double part[8];
   double s = 0;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
      s += (double)a[i] * (double)b[i];
   s = warp_sum(s);
   if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
   __syncthreads();
   if (threadIdx.x < 32) {
      s = threadIdx.x < 8 ? part[threadIdx.x] : 0.0;
      s = warp_sum(s);
      if (threadIdx.x == 0) atomicAdd(out, s);
   }
}

tnlb_status copy_meta(const tnlb::DeviceBuffer& buf, int64_t elems, int32_t* h_out, int64_t count)
{
   TNLB_REQUIRE(count >= elems, TNLB_ERR_INVALID_ARGUMENT,
                "metadata buffer too small: need " + std::to_string(elems) + " elements");
   if (elems > 0) TNLB_CUDA_TRY(cudaMemcpy(h_out, buf.ptr, sizeof(int32_t) * (size_t)elems, cudaMemcpyDeviceToHost));
   return TNLB_OK;
}

}  // namespace
}  // namespace tnlb

using namespace tnlb;

extern "C" {

const char* tnlb_last_error(void) { return g_last_error.c_str(); }

const char* tnlb_version(void) { return "tnlb200 0.1.0 (sm_100a)"; }

tnlb_status tnlb_segments_create(tnlb_format format, tnlb_organization organization, const int32_t* d_sizes,
                                 int32_t segments, tnlb_stream stream, tnlb_segments** out)
{
   clear_error();
   TNLB_REQUIRE(out != nullptr, TNLB_ERR_INVALID_ARGUMENT, "out is null");
   *out = nullptr;
   TNLB_REQUIRE(segments >= 0, TNLB_ERR_INVALID_ARGUMENT, "negative segment count");
   TNLB_REQUIRE(segments == 0 || d_sizes != nullptr, TNLB_ERR_INVALID_ARGUMENT, "sizes are null");
   TNLB_REQUIRE(format >= TNLB_CSR && format <= TNLB_ADAPTIVE_CSR, TNLB_ERR_INVALID_ARGUMENT, "unknown format");
   TNLB_REQUIRE(organization == TNLB_COLUMN_MAJOR || organization == TNLB_ROW_MAJOR, TNLB_ERR_INVALID_ARGUMENT,
                "unknown elements organization");
   tnlb_segments* seg = new (std::nothrow) tnlb_segments();
   TNLB_REQUIRE(seg != nullptr, TNLB_ERR_OUT_OF_MEMORY, "out of host memory");
   seg->format = format;
   seg->organization = organization;
   seg->n = segments;
   TNLB_CUDA_TRY(cudaGetDevice(&seg->device));
   tnlb_status s = build_segments(seg, d_sizes, (cudaStream_t)stream);
   if (s == TNLB_OK) {
      cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
      if (e != cudaSuccess) {
         set_error(std::string("segments build: ") + cudaGetErrorString(e));
         s = TNLB_ERR_CUDA;
      }
   }
   if (s != TNLB_OK) {
      delete seg;
      return s;
   }
   *out = seg;
   return TNLB_OK;
}

tnlb_status tnlb_segments_destroy(tnlb_segments* seg)
{
   clear_error();
   delete seg;
   return TNLB_OK;
}

tnlb_status tnlb_segments_get_info(const tnlb_segments* seg, tnlb_segments_info* info)
{
   clear_error();
   TNLB_REQUIRE(seg && info, TNLB_ERR_INVALID_ARGUMENT, "null argument");
   *info = tnlb_segments_info{};
   info->format = seg->format;
   info->organization = seg->organization;
   info->segments = seg->n;
   info->elements = seg->elements;
   info->storage = seg->storage;
   info->segment_size = seg->segment_size;
   info->aligned_size = seg->aligned_size;
   info->slices = seg->format == TNLB_SLICED_ELLPACK ? seg->slices
                : seg->format == TNLB_CHUNKED_ELLPACK ? seg->ch_slices
                : seg->format == TNLB_BIELLPACK ? seg->strips
                                                : 0;
   info->chunks_in_slice = kChunksInSlice;
   for (int k = 0; k < 6; k++) info->acsr_blocks[k] = seg->acsr_count[k];
   return TNLB_OK;
}

tnlb_status tnlb_segments_read_metadata(const tnlb_segments* seg, tnlb_metadata which, int32_t* h_out, int64_t count)
{
   clear_error();
   TNLB_REQUIRE(seg && (h_out || count == 0), TNLB_ERR_INVALID_ARGUMENT, "null argument");
   const int64_t n = seg->n;
   const bool csr = seg->format == TNLB_CSR || seg->format == TNLB_ADAPTIVE_CSR;
   const bool sell = seg->format == TNLB_SLICED_ELLPACK;
   const bool ch = seg->format == TNLB_CHUNKED_ELLPACK;
   const bool bi = seg->format == TNLB_BIELLPACK;
   const int64_t cs = seg->ch_slices;
   switch (which) {
      case TNLB_META_OFFSETS:
         TNLB_REQUIRE(csr, TNLB_ERR_INVALID_ARGUMENT, "not a CSR format");
         return copy_meta(seg->offsets, n + 1, h_out, count);
      case TNLB_META_SLICE_OFFSETS:
         TNLB_REQUIRE(sell, TNLB_ERR_INVALID_ARGUMENT, "not SlicedEllpack");
         return copy_meta(seg->slice_offsets, (int64_t)seg->slices + 1, h_out, count);
      case TNLB_META_SLICE_SEGMENT_SIZES:
         TNLB_REQUIRE(sell, TNLB_ERR_INVALID_ARGUMENT, "not SlicedEllpack");
         return copy_meta(seg->slice_segment_sizes, seg->slices, h_out, count);
      case TNLB_META_CH_SLICE_SIZE:
         TNLB_REQUIRE(ch, TNLB_ERR_INVALID_ARGUMENT, "not ChunkedEllpack");
         return copy_meta(seg->ch_slice_size, cs, h_out, count);
      case TNLB_META_CH_SLICE_CHUNK_SIZE:
         TNLB_REQUIRE(ch, TNLB_ERR_INVALID_ARGUMENT, "not ChunkedEllpack");
         return copy_meta(seg->ch_slice_chunk_size, cs, h_out, count);
      case TNLB_META_CH_SLICE_FIRST:
         TNLB_REQUIRE(ch, TNLB_ERR_INVALID_ARGUMENT, "not ChunkedEllpack");
         return copy_meta(seg->ch_slice_first, cs, h_out, count);
      case TNLB_META_CH_SLICE_POINTER:
         TNLB_REQUIRE(ch, TNLB_ERR_INVALID_ARGUMENT, "not ChunkedEllpack");
         return copy_meta(seg->ch_slice_pointer, cs, h_out, count);
      case TNLB_META_CH_SEGMENT_TO_CHUNK:
         TNLB_REQUIRE(ch, TNLB_ERR_INVALID_ARGUMENT, "not ChunkedEllpack");
         return copy_meta(seg->ch_segment_to_chunk, n, h_out, count);
      case TNLB_META_CH_SEGMENT_TO_SLICE:
         TNLB_REQUIRE(ch, TNLB_ERR_INVALID_ARGUMENT, "not ChunkedEllpack");
         return copy_meta(seg->ch_segment_to_slice, n, h_out, count);
      case TNLB_META_CH_SEGMENT_POINTERS:
         TNLB_REQUIRE(ch, TNLB_ERR_INVALID_ARGUMENT, "not ChunkedEllpack");
         return copy_meta(seg->ch_segment_pointers, n + 1, h_out, count);
      case TNLB_META_CH_CHUNKS_TO_SEGMENTS:
         TNLB_REQUIRE(ch, TNLB_ERR_INVALID_ARGUMENT, "not ChunkedEllpack");
         return copy_meta(seg->ch_chunks_to_segments, cs * kChunksInSlice, h_out, count);
      case TNLB_META_BI_PERMUTATION:
         TNLB_REQUIRE(bi, TNLB_ERR_INVALID_ARGUMENT, "not BiEllpack");
         return copy_meta(seg->bi_perm, n, h_out, count);
      case TNLB_META_BI_GROUP_POINTERS:
         TNLB_REQUIRE(bi, TNLB_ERR_INVALID_ARGUMENT, "not BiEllpack");
         return copy_meta(seg->bi_group_pointers, (int64_t)seg->strips * kBiGroups + 1, h_out, count);
   }
   set_error("unknown metadata array");
   return TNLB_ERR_INVALID_ARGUMENT;
}

tnlb_status tnlb_segments_read_acsr_blocks(const tnlb_segments* seg, int32_t size_log, tnlb_acsr_block* h_out,
                                           int64_t count)
{
   clear_error();
   TNLB_REQUIRE(seg != nullptr, TNLB_ERR_INVALID_ARGUMENT, "null segments");
   TNLB_REQUIRE(seg->format == TNLB_ADAPTIVE_CSR, TNLB_ERR_INVALID_ARGUMENT, "not AdaptiveCSR");
   TNLB_REQUIRE(size_log >= 0 && size_log < 6, TNLB_ERR_INVALID_ARGUMENT, "size_log must be 0..5");
   const int64_t c = seg->acsr_count[size_log];
   TNLB_REQUIRE(count >= c, TNLB_ERR_INVALID_ARGUMENT, "descriptor buffer too small");
   if (c > 0)
      TNLB_CUDA_TRY(cudaMemcpy(h_out, seg->acsr_blocks[size_log].ptr, sizeof(tnlb_acsr_block) * (size_t)c,
                               cudaMemcpyDeviceToHost));
   return TNLB_OK;
}

tnlb_status tnlb_segments_global_index(const tnlb_segments* seg, const int32_t* d_segment, const int32_t* d_local,
                                       int64_t count, int64_t* d_global, tnlb_stream stream)
{
   clear_error();
   TNLB_REQUIRE(seg != nullptr, TNLB_ERR_INVALID_ARGUMENT, "null segments");
   TNLB_REQUIRE(count == 0 || (d_segment && d_local && d_global), TNLB_ERR_INVALID_ARGUMENT, "null array");
   return global_index(seg, d_segment, d_local, count, d_global, (cudaStream_t)stream);
}

tnlb_status tnlb_matrix_fill_from_csr(const tnlb_segments* seg, tnlb_real real, const int32_t* d_rowptr,
                                      const int32_t* d_src_cols, const void* d_src_values, int32_t* d_cols,
                                      void* d_values, tnlb_stream stream)
{
   clear_error();
   TNLB_REQUIRE(seg != nullptr, TNLB_ERR_INVALID_ARGUMENT, "null segments");
   TNLB_REQUIRE(real == TNLB_F32 || real == TNLB_F64, TNLB_ERR_INVALID_ARGUMENT, "unknown real type");
   TNLB_REQUIRE(seg->n == 0 || (d_rowptr && d_src_cols && d_src_values), TNLB_ERR_INVALID_ARGUMENT,
                "null source array");
   TNLB_REQUIRE(seg->storage == 0 || (d_cols && d_values), TNLB_ERR_INVALID_ARGUMENT, "null target array");
   return fill_from_csr(seg, real, d_rowptr, d_src_cols, d_src_values, d_cols, d_values, (cudaStream_t)stream);
}

tnlb_status tnlb_spmv(const tnlb_segments* seg, tnlb_real real, const int32_t* d_cols, const void* d_values,
                      int32_t columns, const void* d_x, void* d_y, double alpha, double beta, int32_t begin,
                      int32_t end, tnlb_kernel kernel, int32_t threads_per_segment, tnlb_stream stream)
{
   clear_error();
   g_last_launches = 0;
   TNLB_REQUIRE(seg != nullptr, TNLB_ERR_INVALID_ARGUMENT, "null segments");
   TNLB_REQUIRE(real == TNLB_F32 || real == TNLB_F64, TNLB_ERR_INVALID_ARGUMENT, "unknown real type");
   TNLB_REQUIRE(columns >= 0, TNLB_ERR_INVALID_ARGUMENT,
                "vectorProduct: size of the input vector does not match the number of matrix columns");
   if (end == 0) end = seg->n;
   TNLB_REQUIRE(begin >= 0 && begin <= end && end <= seg->n, TNLB_ERR_INVALID_ARGUMENT,
                "vectorProduct: row range [begin, end) outside the matrix");
   TNLB_REQUIRE(threads_per_segment == 0 || (threads_per_segment > 0 && threads_per_segment <= 256 &&
                                             (threads_per_segment & (threads_per_segment - 1)) == 0),
                TNLB_ERR_INVALID_ARGUMENT, "Threads per segment count must be a positive power of two.");
   if (end == begin) return TNLB_OK;
   TNLB_REQUIRE(d_y != nullptr && (seg->storage == 0 || (d_cols && d_values && d_x)), TNLB_ERR_INVALID_ARGUMENT,
                "null array");
   int launches = 0;
   tnlb_status s;
   if (seg->format == TNLB_CSR || seg->format == TNLB_ADAPTIVE_CSR) {
      tnlb_kernel k = kernel;
      if (seg->format == TNLB_ADAPTIVE_CSR && kernel == TNLB_KERNEL_DEFAULT) k = TNLB_KERNEL_ADAPTIVE;
      s = spmv_csr(seg, real, d_cols, d_values, d_x, d_y, alpha, beta, begin, end, k, threads_per_segment,
                   (cudaStream_t)stream, &launches);
   }
   else {
      TNLB_REQUIRE(kernel == TNLB_KERNEL_DEFAULT || kernel == TNLB_KERNEL_VECTOR || kernel == TNLB_KERNEL_SCALAR,
                   TNLB_ERR_INVALID_ARGUMENT, "kernel not available for this format");
      s = spmv_ell_family(seg, real, d_cols, d_values, d_x, d_y, alpha, beta, begin, end, kernel,
                          kernel == TNLB_KERNEL_SCALAR ? 1 : threads_per_segment, (cudaStream_t)stream, &launches);
   }
   g_last_launches = launches;
   return s;
}

int32_t tnlb_spmv_last_launch_count(void) { return g_last_launches; }

tnlb_status tnlb_axpby(tnlb_real real, int64_t n, double alpha, const void* d_x, double beta, void* d_y,
                       tnlb_stream stream)
{
   clear_error();
   TNLB_REQUIRE(real == TNLB_F32 || real == TNLB_F64, TNLB_ERR_INVALID_ARGUMENT, "unknown real type");
   TNLB_REQUIRE(n >= 0, TNLB_ERR_INVALID_ARGUMENT, "negative size");
   if (n == 0) return TNLB_OK;
   TNLB_REQUIRE(d_x && d_y, TNLB_ERR_INVALID_ARGUMENT, "null vector");
   cudaStream_t st = (cudaStream_t)stream;
   unsigned g = grid_for(n, 256 * 4);
   if (g > 148 * 8) g = 148 * 8;
   if (real == TNLB_F64)
      k_axpby<double><<<g, 256, 0, st>>>(n, alpha, (const double*)d_x, beta, (double*)d_y);
   else
      k_axpby<float><<<g, 256, 0, st>>>(n, (float)alpha, (const float*)d_x, (float)beta, (float*)d_y);
   TNLB_CHECK_LAUNCH();
   return TNLB_OK;
}

tnlb_status tnlb_dot(tnlb_real real, int64_t n, const void* d_a, const void* d_b, double* d_result, tnlb_stream stream)
{
   clear_error();
   TNLB_REQUIRE(d_result != nullptr, TNLB_ERR_INVALID_ARGUMENT, "null result");
   TNLB_REQUIRE(n == 0 || (d_a && d_b), TNLB_ERR_INVALID_ARGUMENT, "null vector");
   cudaStream_t st = (cudaStream_t)stream;
   TNLB_CUDA_TRY(cudaMemsetAsync(d_result, 0, sizeof(double), st));
   if (n == 0) return TNLB_OK;
   unsigned g = grid_for(n, 256 * 4);
   if (g > 148 * 8) g = 148 * 8;
   if (real == TNLB_F64)
      k_dot<double><<<g, 256, 0, st>>>(n, (const double*)d_a, (const double*)d_b, d_result);
   else
      k_dot<float><<<g, 256, 0, st>>>(n, (const float*)d_a, (const float*)d_b, d_result);
   TNLB_CHECK_LAUNCH();
   return TNLB_OK;
}

void tnlb_solver_params_default(tnlb_solver_params* p)
{
   if (!p) return;
   *p = tnlb_solver_params{};
   p->max_iterations = 1000000000;    // IterativeSolver.h:226
   p->min_iterations = 0;             // :228
   p->convergence_residue = 1e-6;     // :232
   p->divergence_residue = DBL_MAX;   // :235
   p->gmres_variant = TNLB_GMRES_MGSR;  // GMRES.hpp:23 (configSetup default)
   p->gmres_restarting_min = 10;      // GMRES.h:226
   p->gmres_restarting_max = 10;      // GMRES.h:227
   p->gmres_restarting_step_min = 3;  // GMRES.h:228
   p->gmres_restarting_step_max = 3;  // GMRES.h:229
   p->bicgstab_exact_residue = 0;     // BICGStab.h:102
   p->spmv_kernel = TNLB_KERNEL_DEFAULT;
   p->bicgstab_ell = 1;               // BICGStabL.hpp:17
   p->idr_s = 4;                      // IDRs.hpp:21
   p->idr_residual_smoothing = 0;     // IDRs.hpp:22
   p->reliable_layout = 0;
   p->reliable_operator = 0;
}

static tnlb_status check_solve_args(const tnlb_segments* seg, tnlb_real real, const void* b, void* x)
{
   TNLB_REQUIRE(seg != nullptr, TNLB_ERR_INVALID_ARGUMENT, "null segments");
   TNLB_REQUIRE(real == TNLB_F32 || real == TNLB_F64, TNLB_ERR_INVALID_ARGUMENT, "unknown real type");
   TNLB_REQUIRE(seg->n > 0, TNLB_ERR_INVALID_ARGUMENT, "LinearSolver::setMatrix: the matrix is empty");
   TNLB_REQUIRE(b && x, TNLB_ERR_INVALID_ARGUMENT, "null vector");
   return TNLB_OK;
}

tnlb_status tnlb_solve_preconditioned(tnlb_solver_kind solver, const tnlb_precond* precond,
                                      const tnlb_solver_params* params, const tnlb_segments* seg, tnlb_real real,
                                      const int32_t* d_cols, const void* d_values, const void* d_b, void* d_x,
                                      tnlb_stream stream, tnlb_solve_result* result)
{
   clear_error();
   TNLB_TRY_STATUS(check_solve_args(seg, real, d_b, d_x));
   TNLB_REQUIRE(result != nullptr, TNLB_ERR_INVALID_ARGUMENT, "null result");
   TNLB_REQUIRE(solver >= TNLB_SOLVER_CG && solver <= TNLB_SOLVER_IDRS, TNLB_ERR_INVALID_ARGUMENT, "unknown solver");
   tnlb_solver_params p;
   tnlb_solver_params_default(&p);
   if (params) p = *params;
   *result = tnlb_solve_result{};
   tnlb_status s = tnlb::solve(solver, precond, p, seg, real, d_cols, d_values, d_b, d_x, (cudaStream_t)stream, result);
   if (s != TNLB_OK) result->status_detail = s;
   return s;
}

tnlb_status tnlb_solve(tnlb_solver_kind solver, tnlb_precond_kind precond, const tnlb_solver_params* params,
                       const tnlb_segments* seg, tnlb_real real, const int32_t* d_cols, const void* d_values,
                       const void* d_b, void* d_x, tnlb_stream stream, tnlb_solve_result* result)
{
   clear_error();
   TNLB_TRY_STATUS(check_solve_args(seg, real, d_b, d_x));
   TNLB_REQUIRE(precond >= TNLB_PRECOND_NONE && precond <= TNLB_PRECOND_FSAI2, TNLB_ERR_INVALID_ARGUMENT,
                "unknown preconditioner");
   tnlb_precond* P = nullptr;
   if (precond != TNLB_PRECOND_NONE)
      TNLB_TRY_STATUS(tnlb::precond_create(precond, seg, real, d_cols, d_values, (cudaStream_t)stream, &P));
   tnlb_status s = tnlb_solve_preconditioned(solver, P, params, seg, real, d_cols, d_values, d_b, d_x, stream, result);
   delete P;
   return s;
}

tnlb_status tnlb_true_residual(const tnlb_segments* seg, tnlb_real real, const int32_t* d_cols, const void* d_values,
                               const void* d_b, const void* d_x, tnlb_stream stream, double* h_result)
{
   clear_error();
   TNLB_TRY_STATUS(check_solve_args(seg, real, d_b, (void*)d_x));
   TNLB_REQUIRE(h_result != nullptr, TNLB_ERR_INVALID_ARGUMENT, "null result");
   return tnlb::true_residual(seg, real, d_cols, d_values, d_b, d_x, (cudaStream_t)stream, h_result);
}

tnlb_status tnlb_solve_mixed(const tnlb_solver_params* params, const tnlb_segments* seg, const int32_t* d_cols,
                             const double* d_values, const double* d_b, double* d_x, double inner_tolerance,
                             int32_t max_outer, tnlb_solver_kind inner_solver, tnlb_precond_kind inner_precond,
                             const tnlb_precond* inner, tnlb_stream stream, tnlb_solve_result* result,
                             int32_t* outer_iterations)
{
   clear_error();
   TNLB_TRY_STATUS(check_solve_args(seg, TNLB_F64, d_b, d_x));
   TNLB_REQUIRE(result && outer_iterations, TNLB_ERR_INVALID_ARGUMENT, "null result");
   TNLB_REQUIRE(inner_tolerance > 0 && inner_tolerance < 1, TNLB_ERR_INVALID_ARGUMENT,
                "inner tolerance must lie in (0, 1)");
   TNLB_REQUIRE(max_outer >= 0, TNLB_ERR_INVALID_ARGUMENT, "negative max_outer");
   TNLB_REQUIRE(inner_solver >= TNLB_SOLVER_CG && inner_solver <= TNLB_SOLVER_IDRS, TNLB_ERR_INVALID_ARGUMENT,
                "unknown inner solver");
   TNLB_REQUIRE(inner || (inner_precond >= TNLB_PRECOND_NONE && inner_precond <= TNLB_PRECOND_FSAI2),
                TNLB_ERR_INVALID_ARGUMENT, "unknown preconditioner");
   tnlb_solver_params p;
   tnlb_solver_params_default(&p);
   if (params) p = *params;
   int32_t inner_its = 0;
   *result = tnlb_solve_result{};
   return tnlb::solve_mixed_cg(seg, d_cols, d_values, d_b, d_x, p, inner_tolerance, max_outer, (cudaStream_t)stream,
                               result, &inner_its, outer_iterations, inner_precond, inner, inner_solver);
}

tnlb_status tnlb_solve_mixed_reliable(const tnlb_solver_params* params, const tnlb_segments* seg,
                                      const int32_t* d_cols, const double* d_values, const double* d_b, double* d_x,
                                      double delta, tnlb_real vectors, tnlb_precond_kind inner_precond,
                                      const tnlb_precond* inner, tnlb_stream stream, tnlb_solve_result* result,
                                      int32_t* reliable_updates)
{
   clear_error();
   TNLB_TRY_STATUS(check_solve_args(seg, TNLB_F64, d_b, d_x));
   TNLB_REQUIRE(result && reliable_updates, TNLB_ERR_INVALID_ARGUMENT, "null result");
   TNLB_REQUIRE(delta > 0 && delta < 1, TNLB_ERR_INVALID_ARGUMENT, "delta must lie in (0, 1)");
   TNLB_REQUIRE(vectors == TNLB_F32 || vectors == TNLB_F64, TNLB_ERR_INVALID_ARGUMENT, "unknown vector real type");
   TNLB_REQUIRE(inner || inner_precond == TNLB_PRECOND_NONE || inner_precond == TNLB_PRECOND_JACOBI ||
                   inner_precond == TNLB_PRECOND_FSAI,
                TNLB_ERR_INVALID_ARGUMENT, "the preconditioner must be none, Jacobi or FSAI");
   tnlb_solver_params p;
   tnlb_solver_params_default(&p);
   if (params) p = *params;
   TNLB_REQUIRE(p.max_iterations >= 0, TNLB_ERR_INVALID_ARGUMENT, "negative max_iterations");
   TNLB_REQUIRE(p.reliable_layout >= 0 && p.reliable_layout <= 2, TNLB_ERR_INVALID_ARGUMENT,
                "reliable_layout must be 0, 1 or 2");
   TNLB_REQUIRE(p.reliable_operator == 0 || p.reliable_operator == 1, TNLB_ERR_INVALID_ARGUMENT,
                "reliable_operator must be 0 or 1");
   *result = tnlb_solve_result{};
   *reliable_updates = 0;
   return tnlb::solve_mixed_reliable(seg, d_cols, d_values, d_b, d_x, p, delta, vectors, (cudaStream_t)stream, result,
                                     reliable_updates, inner_precond, inner);
}

tnlb_status tnlb_precond_create(tnlb_precond_kind kind, const tnlb_segments* seg, tnlb_real real,
                                const int32_t* d_cols, const void* d_values, tnlb_stream stream, tnlb_precond** out)
{
   clear_error();
   TNLB_REQUIRE(seg && out, TNLB_ERR_INVALID_ARGUMENT, "null argument");
   TNLB_REQUIRE(real == TNLB_F32 || real == TNLB_F64, TNLB_ERR_INVALID_ARGUMENT, "unknown real type");
   TNLB_REQUIRE(kind >= TNLB_PRECOND_NONE && kind <= TNLB_PRECOND_FSAI2, TNLB_ERR_INVALID_ARGUMENT,
                "unknown preconditioner");
   *out = nullptr;
   return tnlb::precond_create(kind, seg, real, d_cols, d_values, (cudaStream_t)stream, out);
}

tnlb_status tnlb_precond_create_fsai(const tnlb_segments* seg, tnlb_real real, const int32_t* d_cols,
                                     const void* d_values, int32_t level, tnlb_stream stream, tnlb_precond** out)
{
   clear_error();
   TNLB_REQUIRE(seg && out, TNLB_ERR_INVALID_ARGUMENT, "null argument");
   TNLB_REQUIRE(real == TNLB_F32 || real == TNLB_F64, TNLB_ERR_INVALID_ARGUMENT, "unknown real type");
   TNLB_REQUIRE(level == 0 || level == 1, TNLB_ERR_INVALID_ARGUMENT, "the pattern level must be 0 or 1");
   TNLB_REQUIRE(seg->n > 0, TNLB_ERR_INVALID_ARGUMENT, "Preconditioner::update: the matrix is empty");
   *out = nullptr;
   auto* P = new tnlb_precond();
   P->kind = TNLB_PRECOND_FSAI;
   P->real = real;
   P->n = seg->n;
   const tnlb_status s = tnlb::fsai_create(seg, real, d_cols, d_values, true, (cudaStream_t)stream, &P->fsai, false,
                                           level);
   if (s != TNLB_OK) {
      delete P;
      return s;
   }
   *out = P;
   return TNLB_OK;
}

tnlb_status tnlb_precond_create_ilut(const tnlb_segments* seg, tnlb_real real, const int32_t* d_cols,
                                     const void* d_values, int32_t p, double threshold, tnlb_stream stream,
                                     tnlb_precond** out)
{
   clear_error();
   TNLB_REQUIRE(seg && out, TNLB_ERR_INVALID_ARGUMENT, "null argument");
   TNLB_REQUIRE(real == TNLB_F32 || real == TNLB_F64, TNLB_ERR_INVALID_ARGUMENT, "unknown real type");
   *out = nullptr;
   auto* P = new tnlb_precond();
   P->kind = TNLB_PRECOND_ILUT;
   P->real = real;
   P->n = seg->n;
   tnlb_status s = tnlb::ilut_create(seg, real, d_cols, d_values, p, threshold, (cudaStream_t)stream, &P->ilu);
   if (s != TNLB_OK) {
      delete P;
      return s;
   }
   *out = P;
   return TNLB_OK;
}

tnlb_status tnlb_precond_solve(const tnlb_precond* precond, const void* d_b, void* d_x, tnlb_stream stream)
{
   clear_error();
   TNLB_REQUIRE(precond && d_b && d_x, TNLB_ERR_INVALID_ARGUMENT, "null argument");
   return tnlb::precond_apply(precond, d_b, d_x, (cudaStream_t)stream);
}

tnlb_status tnlb_precond_read_factor(const tnlb_precond* precond, int32_t which, int32_t* h_rowptr, int32_t* h_cols,
                                     void* h_values, int64_t capacity)
{
   clear_error();
   TNLB_REQUIRE(precond && h_rowptr && h_cols && h_values, TNLB_ERR_INVALID_ARGUMENT, "null argument");
   if (precond->ilu) {  // ILU(0) / ILUT: the factors as one CSR (L entries, then U from its pivot)
      TNLB_REQUIRE(which == 0, TNLB_ERR_INVALID_ARGUMENT, "an ILU preconditioner has one factor array (which = 0)");
      return tnlb::ilu0_read(precond->ilu, h_rowptr, h_cols, h_values, capacity, precond->real == TNLB_F64 ? 8 : 4);
   }
   TNLB_REQUIRE(precond->fsai != nullptr, TNLB_ERR_INVALID_ARGUMENT, "not an FSAI or ILU preconditioner");
   TNLB_REQUIRE(which == 0 || which == 1, TNLB_ERR_INVALID_ARGUMENT, "which must be 0 or 1");
   const Fsai* F = precond->fsai;
   const tnlb_segments* seg = which == 0 ? F->g : F->gt;
   const int64_t nnz = seg->elements;
   TNLB_REQUIRE(capacity >= nnz, TNLB_ERR_INVALID_ARGUMENT, "buffer too small");
   const size_t rs = F->real == TNLB_F64 ? 8 : 4;
   TNLB_CUDA_TRY(cudaMemcpy(h_rowptr, seg->offsets.ptr, sizeof(int32_t) * ((size_t)F->n + 1), cudaMemcpyDeviceToHost));
   TNLB_CUDA_TRY(cudaMemcpy(h_cols, (which == 0 ? F->g_cols : F->gt_cols).ptr, sizeof(int32_t) * nnz,
                            cudaMemcpyDeviceToHost));
   TNLB_CUDA_TRY(cudaMemcpy(h_values, (which == 0 ? F->g_vals : F->gt_vals).ptr, rs * nnz, cudaMemcpyDeviceToHost));
   return TNLB_OK;
}

tnlb_status tnlb_precond_destroy(tnlb_precond* precond)
{
   clear_error();
   delete precond;
   return TNLB_OK;
}

tnlb_status tnlb_ilu0_factors(const tnlb_segments* seg, tnlb_real real, const int32_t* d_cols, const void* d_values,
                              int32_t* h_rowptr, int32_t* h_cols, void* h_values, int64_t capacity,
                              tnlb_stream stream)
{
   clear_error();
   TNLB_REQUIRE(seg != nullptr && h_rowptr && h_cols && h_values, TNLB_ERR_INVALID_ARGUMENT, "null argument");
   void* ilu = nullptr;
   tnlb_status s = tnlb::ilu0_create(seg, real, d_cols, d_values, (cudaStream_t)stream, &ilu);
   if (s == TNLB_OK) s = tnlb::ilu0_read(ilu, h_rowptr, h_cols, h_values, capacity, real == TNLB_F64 ? 8 : 4);
   if (ilu) tnlb::ilu0_destroy(ilu);
   return s;
}

int64_t tnlb_lfsai_num_params(void) { return kLfParams; }

tnlb_status tnlb_lfsai_create(uint64_t seed, tnlb_stream stream, tnlb_lfsai** out)
{
   clear_error();
   TNLB_REQUIRE(out != nullptr, TNLB_ERR_INVALID_ARGUMENT, "null argument");
   auto* net = new (std::nothrow) tnlb_lfsai();
   TNLB_REQUIRE(net != nullptr, TNLB_ERR_OUT_OF_MEMORY, "out of host memory");
   tnlb_status s = lfsai_init(net, seed, (cudaStream_t)stream);
   if (s != TNLB_OK) {
      delete net;
      return s;
   }
   *out = net;
   return TNLB_OK;
}

tnlb_status tnlb_lfsai_destroy(tnlb_lfsai* net)
{
   clear_error();
   delete net;
   return TNLB_OK;
}

tnlb_status tnlb_lfsai_get_params(const tnlb_lfsai* net, float* h_out, int64_t count)
{
   clear_error();
   TNLB_REQUIRE(net && h_out && count >= kLfParams, TNLB_ERR_INVALID_ARGUMENT, "bad arguments");
   TNLB_CUDA_TRY(cudaMemcpy(h_out, net->theta.ptr, sizeof(float) * kLfParams, cudaMemcpyDeviceToHost));
   return TNLB_OK;
}

tnlb_status tnlb_lfsai_set_params(tnlb_lfsai* net, const float* h_in, int64_t count)
{
   clear_error();
   TNLB_REQUIRE(net && h_in && count >= kLfParams, TNLB_ERR_INVALID_ARGUMENT, "bad arguments");
   TNLB_CUDA_TRY(cudaMemcpy(net->theta.ptr, h_in, sizeof(float) * kLfParams, cudaMemcpyHostToDevice));
   TNLB_CUDA_TRY(cudaMemset(net->m.ptr, 0, sizeof(float) * kLfParams));
   TNLB_CUDA_TRY(cudaMemset(net->v.ptr, 0, sizeof(float) * kLfParams));
   net->step = 0;
   return TNLB_OK;
}

tnlb_status tnlb_lfsai_get_grad(const tnlb_lfsai* net, float* h_out, int64_t count)
{
   clear_error();
   TNLB_REQUIRE(net && h_out && count >= kLfParams, TNLB_ERR_INVALID_ARGUMENT, "bad arguments");
   TNLB_CUDA_TRY(cudaMemcpy(h_out, net->grad.ptr, sizeof(float) * kLfParams, cudaMemcpyDeviceToHost));
   return TNLB_OK;
}

tnlb_status tnlb_lfsai_set_tensor_cores(tnlb_lfsai* net, int32_t enable)
{
   clear_error();
   TNLB_REQUIRE(net != nullptr, TNLB_ERR_INVALID_ARGUMENT, "null network");
   net->use_tc = enable ? 1 : 0;
   return TNLB_OK;
}

tnlb_status tnlb_lfsai_set_level(tnlb_lfsai* net, int32_t level)
{
   clear_error();
   TNLB_REQUIRE(net != nullptr, TNLB_ERR_INVALID_ARGUMENT, "null network");
   TNLB_REQUIRE(level == 0 || level == 1, TNLB_ERR_INVALID_ARGUMENT, "the pattern level must be 0 or 1");
   net->level = level;
   return TNLB_OK;
}

tnlb_status tnlb_lfsai_set_two_factor(tnlb_lfsai* net, int32_t enable)
{
   clear_error();
   TNLB_REQUIRE(net != nullptr, TNLB_ERR_INVALID_ARGUMENT, "null network");
   net->two_factor = enable ? 1 : 0;
   return TNLB_OK;
}

tnlb_status tnlb_lfsai_gradient(tnlb_lfsai* net, int32_t mode, const tnlb_segments* seg, tnlb_real real,
                                const int32_t* d_cols, const void* d_values, const void* d_probes, int32_t nprobes,
                                tnlb_stream stream, double* h_loss)
{
   clear_error();
   TNLB_REQUIRE(net && seg && h_loss, TNLB_ERR_INVALID_ARGUMENT, "null argument");
   TNLB_REQUIRE(mode >= 0 && mode <= 2, TNLB_ERR_INVALID_ARGUMENT,
                "mode must be 0 (probe loss), 1 (warm start) or 2 (Kaporin loss)");
   TNLB_REQUIRE(mode != 0 || (d_probes && nprobes > 0), TNLB_ERR_INVALID_ARGUMENT, "probe vectors required");
   TNLB_REQUIRE(seg->n > 0, TNLB_ERR_INVALID_ARGUMENT, "the matrix is empty");
   return lfsai_gradient(net, seg, real, d_cols, d_values, d_probes, nprobes, mode, (cudaStream_t)stream, h_loss);
}

tnlb_status tnlb_lfsai_adam_step(tnlb_lfsai* net, double lr, tnlb_stream stream)
{
   clear_error();
   TNLB_REQUIRE(net != nullptr, TNLB_ERR_INVALID_ARGUMENT, "null network");
   return lfsai_adam(net, lr, (cudaStream_t)stream);
}

tnlb_status tnlb_lfsai_precond_create(const tnlb_lfsai* net, const tnlb_segments* seg, tnlb_real real,
                                      const int32_t* d_cols, const void* d_values, tnlb_stream stream,
                                      tnlb_precond** out)
{
   clear_error();
   TNLB_REQUIRE(net && seg && out, TNLB_ERR_INVALID_ARGUMENT, "null argument");
   TNLB_REQUIRE(seg->n > 0, TNLB_ERR_INVALID_ARGUMENT, "the matrix is empty");
   *out = nullptr;
   return lfsai_precond(net, seg, real, d_cols, d_values, (cudaStream_t)stream, out);
}

tnlb_status tnlb_lfsai_eval(const tnlb_lfsai* net, const tnlb_segments* seg, tnlb_real real, const int32_t* d_cols,
                            const void* d_values, tnlb_stream stream, float* h_features, float* h_outputs)
{
   clear_error();
   TNLB_REQUIRE(net && seg, TNLB_ERR_INVALID_ARGUMENT, "null argument");
   TNLB_REQUIRE(seg->n > 0, TNLB_ERR_INVALID_ARGUMENT, "the matrix is empty");
   return lfsai_eval(net, seg, real, d_cols, d_values, (cudaStream_t)stream, h_features, h_outputs);
}

}  // extern "C"
