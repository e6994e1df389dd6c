// internal.cuh -- shared definitions of libtnlb200 (not part of the public ABI).
#pragma once

#include <vector>

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <string>

#include "../../include/tnlb200.h"

namespace tnlb {

// ----------------------------------------------------------------- errors

void set_error(const std::string& msg);
void clear_error();

#define TNLB_CUDA_TRY(expr)                                                                                    \
   do {                                                                                                        \
      cudaError_t _e = (expr);                                                                                 \
      if (_e != cudaSuccess) {                                                                                 \
         ::tnlb::set_error(std::string(#expr) + ": " + cudaGetErrorString(_e) + " (" + __FILE__ + ":" +        \
                           std::to_string(__LINE__) + ")");                                                    \
         return _e == cudaErrorMemoryAllocation ? TNLB_ERR_OUT_OF_MEMORY : TNLB_ERR_CUDA;                      \
      }                                                                                                        \
   } while (0)

#define TNLB_CHECK_LAUNCH() TNLB_CUDA_TRY(cudaGetLastError())

#define TNLB_REQUIRE(cond, code, msg)                                                                          \
   do {                                                                                                        \
      if (!(cond)) {                                                                                           \
         ::tnlb::set_error(msg);                                                                               \
         return code;                                                                                          \
      }                                                                                                        \
   } while (0)

#define TNLB_TRY_STATUS(...)                                                                                   \
   do {                                                                                                        \
      tnlb_status _s = (__VA_ARGS__);                                                                          \
      if (_s != TNLB_OK) return _s;                                                                            \
   } while (0)

// ------------------------------------------------------------- constants

constexpr int kWarp = 32;
constexpr int kSellSlice = 32;       // SlicedEllpack SliceSize (SlicedEllpack.h:46)
constexpr int kEllAlignment = 32;    // Ellpack Alignment (Ellpack.h:40)
constexpr int kBiStrip = 32;         // BiEllpack WarpSize
constexpr int kBiGroups = 6;         // log2(32) + 1
constexpr int kChunksInSlice = 256;  // ChunkedEllpackBase.h:291
constexpr int kDesiredChunkSize = 16;  // ChunkedEllpackBase.h:292

// CSR tile kernel geometry: a tile of kTileSize merge items (rows +
// nonzeros) per warp, kTileItems per lane; blocks of kTileThreads threads.
constexpr int kTileThreads = 128;
constexpr int kTileItems = 8;
constexpr int kTileSize = 32 * kTileItems;

// ------------------------------------------------------- device buffers

// Owned device allocation (cudaMalloc / cudaFree).
struct DeviceBuffer {
   void* ptr = nullptr;
   size_t bytes = 0;
   DeviceBuffer() = default;
   DeviceBuffer(const DeviceBuffer&) = delete;
   DeviceBuffer& operator=(const DeviceBuffer&) = delete;
   ~DeviceBuffer() { release(); }
   void release()
   {
      if (ptr) cudaFree(ptr);
      ptr = nullptr;
      bytes = 0;
   }
   tnlb_status alloc(size_t nbytes)
   {
      release();
      if (nbytes == 0) nbytes = 16;
      cudaError_t e = cudaMalloc(&ptr, nbytes);
      if (e != cudaSuccess) {
         ptr = nullptr;
         set_error(std::string("cudaMalloc(") + std::to_string(nbytes) + "): " + cudaGetErrorString(e));
         return TNLB_ERR_OUT_OF_MEMORY;
      }
      bytes = nbytes;
      return TNLB_OK;
   }
   template <typename T>
   T* as() const
   {
      return static_cast<T*>(ptr);
   }
};

}  // namespace tnlb

// ------------------------------------------------------------ segments
// The opaque handle of the C ABI.
struct tnlb_segments {
   int32_t format = TNLB_CSR;
   int32_t organization = TNLB_COLUMN_MAJOR;
   int32_t n = 0;           // segments
   int64_t elements = 0;    // sum of sizes
   int64_t storage = 0;     // slots
   int32_t max_size = 0;    // largest segment size
   int device = 0;

   // CSR / AdaptiveCSR
   tnlb::DeviceBuffer offsets;  // int32[n+1]
   // CSR tile plan: merge-path coordinates of tile boundaries
   int32_t tiles = 0;
   int32_t max_row = -1;  // longest row (CSR), -1 if unknown
   tnlb::DeviceBuffer tile_row;    // int32[tiles+1]
   tnlb::DeviceBuffer tile_nnz;    // int32[tiles+1]
   tnlb::DeviceBuffer carry_row;   // int32[tiles]   (scratch, per call)
   tnlb::DeviceBuffer carry_val;   // double[tiles]  (scratch, per call)
   // AdaptiveCSR descriptors per value-size log
   int64_t acsr_count[6] = {0, 0, 0, 0, 0, 0};
   tnlb::DeviceBuffer acsr_blocks[6];  // tnlb_acsr_block[count]

   // Ellpack
   int32_t segment_size = 0;
   int32_t aligned_size = 0;

   // SlicedEllpack
   int32_t slices = 0;
   tnlb::DeviceBuffer slice_offsets;        // int32[slices+1]
   tnlb::DeviceBuffer slice_segment_sizes;  // int32[slices]
   tnlb::DeviceBuffer slice_order;          // int32[slices]: slices by width, widest first

   // ChunkedEllpack
   int32_t ch_slices = 0;
   tnlb::DeviceBuffer ch_slice_size, ch_slice_chunk_size, ch_slice_first, ch_slice_pointer;  // int32[ch_slices]
   tnlb::DeviceBuffer ch_segment_to_chunk, ch_segment_to_slice;                             // int32[n]
   tnlb::DeviceBuffer ch_segment_pointers;                                                  // int32[n+1]
   tnlb::DeviceBuffer ch_chunks_to_segments;                                                // int32[ch_slices*256]

   // BiEllpack
   int32_t strips = 0;
   tnlb::DeviceBuffer bi_perm;            // int32[n]
   tnlb::DeviceBuffer bi_group_pointers;  // int32[strips*6+1]
};

namespace tnlb {
struct Fsai;
}

// A preconditioner built for one matrix (Preconditioner::update), applied
// by the solvers (Preconditioner::solve).  Opaque in the C ABI.
struct tnlb_precond {
   int32_t kind = TNLB_PRECOND_NONE;
   tnlb_real real = TNLB_F64;
   int32_t n = 0;
   tnlb::DeviceBuffer diag;      // Jacobi
   void* ilu = nullptr;          // ILU(0)
   tnlb::Fsai* fsai = nullptr;   // FSAI / learned FSAI: M^-1 = G^T G
   ~tnlb_precond();
};

namespace tnlb {

// ------------------------------------------------- device-side helpers

// Streaming (read-once) global loads: non-coherent path, no L1 allocation.
__device__ __forceinline__ double ld_stream(const double* p)
{
   double v;
   asm("ld.global.nc.L1::no_allocate.f64 %0, [%1];" : "=d"(v) : "l"(p));
   return v;
}
__device__ __forceinline__ float ld_stream(const float* p)
{
   float v;
   asm("ld.global.nc.L1::no_allocate.f32 %0, [%1];" : "=f"(v) : "l"(p));
   return v;
}
__device__ __forceinline__ int32_t ld_stream(const int32_t* p)
{
   int32_t v;
   asm("ld.global.nc.L1::no_allocate.s32 %0, [%1];" : "=r"(v) : "l"(p));
   return v;
}
// 128-bit streaming loads (address must be 16-byte aligned).
__device__ __forceinline__ double2 ld_stream_v2(const double* p)
{
   double2 v;
   asm("ld.global.nc.L1::no_allocate.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "l"(p));
   return v;
}
__device__ __forceinline__ float4 ld_stream_v4(const float* p)
{
   float4 v;
   asm("ld.global.nc.L1::no_allocate.v4.f32 {%0, %1, %2, %3}, [%4];"
                : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
                : "l"(p));
   return v;
}
__device__ __forceinline__ int4 ld_stream_v4(const int32_t* p)
{
   int4 v;
   asm("ld.global.nc.L1::no_allocate.v4.s32 {%0, %1, %2, %3}, [%4];"
                : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                : "l"(p));
   return v;
}

// Gathered x loads go through the read-only path and may stay cached.
template <typename T>
__device__ __forceinline__ T ld_gather(const T* p)
{
   return __ldg(p);
}

__host__ __device__ __forceinline__ int64_t imin64(int64_t a, int64_t b) { return a < b ? a : b; }
__host__ __device__ __forceinline__ int64_t imax64(int64_t a, int64_t b) { return a > b ? a : b; }

template <typename T>
__device__ __forceinline__ T warp_sum(T v)
{
#pragma unroll
   for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
   return v;
}

// Sum within aligned groups of `G` lanes (G power of two <= 32).
template <int G, typename T>
__device__ __forceinline__ T group_sum(T v)
{
#pragma unroll
   for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
   return v;
}

// The four keep variants of vectorProduct (SparseMatrixBase.hpp:346-392).
template <typename Real>
__device__ __forceinline__ void keep(Real* y, int32_t row, Real value, Real alpha, Real beta)
{
   if (beta == Real(0)) {
      y[row] = (alpha == Real(1)) ? value : alpha * value;
   }
   else {
      y[row] = (alpha == Real(1)) ? beta * y[row] + value : beta * y[row] + alpha * value;
   }
}

inline unsigned grid_for(int64_t work, int per_block)
{
   int64_t g = (work + per_block - 1) / per_block;
   if (g < 1) g = 1;
   if (g > 0x7fffffff) g = 0x7fffffff;
   return (unsigned)g;
}

// -------------------------------------------------- internal interfaces

// builders.cu
tnlb_status build_segments(tnlb_segments* seg, const int32_t* d_sizes, cudaStream_t stream);
// scan.cu
tnlb_status exclusive_scan_i32(const int32_t* d_in, int32_t* d_out, int64_t n, int64_t* h_total, cudaStream_t stream,
                               bool append_total);
tnlb_status inclusive_scan_i32_inplace(int32_t* d_data, int64_t n, cudaStream_t stream);
tnlb_status reduce_max_i32(const int32_t* d_in, int64_t n, int32_t* h_max, cudaStream_t stream);
tnlb_status reduce_sum_i64(const int32_t* d_in, int64_t n, int64_t* h_sum, cudaStream_t stream);
// spmv_csr.cu / spmv_ell.cu
// y = A x with (x, y) summed in the same kernel, for CSR matrices whose rows
// hold at most 16 entries (spmv_dot_fusable); `partials` holds
// spmv_dot_partials(seg) doubles, `counter` starts (and ends) at zero; the
// sum lands in *dot_out (with `self_dot`: (y, y)).  Deterministic.
bool spmv_dot_fusable(const tnlb_segments* seg);
int64_t spmv_dot_partials(const tnlb_segments* seg);
tnlb_status spmv_dot(const tnlb_segments* seg, tnlb_real real, const int32_t* cols, const void* vals, const void* x,
                     void* y, double* partials, unsigned* counter, double* dot_out, cudaStream_t st,
                     const int32_t* skip, bool self_dot = false);
// The same with values, input and output of different real types: FP32
// values with FP64 vectors (F32, F64, F64), or with an FP64 input and an
// FP32 output (F32, F64, F32); rows are summed in the input's type.
tnlb_status spmv_dot_mixed(const tnlb_segments* seg, tnlb_real tv, tnlb_real tx, tnlb_real ty, const int32_t* cols,
                           const void* vals, const void* x, void* y, double* partials, unsigned* counter,
                           double* dot_out, cudaStream_t st, const int32_t* skip, bool self_dot);
// y = A x + (*num / *den) y for the same short-row CSR matrices (types: all
// equal, or FP32 values and input with an FP64 output).
tnlb_status spmv_xpby_mixed(const tnlb_segments* seg, tnlb_real tv, tnlb_real tx, tnlb_real ty, const int32_t* cols,
                            const void* vals, const void* x, void* y, const double* num, const double* den,
                            cudaStream_t st, const int32_t* skip);
// Compact copy of a short-row CSR matrix with FP32 or FP16 values, for the
// FP32 iterations of the reliable-update PCG (compact.cu), in one of two
// layouts:
//   kRel: CSR with 16-bit column offsets (column - row); rowptr is the
//         source segments' own; width = the longest row;
//   kDia: diagonals -- the matrix has `width` <= 8 distinct column - row
//         offsets (diag[], ascending), each row's columns ascending; the
//         value of row i on diagonal j at vals[j * pitch + i], 0 where the
//         row has no such entry; the products' vectors 16-byte aligned.
struct CompactCopy {
   enum Kind { kNone = 0, kRel = 1, kDia = 2 };
   Kind kind = kNone;
   int32_t n = 0, width = 0;
   bool half = false;
   const int32_t* rowptr = nullptr;
   int32_t diag[8] = {};
   int64_t pitch = 0;  // kDia: values of diagonal j at vals[j * pitch ...], pitch a multiple of 8
   // row-excess form (compact.cuh): kDia the slot of offset 0, kRel 0; -1
   // when the diagonal entries hold a_ii
   int32_t self_slot = -1;
   DeviceBuffer off, vals;
};
inline bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }
// Builds the copy (kind kNone when the matrix is not short-row CSR or a
// column lies 32768 or more from its row): kDia when allowed and the
// diagonals hold at least 3/4 of their slots, else kRel.  FP16 values
// (`half`) are stored times `scale`.  With `vals64` (the FP64 values of the
// same entries, FP32 copies only) the copy takes the row-excess form when
// every row holds its diagonal entry: that entry stores the row's FP64 sum
// rounded to FP32.
tnlb_status compact_build(const tnlb_segments* seg, const int32_t* cols, const float* vals, bool half, float scale,
                          bool allow_dia, cudaStream_t st, CompactCopy* out, const double* vals64 = nullptr);
// The power of two that brings the largest |vals| into [2^13, 2^14): FP16
// copies times it neither overflow nor lose normal-range precision (1 for
// an all-zero array).
tnlb_status half_scale(const float* vals, int64_t nnz, cudaStream_t st, float* scale);
// y = A x and (x, y) -- (y, y) with self_dot -- into *dot_out.
tnlb_status compact_spmv_dot(const CompactCopy& A, const float* x, float* y, double* partials, unsigned* counter,
                             double* dot_out, cudaStream_t st, const int32_t* skip, bool self_dot);
// A diagonal copy the bulk-copy-staged kernels take (band.cuh): at most 8
// diagonals, offset 0 among them.
bool compact_band_capable(const CompactCopy& A);
// y = A x + (*num / *den) y.
tnlb_status compact_spmv_xpby(const CompactCopy& A, const float* x, float* y, const double* num, const double* den,
                              cudaStream_t st, const int32_t* skip);
tnlb_status spmv_xpby(const tnlb_segments* seg, tnlb_real real, const int32_t* cols, const void* vals, const void* x,
                      void* y, const double* num, const double* den, cudaStream_t st, const int32_t* skip);
tnlb_status spmv_csr(const tnlb_segments* seg, tnlb_real real, const int32_t* cols, const void* vals, const void* x,
                     void* y, double alpha, double beta, int32_t begin, int32_t end, tnlb_kernel kernel, int32_t tps,
                     cudaStream_t stream, int* launches, const int32_t* skip = nullptr);
tnlb_status spmv_ell_family(const tnlb_segments* seg, tnlb_real real, const int32_t* cols, const void* vals,
                            const void* x, void* y, double alpha, double beta, int32_t begin, int32_t end,
                            tnlb_kernel kernel, int32_t tps, cudaStream_t stream, int* launches);
tnlb_status build_csr_tile_plan(tnlb_segments* seg, cudaStream_t stream);
// solvers.cu / ilu0.cu / fsai.cu
tnlb_status precond_create(int kind, const tnlb_segments* seg, tnlb_real real, const int32_t* cols, const void* vals,
                           cudaStream_t st, tnlb_precond** out);
tnlb_status precond_apply(const tnlb_precond* P, const void* b, void* x, cudaStream_t st);
tnlb_status solve(tnlb_solver_kind solver, const tnlb_precond* P, const tnlb_solver_params& prm,
                  const tnlb_segments* seg, tnlb_real real, const int32_t* cols, const void* vals, const void* b,
                  void* x, cudaStream_t st, tnlb_solve_result* res);
tnlb_status true_residual(const tnlb_segments* seg, tnlb_real real, const int32_t* cols, const void* vals,
                          const void* b, const void* x, cudaStream_t st, double* out);
tnlb_status solve_mixed_cg(const tnlb_segments* seg, const int32_t* cols, const double* vals, const double* b,
                           double* x, const tnlb_solver_params& prm, double inner_tol, int32_t max_outer,
                           cudaStream_t st, tnlb_solve_result* res, int32_t* inner_total, int32_t* outer,
                           int inner_kind, const tnlb_precond* inner_precond, int inner_solver);
tnlb_status solve_mixed_reliable(const tnlb_segments* seg, const int32_t* cols, const double* vals, const double* b,
                                 double* x, const tnlb_solver_params& prm, double delta, tnlb_real vectors,
                                 cudaStream_t st, tnlb_solve_result* res, int32_t* updates, int inner_kind,
                                 const tnlb_precond* inner_precond);
tnlb_status ilu0_create(const tnlb_segments* seg, tnlb_real real, const int32_t* cols, const void* vals,
                        cudaStream_t st, void** out);
tnlb_status ilu0_apply(void* ilu, const void* b, void* x, cudaStream_t st);
// An ILU object over factors computed elsewhere (ILUT): host CSR whose row i
// holds its L entries (columns < i) then its U entries (first = pivot).
tnlb_status ilu_from_factors(tnlb_real real, int32_t n, const std::vector<int32_t>& rp,
                             const std::vector<int32_t>& cols, const void* lu, cudaStream_t st, void** out);
tnlb_status ilut_create(const tnlb_segments* seg, tnlb_real real, const int32_t* cols, const void* vals, int32_t p,
                        double tau, cudaStream_t st, void** out);
tnlb_status ilu0_read(void* ilu, int32_t* h_rowptr, int32_t* h_cols, void* h_vals, int64_t capacity, int real_bytes);
void ilu0_destroy(void* ilu);
tnlb_status fsai_create(const tnlb_segments* seg, tnlb_real real, const int32_t* cols, const void* vals,
                        bool classical, cudaStream_t st, Fsai** out, bool two_factor = false, int level = 0);
tnlb_status fsai_apply(const Fsai* F, const void* r, void* z, cudaStream_t st, const int32_t* skip = nullptr);
tnlb_status fsai_set_values2(Fsai* F, const void* glvals, const void* hvals, cudaStream_t st);
// z = G^T (G r) with (r, z) = |G r|^2 summed inside the G product (symmetric
// FSAI whose G has rows of at most 16 entries: fsai_dot_fusable).
bool fsai_dot_fusable(const Fsai* F);
// The parts of an FSAI preconditioner: G and G^T (segments, columns,
// values of the preconditioner's real type) and its work vector t.
struct FsaiView {
   const tnlb_segments *g = nullptr, *gt = nullptr;
   const int32_t *gcols = nullptr, *gtcols = nullptr;
   const void *gvals = nullptr, *gtvals = nullptr;
   void* tmp = nullptr;
};
FsaiView fsai_view(const Fsai* F);
bool fsai_two_factor(const Fsai* F);
tnlb_status fsai_apply_dot(const Fsai* F, const void* r, void* z, double* partials, unsigned* counter, double* rz_out,
                           cudaStream_t st, const int32_t* skip);
// t = G r with (t, t) into *rz_out, then p = G^T t + (*rz_out / *rz_old) p
// (the preconditioner application and direction update of FSAI-PCG).
// r and p of type `vec` (the factors' own type, or FP64 with FP32 factors).
tnlb_status fsai_apply_dot_xpby(const Fsai* F, tnlb_real vec, const void* r, void* p, double* partials,
                                unsigned* counter, double* rz_out, const double* rz_old, cudaStream_t st,
                                const int32_t* skip);
tnlb_status fsai_set_values(Fsai* F, const void* gvals, cudaStream_t st);
void fsai_destroy(Fsai* F);
tnlb_status spmv_dispatch(const tnlb_segments* seg, tnlb_real real, const int32_t* cols, const void* vals,
                          const void* x, void* y, double alpha, double beta, cudaStream_t st,
                          const int32_t* skip = nullptr);
// fill.cu
tnlb_status fill_from_csr(const tnlb_segments* seg, tnlb_real real, const int32_t* rowptr, const int32_t* src_cols,
                          const void* src_vals, int32_t* cols, void* vals, cudaStream_t stream);
tnlb_status global_index(const tnlb_segments* seg, const int32_t* segs, const int32_t* locals, int64_t count,
                         int64_t* out, cudaStream_t stream);

}  // namespace tnlb
