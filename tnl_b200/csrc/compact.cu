// compact.cu -- compact copies of short-row CSR matrices for the FP32
// iterations of the reliable-update PCG (solvers.cu), with FP32 or FP16
// values.  The solver builds them from its own FP32 copies; the caller's
// matrix and the public formats are untouched.  Two layouts (compact.cuh):
//
//   diagonals (kDia)  a matrix with at most 8 distinct column - row offsets
//                     that fill at least 3/4 of their diagonals (stencils
//                     and their FSAI factors): per row only the D values
//                     are read -- 4 bytes an entry in FP32, 2 in FP16, no
//                     column data and no row offsets -- and every load of a
//                     warp is one contiguous run;
//   16-bit offsets (kRel)  CSR whose columns lie within 32767 of their row:
//                     6 bytes an entry (FP32 value + offset) or 4 (FP16),
//                     plus the row offsets, against 8 in the FP32 CSR.
//
// Rows are summed in FP32 in ascending column order, as the CSR short-row
// kernels do; both layouts give the same row sums bit for bit (see
// compact.cuh).  FP16 copies are stored times a power of two (half_scale)
// that keeps their largest entry below 2^14.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <vector>

#include "band.cuh"
#include "compact.cuh"
#include "internal.cuh"
#include "reduce.cuh"

namespace tnlb {

namespace {

constexpr int32_t kNoDiag = INT_MIN;  // an empty slot of a diagonal table
constexpr int kDiagSlots = 16;        // slots of a table (at most 8 are used)

// offsets[k] = cols[k] - row(k); *bad = 1 if one does not fit in int16
__global__ void k_rel_offsets(const int32_t* __restrict__ rowptr, const int32_t* __restrict__ cols, int32_t n,
                              int16_t* __restrict__ off, int32_t* __restrict__ bad)
{
   const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (r >= n) return;
   for (int32_t k = rowptr[r]; k < rowptr[r + 1]; k++) {
      const int64_t d = (int64_t)cols[k] - r;
      if (cols[k] < 0 || d < -32768 || d > 32767) {
         *bad = 1;
         off[k] = 0;
      }
      else
         off[k] = (int16_t)d;
   }
}

__global__ void k_to_half(const float* __restrict__ a, int64_t n, float scale, __half* __restrict__ b)
{
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
      b[i] = __float2half_rn(a[i] * scale);
}

// *out = max |a| as the bits of a non-negative float (their integer order
// is the float order); NaN entries are skipped.
__global__ void k_absmax(const float* __restrict__ a, int64_t n, unsigned* __restrict__ out)
{
   unsigned m = 0u;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
      const float v = fabsf(a[i]);
      if (v == v) m = max(m, __float_as_uint(v));
   }
   for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
   if ((threadIdx.x & 31) == 0 && m) atomicMax(out, m);
}

__global__ void k_diag_table_init(int32_t* __restrict__ tab, int32_t* __restrict__ flag)
{
   if (threadIdx.x < kDiagSlots) tab[threadIdx.x] = kNoDiag;
   if (threadIdx.x == 0) *flag = 0;
}

// d into the table (shared or global) unless present; false when full.
__device__ bool diag_insert(int32_t* tab, int32_t d)
{
   for (int s = 0; s < kDiagSlots; s++) {
      int32_t cur = *reinterpret_cast<volatile int32_t*>(tab + s);
      if (cur == d) return true;
      if (cur == kNoDiag) {
         cur = atomicCAS(tab + s, kNoDiag, d);
         if (cur == kNoDiag || cur == d) return true;
      }
   }
   return false;
}

// The distinct column - row offsets into `tab`; *flag = 1 when a row's
// columns are not strictly ascending within [0, n) or there are more than
// the table holds.  Each block gathers its own offsets in shared memory.
__global__ void __launch_bounds__(256) k_diag_scan(const int32_t* __restrict__ rowptr,
                                                   const int32_t* __restrict__ cols, int32_t n,
                                                   int32_t* __restrict__ tab, int32_t* __restrict__ flag)
{
   __shared__ int32_t local[kDiagSlots];
   __shared__ int bad;
   if (threadIdx.x < kDiagSlots) local[threadIdx.x] = kNoDiag;
   if (threadIdx.x == 0) bad = 0;
   __syncthreads();
   const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (r < n) {
      int32_t prev = -1;
      for (int32_t k = rowptr[r]; k < rowptr[r + 1]; k++) {
         const int32_t c = cols[k];
         if (c <= prev || c >= n || !diag_insert(local, c - (int32_t)r)) {
            bad = 1;
            break;
         }
         prev = c;
      }
   }
   __syncthreads();
   if (threadIdx.x == 0 && bad) *flag = 1;
   if (threadIdx.x < kDiagSlots && local[threadIdx.x] != kNoDiag && !diag_insert(tab, local[threadIdx.x])) *flag = 1;
}

// vals[j * pitch + r] = value of row r on diagonal j (the buffer zeroed
// before).
template <typename TV>
__global__ void k_diag_fill(const int32_t* __restrict__ rowptr, const int32_t* __restrict__ cols,
                            const float* __restrict__ v, int32_t n, DiaOffsets d, int32_t nd, int64_t pitch,
                            float scale, TV* __restrict__ out)
{
   const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (r >= n) return;
   for (int32_t k = rowptr[r]; k < rowptr[r + 1]; k++) {
      const int32_t o = cols[k] - (int32_t)r;
      int32_t j = 0;
      while (j < nd - 1 && d.o[j] != o) j++;
      out[(int64_t)j * pitch + r] = (TV)(v[k] * scale);
   }
}

// s[r] = the FP64 sum of row r's values in entry order, rounded to FP32
// (the row excess a_rr + sum_{c != r} a_rc); *bad = 1 when a row holds no
// diagonal entry.
__global__ void k_row_excess(const int32_t* __restrict__ rowptr, const int32_t* __restrict__ cols,
                             const double* __restrict__ v, int32_t n, float* __restrict__ s,
                             int32_t* __restrict__ bad)
{
   const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (r >= n) return;
   double t = 0.0;
   bool diag = false;
   for (int32_t k = rowptr[r]; k < rowptr[r + 1]; k++) {
      t += v[k];
      diag |= cols[k] == (int32_t)r;
   }
   s[r] = (float)t;
   if (!diag) *bad = 1;
}

// The diagonal entries of a CSR copy (FP32 values) replaced by s.
__global__ void k_set_diagonal_csr(const int32_t* __restrict__ rowptr, const int32_t* __restrict__ cols,
                                   const float* __restrict__ s, int32_t n, float* __restrict__ vals)
{
   const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (r >= n) return;
   for (int32_t k = rowptr[r]; k < rowptr[r + 1]; k++)
      if (cols[k] == (int32_t)r) vals[k] = s[r];
}

// The row excesses of an FP64 CSR matrix into `s` (n floats); *ok false
// when a row has no diagonal entry.
tnlb_status row_excess(const int32_t* rowptr, const int32_t* cols, const double* v, int32_t n, cudaStream_t st,
                       DeviceBuffer* s, bool* ok)
{
   DeviceBuffer bad;
   TNLB_TRY_STATUS(bad.alloc(sizeof(int32_t)));
   TNLB_TRY_STATUS(s->alloc(sizeof(float) * (n > 0 ? n : 1)));
   TNLB_CUDA_TRY(cudaMemsetAsync(bad.ptr, 0, sizeof(int32_t), st));
   k_row_excess<<<grid_for(n, 256), 256, 0, st>>>(rowptr, cols, v, n, s->as<float>(), bad.as<int32_t>());
   TNLB_CHECK_LAUNCH();
   int32_t h = 0;
   TNLB_CUDA_TRY(cudaMemcpyAsync(&h, bad.ptr, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
   TNLB_CUDA_TRY(cudaStreamSynchronize(st));
   *ok = h == 0;
   return TNLB_OK;
}

// y = A x and (x, y) -- or (y, y) with `self` -- as k_csr_short_dot does.
// Four-row policies (kQuad) store and read the rows' own entries as
// vectors when all four rows exist (the vectors are 16-byte aligned).
template <typename Rows>
__global__ void __launch_bounds__(256, Rows::kMinBlocks) k_cmp_dot(Rows A, const float* __restrict__ x, float* __restrict__ y, int32_t n,
                                                 RedWork w, double* __restrict__ dot_out,
                                                 const int32_t* __restrict__ skip, int self)
{
   if (skip && *skip) return;
   const PlainInput xv{x};
   double d = 0.0;
#pragma unroll 1
   for (int64_t base = A.first(); base < n; base += A.step()) {
      A.prefetch(base + A.step(), n);
      float s[Rows::kR];
      A.rows(base, n, xv, s);
      if constexpr (Rows::kQuad) {
         if (base + 3 < n) {
            *reinterpret_cast<float4*>(y + base) = make_float4(s[0], s[1], s[2], s[3]);
            float o[4] = {0.0f, 0.0f, 0.0f, 0.0f};
            if (!self) xv.quad((int32_t)base, o);
#pragma unroll
            for (int k = 0; k < 4; k++) d += (double)s[k] * (self ? (double)s[k] : (double)o[k]);
            continue;
         }
      }
#pragma unroll
      for (int k = 0; k < Rows::kR; k++) {
         const int64_t i = A.row(base, k);
         if (i < n) {
            y[i] = s[k];
            d += (double)s[k] * (self ? (double)s[k] : (double)__ldg(x + i));
         }
      }
   }
   double vv[1] = {d};
   if (publish_and_arrive<1>(vv, w)) {
      double t[1];
      gather_totals<1>(t, w);
      if (threadIdx.x == 0) *dot_out = t[0];
   }
}

// y = A x + (num / den) y, as k_csr_short_xpby does.
template <typename Rows>
__global__ void __launch_bounds__(256, Rows::kMinBlocks) k_cmp_xpby(Rows A, const float* __restrict__ x, float* __restrict__ y,
                                                  int32_t n, const double* __restrict__ num,
                                                  const double* __restrict__ den, const int32_t* __restrict__ skip)
{
   if (skip && *skip) return;
   const float beta = (float)(*num / *den);
   const PlainInput xv{x};
#pragma unroll 1
   for (int64_t base = A.first(); base < n; base += A.step()) {
      A.prefetch(base + A.step(), n);
      float s[Rows::kR];
      A.rows(base, n, xv, s);
      if constexpr (Rows::kQuad) {
         if (base + 3 < n) {
            float4* yp = reinterpret_cast<float4*>(y + base);
            const float4 yo = *yp;
            *yp = make_float4(s[0] + beta * yo.x, s[1] + beta * yo.y, s[2] + beta * yo.z, s[3] + beta * yo.w);
            continue;
         }
      }
#pragma unroll
      for (int k = 0; k < Rows::kR; k++) {
         const int64_t i = A.row(base, k);
         if (i < n) y[i] = s[k] + beta * y[i];
      }
   }
}

template <typename Rows>
void launch_cmp_dot(const Rows& rows, int32_t n, const float* x, float* y, RedWork w, double* dot_out,
                    cudaStream_t st, const int32_t* skip, int self)
{
   auto* k = k_cmp_dot<Rows>;
   const unsigned g = resident_grid((const void*)k, 256, n, Rows::kR);
   k<<<g, 256, 0, st>>>(rows, x, y, n, w, dot_out, skip, self);
}

template <typename Rows>
void launch_cmp_xpby(const Rows& rows, int32_t n, const float* x, float* y, const double* num, const double* den,
                     cudaStream_t st, const int32_t* skip)
{
   auto* k = k_cmp_xpby<Rows>;
   const unsigned g = resident_grid((const void*)k, 256, n, Rows::kR);
   k<<<g, 256, 0, st>>>(rows, x, y, n, num, den, skip);
}

// The diagonal layout, when the matrix has one: *ok false otherwise.
tnlb_status diag_build(const tnlb_segments* seg, const int32_t* cols, const float* vals, bool half, float scale,
                       const float* excess, cudaStream_t st, CompactCopy* out, bool* ok)
{
   *ok = false;
   const int32_t n = seg->n;
   const int64_t nnz = seg->elements;
   if (n <= 0 || nnz <= 0) return TNLB_OK;
   const int32_t* rp = seg->offsets.as<int32_t>();
   DeviceBuffer tab;
   TNLB_TRY_STATUS(tab.alloc(sizeof(int32_t) * (kDiagSlots + 1)));
   int32_t* flag = tab.as<int32_t>() + kDiagSlots;
   k_diag_table_init<<<1, 32, 0, st>>>(tab.as<int32_t>(), flag);
   TNLB_CHECK_LAUNCH();
   k_diag_scan<<<grid_for(n, 256), 256, 0, st>>>(rp, cols, n, tab.as<int32_t>(), flag);
   TNLB_CHECK_LAUNCH();
   int32_t h[kDiagSlots + 1];
   TNLB_CUDA_TRY(cudaMemcpyAsync(h, tab.ptr, sizeof(h), cudaMemcpyDeviceToHost, st));
   TNLB_CUDA_TRY(cudaStreamSynchronize(st));
   if (h[kDiagSlots]) return TNLB_OK;
   std::vector<int32_t> d;
   for (int s = 0; s < kDiagSlots; s++)
      if (h[s] != kNoDiag) d.push_back(h[s]);
   // at most 8 diagonals, holding at least 3/4 of their slots
   if (d.empty() || d.size() > 8 || 4 * nnz < 3 * (int64_t)d.size() * n) return TNLB_OK;
   std::sort(d.begin(), d.end());
   DiaOffsets dd{};
   for (size_t j = 0; j < d.size(); j++) dd.o[j] = d[j];
   // four-row vector loads stay aligned, and so do bulk copies of 8 FP16
   // values
   const int64_t pitch = ((int64_t)n + 7) / 8 * 8;
   const size_t elem = half ? sizeof(__half) : sizeof(float);
   const size_t bytes = elem * d.size() * (size_t)pitch;
   TNLB_TRY_STATUS(out->vals.alloc(bytes));
   TNLB_CUDA_TRY(cudaMemsetAsync(out->vals.ptr, 0, bytes, st));
   if (half)
      k_diag_fill<__half><<<grid_for(n, 256), 256, 0, st>>>(rp, cols, vals, n, dd, (int32_t)d.size(), pitch,
                                                             scale, out->vals.as<__half>());
   else
      k_diag_fill<float><<<grid_for(n, 256), 256, 0, st>>>(rp, cols, vals, n, dd, (int32_t)d.size(), pitch,
                                                            1.0f, out->vals.as<float>());
   TNLB_CHECK_LAUNCH();
   out->self_slot = -1;
   if (excess && !half) {
      const auto z = std::find(d.begin(), d.end(), 0);
      if (z != d.end()) {
         const int64_t j0 = z - d.begin();
         TNLB_CUDA_TRY(cudaMemcpyAsync(out->vals.as<float>() + j0 * pitch, excess, sizeof(float) * n,
                                       cudaMemcpyDeviceToDevice, st));
         out->self_slot = (int32_t)j0;
      }
   }
   out->kind = CompactCopy::kDia;
   out->n = n;
   out->width = (int32_t)d.size();
   out->pitch = pitch;
   out->half = half;
   out->rowptr = rp;
   for (int j = 0; j < 8; j++) out->diag[j] = dd.o[j];
   *ok = true;
   return TNLB_OK;
}

}  // namespace

tnlb_status half_scale(const float* vals, int64_t nnz, cudaStream_t st, float* scale)
{
   *scale = 1.0f;
   if (nnz <= 0) return TNLB_OK;
   DeviceBuffer m;
   TNLB_TRY_STATUS(m.alloc(sizeof(unsigned)));
   TNLB_CUDA_TRY(cudaMemsetAsync(m.ptr, 0, sizeof(unsigned), st));
   k_absmax<<<grid_for(nnz, 256 * 8), 256, 0, st>>>(vals, nnz, m.as<unsigned>());
   TNLB_CHECK_LAUNCH();
   unsigned h = 0;
   TNLB_CUDA_TRY(cudaMemcpyAsync(&h, m.ptr, sizeof(h), cudaMemcpyDeviceToHost, st));
   TNLB_CUDA_TRY(cudaStreamSynchronize(st));
   float mx;
   std::memcpy(&mx, &h, sizeof(mx));
   if (!(mx > 0.0f) || !std::isfinite(mx)) return TNLB_OK;
   int e = 0;
   std::frexp(mx, &e);  // mx < 2^e
   // 2^(14-e) clamped to FP32's normal exponents, so the scale itself stays
   // finite for entries far below 2^-113 (the copy then keeps them small
   // rather than turning them into inf or NaN)
   *scale = std::ldexp(1.0f, std::min(127, std::max(-126, 14 - e)));
   return TNLB_OK;
}

tnlb_status compact_build(const tnlb_segments* seg, const int32_t* cols, const float* vals, bool half, float scale,
                          bool allow_dia, cudaStream_t st, CompactCopy* out, const double* vals64)
{
   out->kind = CompactCopy::kNone;
   out->self_slot = -1;
   if (!spmv_dot_fusable(seg)) return TNLB_OK;
   if (!half) scale = 1.0f;
   DeviceBuffer excess;
   bool use_excess = false;
   if (vals64 && !half)
      TNLB_TRY_STATUS(row_excess(seg->offsets.as<int32_t>(), cols, vals64, seg->n, st, &excess, &use_excess));
   const float* ex = use_excess ? excess.as<float>() : nullptr;
   if (allow_dia) {
      bool ok = false;
      TNLB_TRY_STATUS(diag_build(seg, cols, vals, half, scale, ex, st, out, &ok));
      if (ok) {
         TNLB_CUDA_TRY(cudaStreamSynchronize(st));  // `excess` is released on return
         return TNLB_OK;
      }
   }
   const int32_t n = seg->n;
   const int64_t nnz = seg->elements;
   out->n = n;
   out->width = seg->max_row;
   out->rowptr = seg->offsets.as<int32_t>();
   out->half = half;
   DeviceBuffer bad;
   TNLB_TRY_STATUS(bad.alloc(sizeof(int32_t)));
   TNLB_CUDA_TRY(cudaMemsetAsync(bad.ptr, 0, sizeof(int32_t), st));
   TNLB_TRY_STATUS(out->off.alloc(sizeof(int16_t) * (nnz > 0 ? nnz : 1)));
   k_rel_offsets<<<grid_for(n, 256), 256, 0, st>>>(out->rowptr, cols, n, out->off.as<int16_t>(), bad.as<int32_t>());
   TNLB_CHECK_LAUNCH();
   if (half) {
      TNLB_TRY_STATUS(out->vals.alloc(sizeof(__half) * (nnz > 0 ? nnz : 1)));
      k_to_half<<<grid_for(nnz, 256 * 8), 256, 0, st>>>(vals, nnz, scale, out->vals.as<__half>());
      TNLB_CHECK_LAUNCH();
   }
   else {
      TNLB_TRY_STATUS(out->vals.alloc(sizeof(float) * (nnz > 0 ? nnz : 1)));
      if (nnz) TNLB_CUDA_TRY(cudaMemcpyAsync(out->vals.ptr, vals, sizeof(float) * nnz, cudaMemcpyDeviceToDevice, st));
      if (ex) {
         k_set_diagonal_csr<<<grid_for(n, 256), 256, 0, st>>>(out->rowptr, cols, ex, n, out->vals.as<float>());
         TNLB_CHECK_LAUNCH();
         out->self_slot = 0;
      }
   }
   int32_t h = 0;
   TNLB_CUDA_TRY(cudaMemcpyAsync(&h, bad.ptr, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
   TNLB_CUDA_TRY(cudaStreamSynchronize(st));
   if (h == 0) out->kind = CompactCopy::kRel;
   return TNLB_OK;
}

tnlb_status compact_spmv_dot(const CompactCopy& A, const float* x, float* y, double* partials, unsigned* counter,
                             double* dot_out, cudaStream_t st, const int32_t* skip, bool self_dot)
{
   TNLB_REQUIRE(A.kind != CompactCopy::kNone, TNLB_ERR_INVALID_ARGUMENT, "compact_spmv_dot: no compact copy");
   TNLB_REQUIRE(A.kind != CompactCopy::kDia || (aligned16(x) && aligned16(y)), TNLB_ERR_INVALID_ARGUMENT,
                "compact_spmv_dot: the vectors of a diagonal copy must be 16-byte aligned");
   const RedWork w{partials, counter};
   const int self = self_dot ? 1 : 0;
   if (A.half)
      TNLB_COMPACT_ROWS(A, __half, launch_cmp_dot(rows_, A.n, x, y, w, dot_out, st, skip, self));
   else
      TNLB_COMPACT_ROWS(A, float, launch_cmp_dot(rows_, A.n, x, y, w, dot_out, st, skip, self));
   TNLB_CHECK_LAUNCH();
   return TNLB_OK;
}

bool compact_band_capable(const CompactCopy& A)
{
   if (A.kind != CompactCopy::kDia || A.width < 1 || A.width > 8 || A.pitch % 8 != 0) return false;
   return band_plan(A.diag, A.width, A.half ? 2 : 4, 1, 0).zero;
}

tnlb_status compact_spmv_xpby(const CompactCopy& A, const float* x, float* y, const double* num, const double* den,
                              cudaStream_t st, const int32_t* skip)
{
   TNLB_REQUIRE(A.kind != CompactCopy::kNone, TNLB_ERR_INVALID_ARGUMENT, "compact_spmv_xpby: no compact copy");
   TNLB_REQUIRE(A.kind != CompactCopy::kDia || (aligned16(x) && aligned16(y)), TNLB_ERR_INVALID_ARGUMENT,
                "compact_spmv_xpby: the vectors of a diagonal copy must be 16-byte aligned");
   if (A.half)
      TNLB_COMPACT_ROWS(A, __half, launch_cmp_xpby(rows_, A.n, x, y, num, den, st, skip));
   else
      TNLB_COMPACT_ROWS(A, float, launch_cmp_xpby(rows_, A.n, x, y, num, den, st, skip));
   TNLB_CHECK_LAUNCH();
   return TNLB_OK;
}

}  // namespace tnlb
