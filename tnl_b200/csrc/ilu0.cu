// ilu0.cu -- ILU(0) preconditioner on the GPU.
//
// The reference implements ILU(0) on the host only; its CUDA specialisation
// throws NotImplementedError (Solvers/Linear/Preconditioners/ILU0.h:121-143).
// Here the factorisation and both triangular solves run on the GPU,
// scheduled by dependency levels: row i of L depends on the rows j < i it
// references, row i of U on the rows j > i.  Levels are computed once on the
// host (one pass over the pattern in row order), rows of a level run in
// parallel, one kernel launch per level; the solves are captured once in a
// CUDA graph and replayed; runs of small levels share one single-block
// launch (a __syncthreads between levels).
//
// Arithmetic per row follows ILU0.hpp:59-118 (IKJ order, L_ik = A_ik/U_kk,
// then the updates of the rest of L_i and of U_i with U(k, j) looked up in
// row k of U, 0 if absent) and Utils/TriangularSolve.h:20-103 (ascending
// column order, unit-diagonal L), with separately rounded multiply and
// subtract, so the factors and the solves are bit-identical to the Host.
#include <algorithm>
#include <vector>

#include "internal.cuh"
#include "segview.cuh"

namespace tnlb {
namespace {

template <typename Real>
__device__ __forceinline__ Real mul_rn(Real a, Real b);
template <>
__device__ __forceinline__ double mul_rn<double>(double a, double b)
{
   return __dmul_rn(a, b);
}
template <>
__device__ __forceinline__ float mul_rn<float>(float a, float b)
{
   return __fmul_rn(a, b);
}
template <typename Real>
__device__ __forceinline__ Real sub_rn(Real a, Real b);
template <>
__device__ __forceinline__ double sub_rn<double>(double a, double b)
{
   return __dsub_rn(a, b);
}
template <>
__device__ __forceinline__ float sub_rn<float>(float a, float b)
{
   return __fsub_rn(a, b);
}
template <typename Real>
__device__ __forceinline__ Real div_rn(Real a, Real b);
template <>
__device__ __forceinline__ double div_rn<double>(double a, double b)
{
   return __ddiv_rn(a, b);
}
template <>
__device__ __forceinline__ float div_rn<float>(float a, float b)
{
   return __fdiv_rn(a, b);
}

// One thread per row of the level.  lu holds A's values and is overwritten by
// the factors; lstart/ustart/uend delimit the L and U parts of each row.
template <typename Real>
__global__ void k_factor_level(const int32_t* __restrict__ rows, int32_t count, const int32_t* __restrict__ cols,
                               Real* __restrict__ lu, const int32_t* __restrict__ lstart,
                               const int32_t* __restrict__ ustart, const int32_t* __restrict__ uend)
{
   const int32_t t = blockIdx.x * blockDim.x + threadIdx.x;
   if (t >= count) return;
   const int32_t i = rows[t];
   const int32_t l0 = lstart[i], u0 = ustart[i], u1 = uend[i];
   for (int32_t ck = l0; ck < u0; ck++) {
      const int32_t k = cols[ck];
      const int32_t k0 = ustart[k], k1 = uend[k];
      // U(k,k): getElement searches row k of U; 0 if absent
      Real ukk = 0;
      for (int32_t q = k0; q < k1; q++)
         if (cols[q] == k) {
            ukk = lu[q];
            break;
         }
      const Real lik = div_rn(lu[ck], ukk);
      lu[ck] = lik;
      // remaining L entries and the U entries of row i, each minus L_ik*U(k,j)
      int32_t q = k0;
      for (int32_t cj = ck + 1; cj < u1; cj++) {
         const int32_t j = cols[cj];
         while (q < k1 && cols[q] < j) q++;
         const Real ukj = (q < k1 && cols[q] == j) ? lu[q] : Real(0);
         lu[cj] = sub_rn(lu[cj], mul_rn(lik, ukj));
      }
   }
}

// Forward substitution with unit-diagonal L for the rows of one level.
template <typename Real>
__global__ void k_lower_level(const int32_t* __restrict__ rows, int32_t count, const int32_t* __restrict__ cols,
                              const Real* __restrict__ lu, const int32_t* __restrict__ lstart,
                              const int32_t* __restrict__ ustart, const Real* __restrict__ b, Real* __restrict__ x)
{
   const int32_t t = blockIdx.x * blockDim.x + threadIdx.x;
   if (t >= count) return;
   const int32_t i = rows[t];
   Real xi = b[i];
   for (int32_t c = lstart[i]; c < ustart[i]; c++) xi = sub_rn(xi, mul_rn(lu[c], x[cols[c]]));
   x[i] = xi;
}

// Back substitution: x_i = (y_i - sum_{j>i} U_ij x_j) / U_ii (diagonal first in U_i).
template <typename Real>
__global__ void k_upper_level(const int32_t* __restrict__ rows, int32_t count, const int32_t* __restrict__ cols,
                              const Real* __restrict__ lu, const int32_t* __restrict__ ustart,
                              const int32_t* __restrict__ uend, Real* __restrict__ x)
{
   const int32_t t = blockIdx.x * blockDim.x + threadIdx.x;
   if (t >= count) return;
   const int32_t i = rows[t];
   const int32_t u0 = ustart[i];
   Real xi = x[i];
   for (int32_t c = u0 + 1; c < uend[i]; c++) xi = sub_rn(xi, mul_rn(lu[c], x[cols[c]]));
   x[i] = div_rn(xi, u0 < uend[i] ? lu[u0] : Real(0));  // an empty U row: pivot 0, as a padding slot
}

// Runs of consecutive small levels in ONE block: the block walks the levels
// in order, a __syncthreads between levels making each level's x visible to
// the next (the same block, so no grid-wide wait); the row arithmetic is
// that of k_lower_level / k_upper_level.
constexpr int kIluRunThreads = 1024;
constexpr int32_t kIluSmallLevel = 2048;

template <typename Real>
__global__ void __launch_bounds__(kIluRunThreads)
   k_lower_run(const int32_t* __restrict__ rows, const int32_t* __restrict__ lvl, int32_t l0, int32_t l1,
               const int32_t* __restrict__ cols, const Real* __restrict__ lu, const int32_t* __restrict__ lstart,
               const int32_t* __restrict__ ustart, const Real* __restrict__ b, Real* __restrict__ x)
{
   for (int32_t l = l0; l < l1; l++) {
      const int32_t s0 = lvl[l], s1 = lvl[l + 1];
      for (int32_t t = s0 + threadIdx.x; t < s1; t += blockDim.x) {
         const int32_t i = rows[t];
         Real xi = b[i];
         for (int32_t c = lstart[i]; c < ustart[i]; c++) xi = sub_rn(xi, mul_rn(lu[c], x[cols[c]]));
         x[i] = xi;
      }
      __syncthreads();
   }
}

template <typename Real>
__global__ void __launch_bounds__(kIluRunThreads)
   k_upper_run(const int32_t* __restrict__ rows, const int32_t* __restrict__ lvl, int32_t l0, int32_t l1,
               const int32_t* __restrict__ cols, const Real* __restrict__ lu, const int32_t* __restrict__ ustart,
               const int32_t* __restrict__ uend, Real* __restrict__ x)
{
   for (int32_t l = l0; l < l1; l++) {
      const int32_t s0 = lvl[l], s1 = lvl[l + 1];
      for (int32_t t = s0 + threadIdx.x; t < s1; t += blockDim.x) {
         const int32_t i = rows[t];
         const int32_t u0 = ustart[i];
         Real xi = x[i];
         for (int32_t c = u0 + 1; c < uend[i]; c++) xi = sub_rn(xi, mul_rn(lu[c], x[cols[c]]));
         x[i] = div_rn(xi, u0 < uend[i] ? lu[u0] : Real(0));
      }
      __syncthreads();
   }
}

// Level-ordered packed factors: position t of the level order (row
// rows[t]) holds its K (padded) L entries at pc/pv[t*K ..] (column -1 pads),
// and for U its off-diagonal entries plus the diagonal at dv[t]; the
// solve's input is permuted to the same order first (in[t] = b[rows[t]]).
// A row then needs one load of its own data and the gathers of x.
template <typename Real>
__global__ void k_permute(const int32_t* __restrict__ rows, int32_t n, const Real* __restrict__ src,
                          Real* __restrict__ dst)
{
   const int32_t t = blockIdx.x * blockDim.x + threadIdx.x;
   if (t < n) dst[t] = src[rows[t]];
}

template <typename Real>
__global__ void k_pack_vals(const int64_t* __restrict__ src, int64_t count, const Real* __restrict__ lu,
                            Real* __restrict__ dst)
{
   const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (k < count) dst[k] = src[k] >= 0 ? lu[src[k]] : Real(0);
}

// Rows of one (large) level, packed: x_i = in_t - sum_j L_ij x_j.
template <typename Real, int K>
__global__ void k_lower_packed(int32_t t0, int32_t count, const int32_t* __restrict__ rows,
                               const int32_t* __restrict__ pc, const Real* __restrict__ pv,
                               const Real* __restrict__ in, Real* x)
{
   const int32_t t = t0 + blockIdx.x * blockDim.x + threadIdx.x;
   if (t >= t0 + count) return;
   int32_t c[K];
   Real v[K];
#pragma unroll
   for (int j = 0; j < K; j++) {
      c[j] = pc[(int64_t)t * K + j];
      v[j] = pv[(int64_t)t * K + j];
   }
   const int32_t i = rows[t];
   Real xi = in[t];
#pragma unroll
   for (int j = 0; j < K; j++)
      if (c[j] >= 0) xi = sub_rn(xi, mul_rn(v[j], x[c[j]]));
   x[i] = xi;
}

// x_i = (in_t - sum_{j>i} U_ij x_j) / U_ii for the rows of one level, packed.
template <typename Real, int K>
__global__ void k_upper_packed(int32_t t0, int32_t count, const int32_t* __restrict__ rows,
                               const int32_t* __restrict__ pc, const Real* __restrict__ pv,
                               const Real* __restrict__ dv, const Real* __restrict__ in, Real* x)
{
   const int32_t t = t0 + blockIdx.x * blockDim.x + threadIdx.x;
   if (t >= t0 + count) return;
   int32_t c[K];
   Real v[K];
#pragma unroll
   for (int j = 0; j < K; j++) {
      c[j] = pc[(int64_t)t * K + j];
      v[j] = pv[(int64_t)t * K + j];
   }
   const int32_t i = rows[t];
   Real xi = in[t];
#pragma unroll
   for (int j = 0; j < K; j++)
      if (c[j] >= 0) xi = sub_rn(xi, mul_rn(v[j], x[c[j]]));
   x[i] = div_rn(xi, dv[t]);
}

// Runs of levels of at most kIluPipeThreads rows in one block, one row per
// thread per level, software-pipelined: the packed data and input of a
// thread's row in level l+1 (independent of x) are loaded while level l is
// solved, so after each __syncthreads only the gathers of x wait.
constexpr int kIluPipeThreads = 1024;
constexpr int32_t kIluPipeMaxLevels = 4096;

template <typename Real, int K, bool Upper>
__global__ void __launch_bounds__(kIluPipeThreads)
   k_solve_pipe(const int32_t* __restrict__ lvl, int32_t l0, int32_t l1, const int32_t* __restrict__ rows,
                const int32_t* __restrict__ pc, const Real* __restrict__ pv, const Real* __restrict__ dv,
                const Real* __restrict__ in, Real* x)
{
   __shared__ int32_t s_lvl[kIluPipeMaxLevels + 1];
   for (int32_t k = threadIdx.x; k <= l1 - l0; k += blockDim.x) s_lvl[k] = lvl[l0 + k];
   __syncthreads();
   int32_t i_n = -1, c_n[K];
   Real v_n[K], in_n = Real(0), d_n = Real(1);
   auto load = [&](int32_t l) {
      i_n = -1;
      if (l >= l1) return;
      const int32_t t = s_lvl[l - l0] + (int32_t)threadIdx.x;
      if (t >= s_lvl[l - l0 + 1]) return;
      i_n = rows[t];
      in_n = in[t];
      if (Upper) d_n = dv[t];
#pragma unroll
      for (int j = 0; j < K; j++) {
         c_n[j] = pc[(int64_t)t * K + j];
         v_n[j] = pv[(int64_t)t * K + j];
      }
   };
   load(l0);
   for (int32_t l = l0; l < l1; l++) {
      const int32_t i = i_n;
      int32_t c[K];
      Real v[K];
#pragma unroll
      for (int j = 0; j < K; j++) {
         c[j] = c_n[j];
         v[j] = v_n[j];
      }
      Real xi = in_n;
      const Real di = d_n;
      load(l + 1);
      if (i >= 0) {
#pragma unroll
         for (int j = 0; j < K; j++)
            if (c[j] >= 0) xi = sub_rn(xi, mul_rn(v[j], x[c[j]]));
         x[i] = Upper ? div_rn(xi, di) : xi;
      }
      __syncthreads();
   }
}

struct Ilu0Base {
   virtual ~Ilu0Base() = default;
   virtual tnlb_status apply(const void* b, void* x, cudaStream_t st) = 0;
};

template <typename Real>
struct Ilu0 : Ilu0Base {
   int32_t n = 0;
   DeviceBuffer rp, cols, lu, lstart, ustart, uend, lrows, urows, tmp, dlptr, duptr;
   // packed level-ordered factors (when every row has <= 8 L and <= 8
   // off-diagonal U entries): strides kl / ku
   int kl = 0, ku = 0;
   DeviceBuffer lpc, lpv, upc, upv, udv, perm;
   std::vector<int32_t> lptr, uptr;  // level boundaries into lrows / urows
   cudaGraphExec_t exec = nullptr;
   const Real* g_b = nullptr;
   Real* g_x = nullptr;
   cudaStream_t cs = nullptr;

   ~Ilu0() override
   {
      if (exec) cudaGraphExecDestroy(exec);
      if (cs) cudaStreamDestroy(cs);
   }

   template <int KL, int KU>
   void enqueue_packed(const Real* b, Real* x, cudaStream_t st)
   {
      Real* in = perm.as<Real>();
      const unsigned g = (unsigned)((n + 255) / 256);
      k_permute<Real><<<g, 256, 0, st>>>(lrows.as<int32_t>(), n, b, in);
      const int32_t nl = (int32_t)lptr.size() - 1;
      for (int32_t l = 0; l < nl;) {
         if (lptr[l + 1] - lptr[l] <= kIluPipeThreads) {
            int32_t e = l;
            while (e < nl && e - l < kIluPipeMaxLevels && lptr[e + 1] - lptr[e] <= kIluPipeThreads) e++;
            k_solve_pipe<Real, KL, false><<<1, kIluPipeThreads, 0, st>>>(
               dlptr.as<int32_t>(), l, e, lrows.as<int32_t>(), lpc.as<int32_t>(), lpv.as<Real>(), nullptr, in, x);
            l = e;
            continue;
         }
         const int32_t cnt = lptr[l + 1] - lptr[l];
         k_lower_packed<Real, KL><<<(cnt + 127) / 128, 128, 0, st>>>(lptr[l], cnt, lrows.as<int32_t>(),
                                                                     lpc.as<int32_t>(), lpv.as<Real>(), in, x);
         l++;
      }
      k_permute<Real><<<g, 256, 0, st>>>(urows.as<int32_t>(), n, x, in);
      const int32_t nu = (int32_t)uptr.size() - 1;
      for (int32_t l = 0; l < nu;) {
         if (uptr[l + 1] - uptr[l] <= kIluPipeThreads) {
            int32_t e = l;
            while (e < nu && e - l < kIluPipeMaxLevels && uptr[e + 1] - uptr[e] <= kIluPipeThreads) e++;
            k_solve_pipe<Real, KU, true><<<1, kIluPipeThreads, 0, st>>>(
               duptr.as<int32_t>(), l, e, urows.as<int32_t>(), upc.as<int32_t>(), upv.as<Real>(), udv.as<Real>(),
               in, x);
            l = e;
            continue;
         }
         const int32_t cnt = uptr[l + 1] - uptr[l];
         k_upper_packed<Real, KU><<<(cnt + 127) / 128, 128, 0, st>>>(uptr[l], cnt, urows.as<int32_t>(),
                                                                     upc.as<int32_t>(), upv.as<Real>(),
                                                                     udv.as<Real>(), in, x);
         l++;
      }
   }

   template <int KL>
   void enqueue_packed_u(const Real* b, Real* x, cudaStream_t st)
   {
      if (ku <= 1) enqueue_packed<KL, 1>(b, x, st);
      else if (ku <= 2) enqueue_packed<KL, 2>(b, x, st);
      else if (ku <= 4) enqueue_packed<KL, 4>(b, x, st);
      else enqueue_packed<KL, 8>(b, x, st);
   }

   // Levels in order.  Packed factors: runs of levels of at most
   // kIluPipeThreads rows go to one pipelined single-block launch, a larger
   // level to its own grid.  Otherwise (a row with more than 8 entries in L
   // or U): runs of levels of at most kIluSmallLevel rows in one
   // single-block launch, larger levels to their own grids.
   void enqueue(const Real* b, Real* x, cudaStream_t st)
   {
      if (kl > 0) {
         if (kl <= 1) enqueue_packed_u<1>(b, x, st);
         else if (kl <= 2) enqueue_packed_u<2>(b, x, st);
         else if (kl <= 4) enqueue_packed_u<4>(b, x, st);
         else enqueue_packed_u<8>(b, x, st);
         return;
      }
      const int32_t nl = (int32_t)lptr.size() - 1;
      for (int32_t l = 0; l < nl;) {
         if (lptr[l + 1] - lptr[l] <= kIluSmallLevel) {
            int32_t e = l;
            while (e < nl && lptr[e + 1] - lptr[e] <= kIluSmallLevel) e++;
            k_lower_run<Real><<<1, kIluRunThreads, 0, st>>>(lrows.as<int32_t>(), dlptr.as<int32_t>(), l, e,
                                                            cols.as<int32_t>(), lu.as<Real>(), lstart.as<int32_t>(),
                                                            ustart.as<int32_t>(), b, x);
            l = e;
            continue;
         }
         const int32_t cnt = lptr[l + 1] - lptr[l];
         k_lower_level<Real><<<(cnt + 127) / 128, 128, 0, st>>>(lrows.as<int32_t>() + lptr[l], cnt, cols.as<int32_t>(),
                                                               lu.as<Real>(), lstart.as<int32_t>(),
                                                               ustart.as<int32_t>(), b, x);
         l++;
      }
      const int32_t nu = (int32_t)uptr.size() - 1;
      for (int32_t l = 0; l < nu;) {
         if (uptr[l + 1] - uptr[l] <= kIluSmallLevel) {
            int32_t e = l;
            while (e < nu && uptr[e + 1] - uptr[e] <= kIluSmallLevel) e++;
            k_upper_run<Real><<<1, kIluRunThreads, 0, st>>>(urows.as<int32_t>(), duptr.as<int32_t>(), l, e,
                                                            cols.as<int32_t>(), lu.as<Real>(), ustart.as<int32_t>(),
                                                            uend.as<int32_t>(), x);
            l = e;
            continue;
         }
         const int32_t cnt = uptr[l + 1] - uptr[l];
         k_upper_level<Real><<<(cnt + 127) / 128, 128, 0, st>>>(urows.as<int32_t>() + uptr[l], cnt, cols.as<int32_t>(),
                                                               lu.as<Real>(), ustart.as<int32_t>(),
                                                               uend.as<int32_t>(), x);
         l++;
      }
   }

   tnlb_status apply(const void* bv, void* xv, cudaStream_t st) override
   {
      const Real* b = static_cast<const Real*>(bv);
      Real* x = static_cast<Real*>(xv);
      // Solves are replayed from a graph captured for fixed (b, x) buffers:
      // copy in/out of the graph's own buffers when the caller's differ.
      if (!exec) {
         TNLB_TRY_STATUS(tmp.alloc(sizeof(Real) * 2 * (size_t)(n > 0 ? n : 1)));
         g_b = tmp.as<Real>();
         g_x = tmp.as<Real>() + n;
         TNLB_CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
         cudaGraph_t graph = nullptr;
         TNLB_CUDA_TRY(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
         enqueue(g_b, g_x, cs);
         TNLB_CUDA_TRY(cudaStreamEndCapture(cs, &graph));
         cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
         cudaGraphDestroy(graph);
         TNLB_CUDA_TRY(e);
      }
      cudaEvent_t ev;
      TNLB_CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
      TNLB_CUDA_TRY(cudaMemcpyAsync((void*)g_b, b, sizeof(Real) * n, cudaMemcpyDeviceToDevice, st));
      TNLB_CUDA_TRY(cudaEventRecord(ev, st));
      TNLB_CUDA_TRY(cudaStreamWaitEvent(cs, ev, 0));
      TNLB_CUDA_TRY(cudaGraphLaunch(exec, cs));
      TNLB_CUDA_TRY(cudaEventRecord(ev, cs));
      TNLB_CUDA_TRY(cudaStreamWaitEvent(st, ev, 0));
      TNLB_CUDA_TRY(cudaMemcpyAsync(x, g_x, sizeof(Real) * n, cudaMemcpyDeviceToDevice, st));
      cudaEventDestroy(ev);
      return TNLB_OK;
   }
};

template <typename Real>
tnlb_status analyze_t(Ilu0<Real>* P, const std::vector<int32_t>& rp, const std::vector<int32_t>& cols, bool factorize,
                      cudaStream_t st);

template <typename Real>
tnlb_status create_t(const tnlb_segments* seg, const int32_t* cols_in, const Real* vals_in, cudaStream_t st,
                     Ilu0<Real>** out)
{
   const int32_t n = seg->n;
   auto* P = new Ilu0<Real>();
   P->n = n;
   // CSR copy of the matrix (rows in slot order, padding dropped)
   TNLB_TRY_STATUS(gather_csr(view_of(seg), sizeof(Real) == 8 ? TNLB_F64 : TNLB_F32, cols_in, vals_in, P->rp, P->cols,
                              P->lu, st));
   int64_t nnz = 0;
   {
      int32_t t = 0;
      TNLB_CUDA_TRY(cudaMemcpyAsync(&t, P->rp.template as<int32_t>() + n, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
      TNLB_CUDA_TRY(cudaStreamSynchronize(st));
      nnz = t;
   }
   // host analysis: L/U split and dependency levels
   std::vector<int32_t> rp(n + 1), cols(nnz);
   TNLB_CUDA_TRY(cudaMemcpyAsync(rp.data(), P->rp.ptr, sizeof(int32_t) * (n + 1), cudaMemcpyDeviceToHost, st));
   if (nnz) TNLB_CUDA_TRY(cudaMemcpyAsync(cols.data(), P->cols.ptr, sizeof(int32_t) * nnz, cudaMemcpyDeviceToHost, st));
   TNLB_CUDA_TRY(cudaStreamSynchronize(st));
   TNLB_TRY_STATUS(analyze_t(P, rp, cols, true, st));
   *out = P;
   return TNLB_OK;
}

// Factors given on the host (ILUT): row i holds its L entries (columns < i)
// then its U entries, the first U entry the pivot; the level analysis,
// packing and solves are those of ILU(0).
template <typename Real>
tnlb_status create_from_factors_t(int32_t n, const std::vector<int32_t>& rp, const std::vector<int32_t>& cols,
                                  const std::vector<Real>& lu, cudaStream_t st, Ilu0<Real>** out)
{
   auto* P = new Ilu0<Real>();
   P->n = n;
   const size_t nnz = (size_t)rp[n];
   TNLB_TRY_STATUS(P->rp.alloc(sizeof(int32_t) * ((size_t)n + 1)));
   TNLB_TRY_STATUS(P->cols.alloc(sizeof(int32_t) * (nnz ? nnz : 1)));
   TNLB_TRY_STATUS(P->lu.alloc(sizeof(Real) * (nnz ? nnz : 1)));
   TNLB_CUDA_TRY(cudaMemcpyAsync(P->rp.ptr, rp.data(), sizeof(int32_t) * ((size_t)n + 1), cudaMemcpyHostToDevice, st));
   if (nnz) {
      TNLB_CUDA_TRY(cudaMemcpyAsync(P->cols.ptr, cols.data(), sizeof(int32_t) * nnz, cudaMemcpyHostToDevice, st));
      TNLB_CUDA_TRY(cudaMemcpyAsync(P->lu.ptr, lu.data(), sizeof(Real) * nnz, cudaMemcpyHostToDevice, st));
   }
   TNLB_TRY_STATUS(analyze_t(P, rp, cols, false, st));
   *out = P;
   return TNLB_OK;
}

// L/U split, dependency levels, level order and packed copies of the factors;
// with `factorize`, the ILU(0) factorisation of P->lu in place first.
template <typename Real>
tnlb_status analyze_t(Ilu0<Real>* P, const std::vector<int32_t>& rp, const std::vector<int32_t>& cols, bool factorize,
                      cudaStream_t st)
{
   const int32_t n = P->n;
   std::vector<int32_t> ls(n), us(n), ue(n), llev(n, 0), ulev(n, 0);
   int32_t lmax = 0, umax = 0;
   for (int32_t i = 0; i < n; i++) {
      int32_t c = rp[i];
      // ILU0.hpp:35-55: columns < i -> L, i <= column < N -> U (sorted rows)
      ls[i] = c;
      while (c < rp[i + 1] && cols[c] < i) c++;
      us[i] = c;
      while (c < rp[i + 1] && cols[c] < n) c++;
      ue[i] = c;
      int32_t lv = 0;
      for (int32_t q = ls[i]; q < us[i]; q++) lv = std::max(lv, llev[cols[q]] + 1);
      llev[i] = lv;
      lmax = std::max(lmax, lv);
   }
   for (int32_t i = n - 1; i >= 0; i--) {
      int32_t lv = 0;
      for (int32_t q = us[i] + 1; q < ue[i]; q++) lv = std::max(lv, ulev[cols[q]] + 1);
      ulev[i] = lv;
      umax = std::max(umax, lv);
   }
   auto bucket = [&](const std::vector<int32_t>& lev, int32_t maxl, std::vector<int32_t>& ptr,
                     std::vector<int32_t>& rows) {
      ptr.assign(maxl + 2, 0);
      for (int32_t i = 0; i < n; i++) ptr[lev[i] + 1]++;
      for (int32_t l = 0; l <= maxl; l++) ptr[l + 1] += ptr[l];
      rows.resize(n);
      std::vector<int32_t> pos(ptr.begin(), ptr.end() - 1);
      for (int32_t i = 0; i < n; i++) rows[pos[lev[i]]++] = i;
   };
   std::vector<int32_t> lrows, urows;
   bucket(llev, n > 0 ? lmax : -1, P->lptr, lrows);
   bucket(ulev, n > 0 ? umax : -1, P->uptr, urows);
   TNLB_TRY_STATUS(P->lstart.alloc(sizeof(int32_t) * (n ? n : 1)));
   TNLB_TRY_STATUS(P->ustart.alloc(sizeof(int32_t) * (n ? n : 1)));
   TNLB_TRY_STATUS(P->uend.alloc(sizeof(int32_t) * (n ? n : 1)));
   TNLB_TRY_STATUS(P->lrows.alloc(sizeof(int32_t) * (n ? n : 1)));
   TNLB_TRY_STATUS(P->urows.alloc(sizeof(int32_t) * (n ? n : 1)));
   TNLB_CUDA_TRY(cudaMemcpyAsync(P->lstart.ptr, ls.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, st));
   TNLB_CUDA_TRY(cudaMemcpyAsync(P->ustart.ptr, us.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, st));
   TNLB_CUDA_TRY(cudaMemcpyAsync(P->uend.ptr, ue.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, st));
   TNLB_CUDA_TRY(cudaMemcpyAsync(P->lrows.ptr, lrows.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, st));
   TNLB_CUDA_TRY(cudaMemcpyAsync(P->urows.ptr, urows.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, st));
   TNLB_TRY_STATUS(P->dlptr.alloc(sizeof(int32_t) * P->lptr.size()));
   TNLB_TRY_STATUS(P->duptr.alloc(sizeof(int32_t) * P->uptr.size()));
   TNLB_CUDA_TRY(cudaMemcpyAsync(P->dlptr.ptr, P->lptr.data(), sizeof(int32_t) * P->lptr.size(), cudaMemcpyHostToDevice,
                                 st));
   TNLB_CUDA_TRY(cudaMemcpyAsync(P->duptr.ptr, P->uptr.data(), sizeof(int32_t) * P->uptr.size(), cudaMemcpyHostToDevice,
                                 st));
   // factorisation, level by level of L
   for (size_t l = 0; factorize && l + 1 < P->lptr.size(); l++) {
      const int32_t c = P->lptr[l + 1] - P->lptr[l];
      k_factor_level<Real><<<(c + 127) / 128, 128, 0, st>>>(P->lrows.template as<int32_t>() + P->lptr[l], c, P->cols.template as<int32_t>(),
                                                           P->lu.template as<Real>(), P->lstart.template as<int32_t>(),
                                                           P->ustart.template as<int32_t>(), P->uend.template as<int32_t>());
   }
   TNLB_CHECK_LAUNCH();
   // packed level-ordered copies of the factors
   int32_t ml = 0, mu = 0;
   for (int32_t i = 0; i < n; i++) {
      ml = std::max(ml, us[i] - ls[i]);
      mu = std::max(mu, ue[i] - us[i] - 1);
   }
   if (ml <= 8 && mu <= 8) {
      auto stride = [](int32_t m) { return m <= 1 ? 1 : m <= 2 ? 2 : m <= 4 ? 4 : 8; };
      const int kl = stride(ml), ku = stride(mu);
      std::vector<int32_t> lpc((size_t)n * kl, -1), upc((size_t)n * ku, -1);
      std::vector<int64_t> lsrc((size_t)n * kl, -1), usrc((size_t)n * ku, -1), dsrc(n, -1);
      for (int32_t t = 0; t < n; t++) {
         const int32_t i = lrows[t];
         for (int32_t j = 0; j < us[i] - ls[i]; j++) {
            lpc[(size_t)t * kl + j] = cols[ls[i] + j];
            lsrc[(size_t)t * kl + j] = ls[i] + j;
         }
         const int32_t r = urows[t];
         for (int32_t j = 0; j < ue[r] - us[r] - 1; j++) {
            upc[(size_t)t * ku + j] = cols[us[r] + 1 + j];
            usrc[(size_t)t * ku + j] = us[r] + 1 + j;
         }
         dsrc[t] = us[r] < ue[r] ? us[r] : -1;
      }
      DeviceBuffer src;
      TNLB_TRY_STATUS(src.alloc(sizeof(int64_t) * (size_t)n * std::max(kl, ku)));
      TNLB_TRY_STATUS(P->lpc.alloc(sizeof(int32_t) * (size_t)n * kl));
      TNLB_TRY_STATUS(P->upc.alloc(sizeof(int32_t) * (size_t)n * ku));
      TNLB_TRY_STATUS(P->lpv.alloc(sizeof(Real) * (size_t)n * kl));
      TNLB_TRY_STATUS(P->upv.alloc(sizeof(Real) * (size_t)n * ku));
      TNLB_TRY_STATUS(P->udv.alloc(sizeof(Real) * (size_t)n));
      TNLB_TRY_STATUS(P->perm.alloc(sizeof(Real) * (size_t)n));
      TNLB_CUDA_TRY(cudaMemcpyAsync(P->lpc.ptr, lpc.data(), sizeof(int32_t) * lpc.size(), cudaMemcpyHostToDevice, st));
      TNLB_CUDA_TRY(cudaMemcpyAsync(P->upc.ptr, upc.data(), sizeof(int32_t) * upc.size(), cudaMemcpyHostToDevice, st));
      // one staging buffer for the three gathers: synchronise between them
      auto pack = [&](const std::vector<int64_t>& h, DeviceBuffer& dst) -> tnlb_status {
         TNLB_CUDA_TRY(cudaMemcpyAsync(src.ptr, h.data(), sizeof(int64_t) * h.size(), cudaMemcpyHostToDevice, st));
         const int64_t cnt = (int64_t)h.size();
         k_pack_vals<Real><<<(unsigned)((cnt + 255) / 256), 256, 0, st>>>(src.as<int64_t>(), cnt,
                                                                          P->lu.template as<Real>(),
                                                                          dst.template as<Real>());
         TNLB_CHECK_LAUNCH();
         TNLB_CUDA_TRY(cudaStreamSynchronize(st));
         return TNLB_OK;
      };
      TNLB_TRY_STATUS(pack(lsrc, P->lpv));
      TNLB_TRY_STATUS(pack(usrc, P->upv));
      TNLB_TRY_STATUS(pack(dsrc, P->udv));
      P->kl = kl;
      P->ku = ku;
   }
   TNLB_CUDA_TRY(cudaStreamSynchronize(st));
   return TNLB_OK;
}

}  // namespace

tnlb_status ilu0_create(const tnlb_segments* seg, tnlb_real real, const int32_t* cols, const void* vals,
                        cudaStream_t st, void** out)
{
   TNLB_REQUIRE(seg->n > 0, TNLB_ERR_INVALID_ARGUMENT, "ILU0::update: the matrix is empty");
   if (real == TNLB_F64) {
      Ilu0<double>* p = nullptr;
      tnlb_status s = create_t<double>(seg, cols, (const double*)vals, st, &p);
      *out = static_cast<Ilu0Base*>(p);
      return s;
   }
   Ilu0<float>* p = nullptr;
   tnlb_status s = create_t<float>(seg, cols, (const float*)vals, st, &p);
   *out = static_cast<Ilu0Base*>(p);
   return s;
}

tnlb_status ilu_from_factors(tnlb_real real, int32_t n, const std::vector<int32_t>& rp,
                             const std::vector<int32_t>& cols, const void* lu, cudaStream_t st, void** out)
{
   if (real == TNLB_F64) {
      Ilu0<double>* p = nullptr;
      const double* v = static_cast<const double*>(lu);
      tnlb_status s = create_from_factors_t<double>(n, rp, cols, std::vector<double>(v, v + rp[n]), st, &p);
      *out = static_cast<Ilu0Base*>(p);
      return s;
   }
   Ilu0<float>* p = nullptr;
   const float* v = static_cast<const float*>(lu);
   tnlb_status s = create_from_factors_t<float>(n, rp, cols, std::vector<float>(v, v + rp[n]), st, &p);
   *out = static_cast<Ilu0Base*>(p);
   return s;
}

tnlb_status ilu0_apply(void* ilu, const void* b, void* x, cudaStream_t st)
{
   return static_cast<Ilu0Base*>(ilu)->apply(b, x, st);
}

void ilu0_destroy(void* ilu) { delete static_cast<Ilu0Base*>(ilu); }

// Factors for inspection: CSR pattern (rowptr n+1, cols nnz) and LU values
// (L strictly below the diagonal, U from the diagonal on), copied to the host.
tnlb_status ilu0_read(void* ilu, int32_t* h_rowptr, int32_t* h_cols, void* h_vals, int64_t capacity, int real_bytes)
{
   auto* b = static_cast<Ilu0Base*>(ilu);
   if (real_bytes == 8) {
      auto* p = dynamic_cast<Ilu0<double>*>(b);
      TNLB_REQUIRE(p, TNLB_ERR_INVALID_ARGUMENT, "real type mismatch");
      int32_t nnz = 0;
      TNLB_CUDA_TRY(cudaMemcpy(&nnz, p->rp.as<int32_t>() + p->n, sizeof(int32_t), cudaMemcpyDeviceToHost));
      TNLB_REQUIRE(capacity >= nnz, TNLB_ERR_INVALID_ARGUMENT, "buffer too small");
      TNLB_CUDA_TRY(cudaMemcpy(h_rowptr, p->rp.ptr, sizeof(int32_t) * (p->n + 1), cudaMemcpyDeviceToHost));
      TNLB_CUDA_TRY(cudaMemcpy(h_cols, p->cols.ptr, sizeof(int32_t) * nnz, cudaMemcpyDeviceToHost));
      TNLB_CUDA_TRY(cudaMemcpy(h_vals, p->lu.ptr, sizeof(double) * nnz, cudaMemcpyDeviceToHost));
      return TNLB_OK;
   }
   auto* p = dynamic_cast<Ilu0<float>*>(b);
   TNLB_REQUIRE(p, TNLB_ERR_INVALID_ARGUMENT, "real type mismatch");
   int32_t nnz = 0;
   TNLB_CUDA_TRY(cudaMemcpy(&nnz, p->rp.as<int32_t>() + p->n, sizeof(int32_t), cudaMemcpyDeviceToHost));
   TNLB_REQUIRE(capacity >= nnz, TNLB_ERR_INVALID_ARGUMENT, "buffer too small");
   TNLB_CUDA_TRY(cudaMemcpy(h_rowptr, p->rp.ptr, sizeof(int32_t) * (p->n + 1), cudaMemcpyDeviceToHost));
   TNLB_CUDA_TRY(cudaMemcpy(h_cols, p->cols.ptr, sizeof(int32_t) * nnz, cudaMemcpyDeviceToHost));
   TNLB_CUDA_TRY(cudaMemcpy(h_vals, p->lu.ptr, sizeof(float) * nnz, cudaMemcpyDeviceToHost));
   return TNLB_OK;
}

}  // namespace tnlb
