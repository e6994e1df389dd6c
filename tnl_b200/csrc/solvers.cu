// solvers.cu -- CG, BiCGStab and GMRES on the GPU with the Jacobi (Diagonal)
// and ILU(0) preconditioners, plus FP32-inner / FP64 iterative refinement.
//
// The iteration logic and stopping rules follow the reference exactly:
// CG.hpp:12-109, BICGStab.hpp:34-164, GMRES.hpp:73-347/436-465/648-770,
// IterativeSolver.hpp:98-143 (nextIteration checks, then increments; solve()
// returns checkConvergence()).  What changes is where the scalars live: every
// dot product and norm is reduced on the device into a DevState record, and
// the scalar recurrences (alpha, beta, residue, the stopping test) run in the
// last block of the reduction.  CG never waits for the host inside an
// iteration: batches of iterations are captured once in a CUDA graph and
// replayed; kernels of iterations past the stopping point return at once on
// the device `done` flag, so the iteration count is exact.  BiCGStab and
// GMRES read the state once per iteration / Arnoldi step.  GMRES keeps the
// small Hessenberg least-squares problem (Givens rotations, back
// substitution) on the host in FP64, as the reference does.
#include <cfloat>
#include <cmath>
#include <random>
#include <vector>

#include "internal.cuh"
#include "reduce.cuh"
#include "segview.cuh"
#include "compact.cuh"
#include "band.cuh"

namespace tnlb {

// Device-resident solver scalars.
struct DevState {
   double normb, s1, s2, alpha, beta, omega, rho, rho_old, r_ast_sqnorm, residue;
   double conv, div;
   int32_t it, done, maxit, minit;
   int32_t flag;
   uint32_t loops;  // bodies run by the current launch of a looping iteration graph
};

__device__ __forceinline__ bool check_next(const DevState& S)
{
   return !(isnan(S.residue) || S.it > S.maxit || (S.residue > S.div && S.it >= S.minit) ||
            (S.residue < S.conv && S.it >= S.minit));
}

// IterativeSolver::nextIteration (IterativeSolver.hpp:98-108).
__device__ __forceinline__ void next_iteration(DevState& S)
{
   const bool c = check_next(S);
   S.it++;
   if (!c) S.done = 1;
}

// IterativeSolver::checkConvergence (IterativeSolver.hpp:121-143).
static bool check_convergence(double residue, int it, int maxit, int minit, double conv, double div)
{
   if (std::isnan(residue)) return false;
   if (residue > div && it > minit) return false;
   if (it >= maxit) return false;
   if (residue > conv) return false;
   return true;
}

namespace {

// ----------------------------------------------------------- diagonal
// d_i = A(i,i) by a search of row i's slots (getElement semantics: 0 if absent).
template <typename Real>
__global__ void k_diag(SegView v, const int32_t* __restrict__ cols, const Real* __restrict__ vals, Real* __restrict__ d)
{
   const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   if (i >= v.n) return;
   Real val = 0;
   for (int32_t k = 0;; k++) {
      const int64_t g = global_index_of(v, (int32_t)i, k);
      if (g < 0) break;
      if (cols[g] == i) {
         val = vals[g];
         break;
      }
   }
   d[i] = val;
}

template <typename To, typename From>
__global__ void k_convert(int64_t n, const From* __restrict__ a, To* __restrict__ b)
{
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
      b[i] = (To)a[i];
}

// ------------------------------------------------------------------ CG
// normb = ||M^-1 b|| (Jacobi) or ||b||
template <typename Real>
__global__ void __launch_bounds__(kRedThreads) k_normb(int64_t n, const Real* __restrict__ b, const Real* __restrict__ d,
                                                       RedWork w, DevState* S)
{
   double acc = 0;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
      const double v = d ? (double)(b[i] / d[i]) : (double)b[i];
      acc += v * v;
   }
   double v[1] = {acc};
   if (publish_and_arrive<1>(v, w)) {
      double t[1];
      gather_totals<1>(t, w);
      if (threadIdx.x == 0) S->normb = sqrt(t[0]);
   }
}

// z = M^-1 r; p = z; s1 = (r, z); residue; nextIteration.
template <typename Real>
__global__ void __launch_bounds__(kRedThreads) k_cg_init(int64_t n, const Real* __restrict__ r, Real* __restrict__ z,
                                                         Real* __restrict__ p, const Real* __restrict__ d, RedWork w,
                                                         DevState* S)
{
   double acc = 0;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
      const Real ri = r[i];
      const Real zi = d ? ri / d[i] : ri;
      if (d) z[i] = zi;
      p[i] = zi;
      acc += (double)ri * (double)zi;
   }
   double v[1] = {acc};
   if (publish_and_arrive<1>(v, w)) {
      double t[1];
      gather_totals<1>(t, w);
      if (threadIdx.x == 0) {
         DevState s = *S;
         s.s1 = t[0];
         s.residue = sqrt(s.s1) / s.normb;
         s.it = 0;
         s.done = 0;
         s.flag = 0;
         next_iteration(s);
         *S = s;
      }
   }
}

// s2 = (Ap, p); s2 == 0 -> residue 0 and stop (CG.hpp:64-68); alpha = s1/s2.
template <typename Real>
__global__ void __launch_bounds__(kRedThreads) k_cg_s2(int64_t n, const Real* __restrict__ Ap, const Real* __restrict__ p,
                                                       RedWork w, DevState* S)
{
   if (S->done) return;
   double acc = 0;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
      acc += (double)Ap[i] * (double)p[i];
   double v[1] = {acc};
   if (publish_and_arrive<1>(v, w)) {
      double t[1];
      gather_totals<1>(t, w);
      if (threadIdx.x == 0) {
         S->s2 = t[0];
         if (t[0] == 0.0) {
            S->residue = 0.0;
            S->done = 1;
            S->flag = 1;
         }
         else
            S->alpha = S->s1 / t[0];
      }
   }
}

// s2 = (p, Ap) from the fused product's sum; alpha = s1 / s2 (the epilogue
// of k_cg_s2).
__global__ void k_cg_alpha(const double* __restrict__ s2, DevState* S)
{
   if (S->done || threadIdx.x != 0) return;
   const double t = *s2;
   S->s2 = t;
   if (t == 0.0) {
      S->residue = 0.0;
      S->done = 1;
      S->flag = 1;
   }
   else
      S->alpha = S->s1 / t;
}

// x += alpha p; r -= alpha Ap; z = M^-1 r; s1 = (r, z); beta; residue; nextIteration.
template <typename Real>
__global__ void __launch_bounds__(kRedThreads) k_cg_update(int64_t n, Real* __restrict__ x, Real* __restrict__ r,
                                                           const Real* __restrict__ p, const Real* __restrict__ Ap,
                                                           Real* __restrict__ z, const Real* __restrict__ d, RedWork w,
                                                           DevState* S)
{
   if (S->done) return;
   const Real alpha = (Real)S->alpha;
   double acc = 0;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
      x[i] += alpha * p[i];
      const Real ri = r[i] - alpha * Ap[i];
      r[i] = ri;
      Real zi = ri;
      if (d) {
         zi = ri / d[i];
         z[i] = zi;
      }
      acc += (double)ri * (double)zi;
   }
   double v[1] = {acc};
   if (publish_and_arrive<1>(v, w)) {
      double t[1];
      gather_totals<1>(t, w);
      if (threadIdx.x == 0) {
         DevState s = *S;
         s.s2 = s.s1;
         s.s1 = t[0];
         s.beta = (s.s2 == 0.0) ? 0.0 : s.s1 / s.s2;
         s.residue = sqrt(s.s1) / s.normb;
         next_iteration(s);
         *S = s;
      }
   }
}

// x += alpha p; r -= alpha Ap (z and (r, z) follow after M^-1 is applied).
template <typename Real>
__global__ void k_cg_xr(int64_t n, Real* __restrict__ x, Real* __restrict__ r, const Real* __restrict__ p,
                        const Real* __restrict__ Ap, const DevState* S)
{
   if (S->done) return;
   const Real alpha = (Real)S->alpha;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
      x[i] += alpha * p[i];
      r[i] -= alpha * Ap[i];
   }
}

// s1 = (r, z) after z = M^-1 r; beta; residue; nextIteration.  With
// `init`, also p = z and the first nextIteration of the solve.
template <typename Real>
__global__ void __launch_bounds__(kRedThreads) k_cg_rz(int64_t n, const Real* __restrict__ r,
                                                       const Real* __restrict__ z, Real* __restrict__ p, int init,
                                                       RedWork w, DevState* S)
{
   if (!init && S->done) return;
   double acc = 0;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
      if (init) p[i] = z[i];
      acc += (double)r[i] * (double)z[i];
   }
   double v[1] = {acc};
   if (publish_and_arrive<1>(v, w)) {
      double t[1];
      gather_totals<1>(t, w);
      if (threadIdx.x == 0) {
         DevState s = *S;
         if (init) {
            s.s1 = t[0];
            s.it = 0;
            s.done = 0;
            s.flag = 0;
         }
         else {
            s.s2 = s.s1;
            s.s1 = t[0];
            s.beta = (s.s2 == 0.0) ? 0.0 : s.s1 / s.s2;
         }
         s.residue = sqrt(s.s1) / s.normb;
         next_iteration(s);
         *S = s;
      }
   }
}

// p = z + beta p (the beta of this iteration; skipped once stopped).
template <typename Real>
__global__ void k_cg_p(int64_t n, Real* __restrict__ p, const Real* __restrict__ z, const DevState* S, int32_t it_expected)
{
   // The update belongs to iteration it_expected; if the state moved past
   // the stop, p is no longer needed.
   if (S->done) return;
   const Real beta = (Real)S->beta;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
      p[i] = z[i] + beta * p[i];
}

// ---------------------------------------------------- generic vector ops

template <typename Real>
__global__ void k_axpby(int64_t n, Real a, const Real* __restrict__ x, Real b, Real* __restrict__ y)
{
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
      y[i] = a * x[i] + b * y[i];
}

// out = M^-1 in (Jacobi) or copy
template <typename Real>
__global__ void k_jacobi(int64_t n, const Real* __restrict__ in, const Real* __restrict__ d, Real* __restrict__ out)
{
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
      out[i] = d ? in[i] / d[i] : in[i];
}

// Up to two dot products into slots of DevState-external results.
template <typename Real>
__global__ void __launch_bounds__(kRedThreads) k_dots(int64_t n, const Real* __restrict__ a0, const Real* __restrict__ b0,
                                                      const Real* __restrict__ a1, const Real* __restrict__ b1, RedWork w,
                                                      double* __restrict__ out)
{
   double acc0 = 0, acc1 = 0;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
      acc0 += (double)a0[i] * (double)b0[i];
      if (a1) acc1 += (double)a1[i] * (double)b1[i];
   }
   double v[2] = {acc0, acc1};
   if (publish_and_arrive<2>(v, w)) {
      double t[2];
      gather_totals<2>(t, w);
      if (threadIdx.x == 0) {
         out[0] = t[0];
         out[1] = t[1];
      }
   }
}

// ------------------------------------------------------------- BiCGStab

// x += alpha p + omega s; r = s - omega As; dots (r, r_ast), (r, r)
template <typename Real>
__global__ void __launch_bounds__(kRedThreads) k_bicg_xr(int64_t n, Real* __restrict__ x, Real* __restrict__ r,
                                                         const Real* __restrict__ p, const Real* __restrict__ s,
                                                         const Real* __restrict__ As, const Real* __restrict__ r_ast,
                                                         Real alpha, Real omega, RedWork w, double* __restrict__ out)
{
   double acc0 = 0, acc1 = 0;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
      x[i] += alpha * p[i] + omega * s[i];
      const Real ri = s[i] - omega * As[i];
      r[i] = ri;
      acc0 += (double)ri * (double)r_ast[i];
      acc1 += (double)ri * (double)ri;
   }
   double v[2] = {acc0, acc1};
   if (publish_and_arrive<2>(v, w)) {
      double t[2];
      gather_totals<2>(t, w);
      if (threadIdx.x == 0) {
         out[0] = t[0];
         out[1] = t[1];
      }
   }
}

// p = r + beta p - (beta omega) Ap
template <typename Real>
__global__ void k_bicg_p(int64_t n, Real* __restrict__ p, const Real* __restrict__ r, const Real* __restrict__ Ap,
                         Real beta, Real bo)
{
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
      p[i] = r[i] + beta * p[i] - bo * Ap[i];
}

// ---------------------------------------------------------------- GMRES

// H_l[k] = (V_k, w) for k <= i: one block-row pass over V; per-block
// partials then the last block sums them (deterministic).
template <typename Real>
__global__ void __launch_bounds__(kRedThreads) k_gmres_vtw(int64_t n, int64_t ld, int cols, const Real* __restrict__ V,
                                                           const Real* __restrict__ w, double* __restrict__ partials,
                                                           unsigned* counter, double* __restrict__ out)
{
   // partials layout: [col][block]
   __shared__ bool s_last;
   for (int k = 0; k < cols; k++) {
      double acc = 0;
      const Real* vk = V + (int64_t)k * ld;
      for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
         acc += (double)vk[i] * (double)w[i];
      acc = block_sum(acc);
      if (threadIdx.x == 0) partials[(int64_t)k * kRedMaxBlocks + blockIdx.x] = acc;
   }
   if (threadIdx.x == 0) {
      __threadfence();
      s_last = atomicAdd(counter, 1u) == gridDim.x - 1;
   }
   __syncthreads();
   if (!s_last) return;
   for (int k = 0; k < cols; k++) {
      double v = 0;
      for (unsigned b = threadIdx.x; b < gridDim.x; b += kRedThreads) v += __ldcg(partials + (int64_t)k * kRedMaxBlocks + b);
      v = block_sum(v);
      if (threadIdx.x == 0) out[k] = v;
   }
   if (threadIdx.x == 0) *counter = 0;
}

// w = w - V h (h on the device, cols entries), optional norm of the result.
template <typename Real>
__global__ void __launch_bounds__(kRedThreads) k_gmres_wmvh(int64_t n, int64_t ld, int cols, const Real* __restrict__ V,
                                                            const double* __restrict__ h, Real* __restrict__ w,
                                                            RedWork red, double* __restrict__ norm_out)
{
   __shared__ double sh[64];
   if (threadIdx.x < cols && threadIdx.x < 64) sh[threadIdx.x] = h[threadIdx.x];
   __syncthreads();
   double acc = 0;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
      Real s = w[i];
      for (int k = 0; k < cols; k++) s -= (Real)sh[k] * V[(int64_t)k * ld + i];
      w[i] = s;
      acc += (double)s * (double)s;
   }
   if (!norm_out) return;
   double v[1] = {acc};
   if (publish_and_arrive<1>(v, red)) {
      double t[1];
      gather_totals<1>(t, red);
      if (threadIdx.x == 0) *norm_out = sqrt(t[0]);
   }
}

// w -= h[0] v (one MGS step), with (w_new, v_next) for the next step.
template <typename Real>
__global__ void __launch_bounds__(kRedThreads) k_mgs_step(int64_t n, const Real* __restrict__ v, const double* __restrict__ h,
                                                          Real* __restrict__ w, const Real* __restrict__ vnext,
                                                          RedWork red, double* __restrict__ out)
{
   const Real hk = h ? (Real)h[0] : Real(0);
   double acc = 0;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
      Real wi = w[i];
      if (h) wi = wi - hk * v[i];
      w[i] = wi;
      acc += vnext ? (double)wi * (double)vnext[i] : (double)wi * (double)wi;
   }
   double vv[1] = {acc};
   if (publish_and_arrive<1>(vv, red)) {
      double t[1];
      gather_totals<1>(t, red);
      if (threadIdx.x == 0) out[0] = vnext ? t[0] : sqrt(t[0]);
   }
}

// x += a * d (FP64 solution, FP32 correction)
__global__ void k_axpby_mixed(int64_t n, double a, const float* __restrict__ d, double* __restrict__ x)
{
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
      x[i] += a * (double)d[i];
}

// dst = scale * src
template <typename Real>
__global__ void k_scale(int64_t n, Real scale, const Real* __restrict__ src, Real* __restrict__ dst)
{
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
      dst[i] = scale * src[i];
}

// x += V y (y on the device, k+1 entries)
template <typename Real>
__global__ void k_gmres_update(int64_t n, int64_t ld, int cols, const Real* __restrict__ V, const double* __restrict__ y,
                               Real* __restrict__ x)
{
   __shared__ double sy[64];
   if (threadIdx.x < cols && threadIdx.x < 64) sy[threadIdx.x] = y[threadIdx.x];
   __syncthreads();
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
      double acc = 0;
      for (int k = 0; k < cols; k++) acc += (double)V[(int64_t)k * ld + i] * sy[k];
      x[i] = (Real)(acc + (double)x[i]);
   }
}

// out = alpha * Y c + beta * in (in == nullptr: beta term absent), then
// out[unit_row] = 1 + out[unit_row] when unit_row >= 0 -- the gemv of
// MatrixOperations::gemv (Matrices/MatrixOperations.h) as the CWY steps use
// it; c has `cols` <= 128 entries on the device, alpha applied to c first.
template <typename Real>
__global__ void k_gemv_cols(int64_t n, int64_t ld, int cols, const Real* __restrict__ Y, const double* __restrict__ c,
                            double alpha, const Real* in, double beta, Real* out, int64_t unit_row)
{
   __shared__ double sc[128];
   if (threadIdx.x < cols && threadIdx.x < 128) sc[threadIdx.x] = alpha * c[threadIdx.x];
   __syncthreads();
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
      double acc = 0;
      for (int k = 0; k < cols; k++) acc += (double)Y[(int64_t)k * ld + i] * sc[k];
      Real v = in ? (Real)(acc + beta * (double)in[i]) : (Real)acc;
      if (i == unit_row) v = (Real)1 + v;
      out[i] = v;
   }
}

// y_i = z with the entries above row i set to zero (hauseholder_generate)
template <typename Real>
__global__ void k_truncate(int64_t n, int64_t i0, const Real* __restrict__ z, Real* __restrict__ y)
{
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
      y[i] = i < i0 ? Real(0) : z[i];
}

// x[j] = x[j] + y[j] for j < k (the CWY update's x += sum_j y_j e_j)
template <typename Real>
__global__ void k_add_head(int k, const double* __restrict__ y, Real* __restrict__ x)
{
   const int j = threadIdx.x;
   if (j < k) x[j] = x[j] + (Real)y[j];
}

}  // namespace

// ------------------------------------------------------------------ host

tnlb_status spmv_dispatch(const tnlb_segments* seg, tnlb_real real, const int32_t* cols, const void* vals, const void* x,
                          void* y, double alpha, double beta, cudaStream_t st, const int32_t* skip)
{
   int launches = 0;
   if (seg->format == TNLB_CSR || seg->format == TNLB_ADAPTIVE_CSR)
      return spmv_csr(seg, real, cols, vals, x, y, alpha, beta, 0, seg->n,
                      seg->format == TNLB_ADAPTIVE_CSR ? TNLB_KERNEL_ADAPTIVE : TNLB_KERNEL_DEFAULT, 0, st, &launches,
                      seg->format == TNLB_CSR ? skip : nullptr);
   return spmv_ell_family(seg, real, cols, vals, x, y, alpha, beta, 0, seg->n, TNLB_KERNEL_DEFAULT, 0, st, &launches);
}

namespace {

// Preconditioner view for one real type over a tnlb_precond object.
template <typename Real>
struct Precond {
   const tnlb_precond* obj = nullptr;
   int kind = TNLB_PRECOND_NONE;
   const Real* d() const { return kind == TNLB_PRECOND_JACOBI ? obj->diag.as<Real>() : nullptr; }
   // true when M^-1 is applied by separate kernels (FSAI: two SpMVs)
   bool general() const { return kind == TNLB_PRECOND_FSAI; }
   // out = M^-1 in (`skip`: the solver's done flag, for kernels in graphs)
   tnlb_status apply(int64_t n, const Real* in, Real* out, cudaStream_t st, const int32_t* skip = nullptr) const
   {
      if (kind == TNLB_PRECOND_ILU0 || kind == TNLB_PRECOND_ILUT) return ilu0_apply(obj->ilu, in, out, st);
      if (kind == TNLB_PRECOND_FSAI) return fsai_apply(obj->fsai, in, out, st, skip);
      k_jacobi<Real><<<vec_grid(n), kRedThreads, 0, st>>>(n, in, d(), out);
      TNLB_CHECK_LAUNCH();
      return TNLB_OK;
   }
};

template <typename Real>
Precond<Real> view(const tnlb_precond* P)
{
   Precond<Real> v;
   v.obj = P;
   v.kind = P ? P->kind : TNLB_PRECOND_NONE;
   return v;
}

struct Work {
   DeviceBuffer state, partials, counter, scratch;
   tnlb_status alloc()
   {
      TNLB_TRY_STATUS(state.alloc(sizeof(DevState)));
      TNLB_TRY_STATUS(partials.alloc(sizeof(double) * kRedMaxBlocks * 64));
      TNLB_TRY_STATUS(counter.alloc(sizeof(unsigned) * 4));
      TNLB_TRY_STATUS(scratch.alloc(sizeof(double) * 256));
      TNLB_CUDA_TRY(cudaMemset(counter.ptr, 0, sizeof(unsigned) * 4));
      return TNLB_OK;
   }
   RedWork red() const { return {partials.as<double>(), counter.as<unsigned>()}; }
   DevState* S() const { return state.as<DevState>(); }
};

// The iteration graph of a solver, captured on stream s: preferably a
// conditional WHILE node whose body is body(s) followed by cont(loop, s), a
// one-thread kernel that sets the loop's condition, so that the device
// repeats the body with no host round trip; where the driver cannot build
// that node, body(s) alone. Returns whether the graph loops. When capture
// fails both ways, *exec stays null and the caller launches the body's
// kernels directly.
template <typename Body, typename Cont>
bool build_iteration_graph(cudaStream_t s, Body&& body, Cont&& cont, cudaGraph_t* graph, cudaGraphExec_t* exec)
{
   *graph = nullptr;
   *exec = nullptr;
   if (cudaGraphCreate(graph, 0) == cudaSuccess) {
      cudaGraphConditionalHandle loop{};
      cudaGraphNodeParams np{};
      np.type = cudaGraphNodeTypeConditional;
      cudaGraphNode_t node = nullptr;
      bool ok = cudaGraphConditionalHandleCreate(&loop, *graph, 1, cudaGraphCondAssignDefault) == cudaSuccess;
      if (ok) {
         np.conditional.handle = loop;
         np.conditional.type = cudaGraphCondTypeWhile;
         np.conditional.size = 1;
         ok = cudaGraphAddNode(&node, *graph, nullptr, 0, &np) == cudaSuccess;
      }
      if (ok)
         ok = cudaStreamBeginCaptureToGraph(s, np.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                            cudaStreamCaptureModeThreadLocal) == cudaSuccess;
      if (ok) {
         const tnlb_status rc = body(s);
         if (rc == TNLB_OK) cont(loop, s);
         cudaGraph_t captured = nullptr;
         ok = cudaStreamEndCapture(s, &captured) == cudaSuccess && rc == TNLB_OK &&
              cudaGetLastError() == cudaSuccess && cudaGraphInstantiate(exec, *graph, 0) == cudaSuccess;
      }
      clear_error();
      if (ok) return true;
      cudaGetLastError();
      if (*exec) cudaGraphExecDestroy(*exec);
      cudaGraphDestroy(*graph);
      *exec = nullptr;
      *graph = nullptr;
   }
   else
      cudaGetLastError();
   if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
      const tnlb_status rc = body(s);
      cudaError_t e = cudaStreamEndCapture(s, graph);
      if (e == cudaSuccess && rc == TNLB_OK) e = cudaGraphInstantiate(exec, *graph, 0);
      if (e != cudaSuccess) {
         cudaGetLastError();
         *exec = nullptr;
      }
      clear_error();
   }
   else
      cudaGetLastError();
   return false;
}

// Last node of CG's looping batch body: run the body again until the state
// is done, at most `cap` bodies per launch, after which the host reads the
// state and launches again. The counter restarts at each exit, and a counter
// found at `cap` or above ends the loop at once.
__global__ void k_cg_continue(cudaGraphConditionalHandle loop, DevState* S, uint32_t cap)
{
   if (threadIdx.x != 0) return;
   const uint32_t l = S->loops + 1u;
   const bool go = !S->done && l < cap;
   S->loops = go ? l : 0u;
   cudaGraphSetConditional(loop, go ? 1u : 0u);
}

DevState initial_state(const tnlb_solver_params& p)
{
   DevState s{};
   s.conv = p.convergence_residue;
   s.div = p.divergence_residue;
   s.maxit = p.max_iterations;
   s.minit = p.min_iterations;
   return s;
}

template <typename Real>
struct Ctx {
   const tnlb_segments* seg;
   tnlb_real real;
   const int32_t* cols;
   const Real* vals;
   int64_t n;
   cudaStream_t st;
   tnlb_status spmv(const Real* x, Real* y, double alpha = 1.0, double beta = 0.0) const
   {
      return spmv_dispatch(seg, real, cols, vals, x, y, alpha, beta, st);
   }
};

// ------------------------------------------------------------------ CG

template <typename Real>
tnlb_status cg_solve(const Ctx<Real>& c, const Precond<Real>& P, const tnlb_solver_params& prm, const Real* b, Real* x,
                     tnlb_solve_result* res)
{
   const int64_t n = c.n;
   Work W;
   TNLB_TRY_STATUS(W.alloc());
   DeviceBuffer r, p, Ap, z;
   TNLB_TRY_STATUS(r.alloc(sizeof(Real) * n));
   TNLB_TRY_STATUS(p.alloc(sizeof(Real) * n));
   TNLB_TRY_STATUS(Ap.alloc(sizeof(Real) * n));
   TNLB_TRY_STATUS(z.alloc(sizeof(Real) * n));
   DevState s0 = initial_state(prm);
   TNLB_CUDA_TRY(cudaMemcpyAsync(W.S(), &s0, sizeof(s0), cudaMemcpyHostToDevice, c.st));
   const unsigned G = vec_grid(n);
   const bool gen = P.general();
   const int32_t* done = &W.S()->done;
   // normb = ||M^-1 b|| (CG.hpp:24-29)
   if (gen) {
      TNLB_TRY_STATUS(P.apply(n, b, z.as<Real>(), c.st));
      k_normb<Real><<<G, kRedThreads, 0, c.st>>>(n, z.as<Real>(), nullptr, W.red(), W.S());
   }
   else
      k_normb<Real><<<G, kRedThreads, 0, c.st>>>(n, b, P.d(), W.red(), W.S());
   TNLB_CHECK_LAUNCH();
   DevState h{};
   TNLB_CUDA_TRY(cudaMemcpyAsync(&h, W.S(), sizeof(h), cudaMemcpyDeviceToHost, c.st));
   TNLB_CUDA_TRY(cudaStreamSynchronize(c.st));
   if (h.normb == 0) {
      TNLB_CUDA_TRY(cudaMemsetAsync(x, 0, sizeof(Real) * n, c.st));
      TNLB_CUDA_TRY(cudaStreamSynchronize(c.st));
      *res = tnlb_solve_result{1, 0, 0.0, 0, 0};
      return TNLB_OK;
   }
   // r = b - A x; z = M^-1 r; p = z; s1 = (r, z); first nextIteration
   TNLB_CUDA_TRY(cudaMemcpyAsync(r.ptr, b, sizeof(Real) * n, cudaMemcpyDeviceToDevice, c.st));
   TNLB_TRY_STATUS(c.spmv(x, r.as<Real>(), -1.0, 1.0));
   Real* zp = (P.kind == TNLB_PRECOND_NONE) ? nullptr : z.as<Real>();
   if (gen) {
      TNLB_TRY_STATUS(P.apply(n, r.as<Real>(), z.as<Real>(), c.st));
      k_cg_rz<Real><<<G, kRedThreads, 0, c.st>>>(n, r.as<Real>(), z.as<Real>(), p.as<Real>(), 1, W.red(), W.S());
   }
   else
      k_cg_init<Real><<<G, kRedThreads, 0, c.st>>>(n, r.as<Real>(), z.as<Real>(), p.as<Real>(), P.d(), W.red(), W.S());
   TNLB_CHECK_LAUNCH();
   // One iteration (CG.hpp:60-107): every kernel returns at once when the
   // device `done` flag is set, so batches may run past the stopping point.
   // short-row CSR: (p, Ap) summed inside the product's kernel
   const bool fused = spmv_dot_fusable(c.seg);
   DeviceBuffer dot_parts, dot_ctr, dot_val;
   if (fused) {
      TNLB_TRY_STATUS(dot_parts.alloc(sizeof(double) * spmv_dot_partials(c.seg)));
      TNLB_TRY_STATUS(dot_ctr.alloc(sizeof(unsigned)));
      TNLB_TRY_STATUS(dot_val.alloc(sizeof(double)));
      TNLB_CUDA_TRY(cudaMemsetAsync(dot_ctr.ptr, 0, sizeof(unsigned), c.st));
   }
   const unsigned Gs2 = resident_grid((const void*)k_cg_s2<Real>, kRedThreads, n, 4);
   const unsigned Gxr = resident_grid((const void*)k_cg_xr<Real>, kRedThreads, n, 4);
   const unsigned Grz = resident_grid((const void*)k_cg_rz<Real>, kRedThreads, n, 4);
   const unsigned Gup = resident_grid((const void*)k_cg_update<Real>, kRedThreads, n, 4);
   const unsigned Gp = resident_grid((const void*)k_cg_p<Real>, kRedThreads, n, 4);
   auto enqueue_iteration = [&](cudaStream_t st) -> tnlb_status {
      if (fused) {
         TNLB_TRY_STATUS(spmv_dot(c.seg, c.real, c.cols, c.vals, p.as<Real>(), Ap.as<Real>(), dot_parts.as<double>(),
                                  dot_ctr.as<unsigned>(), dot_val.as<double>(), st, done));
         k_cg_alpha<<<1, 32, 0, st>>>(dot_val.as<double>(), W.S());
      }
      else {
         TNLB_TRY_STATUS(
            spmv_dispatch(c.seg, c.real, c.cols, c.vals, p.as<Real>(), Ap.as<Real>(), 1.0, 0.0, st, done));
         k_cg_s2<Real><<<Gs2, kRedThreads, 0, st>>>(n, Ap.as<Real>(), p.as<Real>(), W.red(), W.S());
      }
      if (gen) {
         k_cg_xr<Real><<<Gxr, kRedThreads, 0, st>>>(n, x, r.as<Real>(), p.as<Real>(), Ap.as<Real>(), W.S());
         TNLB_TRY_STATUS(P.apply(n, r.as<Real>(), z.as<Real>(), st, done));
         k_cg_rz<Real><<<Grz, kRedThreads, 0, st>>>(n, r.as<Real>(), z.as<Real>(), nullptr, 0, W.red(), W.S());
      }
      else
         k_cg_update<Real><<<Gup, kRedThreads, 0, st>>>(n, x, r.as<Real>(), p.as<Real>(), Ap.as<Real>(), zp, P.d(),
                                                        W.red(), W.S());
      k_cg_p<Real><<<Gp, kRedThreads, 0, st>>>(n, p.as<Real>(), zp ? zp : r.as<Real>(), W.S(), 0);
      TNLB_CHECK_LAUNCH();
      return TNLB_OK;
   };
   // Batches of iterations replayed from a CUDA graph (captured on a side
   // stream), looped on the device up to kCap batches per launch where the
   // driver builds the conditional node.
   const int kBatch = n < (1 << 22) ? 32 : 8;
   constexpr uint32_t kCap = 64;
   cudaStream_t cs;
   TNLB_CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
   cudaEvent_t ev;
   TNLB_CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
   TNLB_CUDA_TRY(cudaEventRecord(ev, c.st));
   TNLB_CUDA_TRY(cudaStreamWaitEvent(cs, ev, 0));
   cudaGraph_t graph = nullptr;
   cudaGraphExec_t exec = nullptr;
   tnlb_status status = TNLB_OK;
   // a failed capture falls back to direct launches
   build_iteration_graph(
      cs,
      [&](cudaStream_t s) {
         tnlb_status rc = TNLB_OK;
         for (int k = 0; k < kBatch && rc == TNLB_OK; k++) rc = enqueue_iteration(s);
         return rc;
      },
      [&](cudaGraphConditionalHandle loop, cudaStream_t s) { k_cg_continue<<<1, 32, 0, s>>>(loop, W.S(), kCap); },
      &graph, &exec);
   // One launch stays queued ahead of the host's check of the state (a launch
   // after the stop runs one batch that returns at once, kernel by kernel).
   DevState* hs = nullptr;
   cudaEvent_t copied = nullptr;
   auto launch_batch = [&]() {
      if (exec) {
         if (cudaGraphLaunch(exec, cs) != cudaSuccess) {
            set_error("CG: graph launch failed");
            status = TNLB_ERR_CUDA;
         }
      }
      else
         for (int k = 0; k < kBatch && status == TNLB_OK; k++) status = enqueue_iteration(cs);
   };
   if (cudaMallocHost(&hs, sizeof(DevState)) != cudaSuccess ||
       cudaEventCreateWithFlags(&copied, cudaEventDisableTiming) != cudaSuccess) {
      set_error("CG: pinned state allocation failed");
      status = TNLB_ERR_CUDA;
   }
   if (status == TNLB_OK) {
      launch_batch();
      cudaMemcpyAsync(hs, W.S(), sizeof(DevState), cudaMemcpyDeviceToHost, cs);
      cudaEventRecord(copied, cs);
   }
   while (status == TNLB_OK) {
      launch_batch();
      if (cudaEventSynchronize(copied) != cudaSuccess) {
         set_error("CG: state read failed");
         status = TNLB_ERR_CUDA;
         break;
      }
      h = *hs;
      if (h.done) break;
      cudaMemcpyAsync(hs, W.S(), sizeof(DevState), cudaMemcpyDeviceToHost, cs);
      cudaEventRecord(copied, cs);
   }
   cudaStreamSynchronize(cs);
   if (hs) cudaFreeHost(hs);
   if (copied) cudaEventDestroy(copied);
   if (exec) cudaGraphExecDestroy(exec);
   if (graph) cudaGraphDestroy(graph);
   cudaEventDestroy(ev);
   cudaStreamDestroy(cs);
   TNLB_TRY_STATUS(status);
   res->iterations = h.it;
   res->residue = h.residue;
   res->converged = check_convergence(h.residue, h.it, h.maxit, h.minit, h.conv, h.div);
   res->status_detail = 0;
   return TNLB_OK;
}

// CG with a general preconditioner applied by a separate call (ILU(0)).
template <typename Real>
tnlb_status pcg_general(const Ctx<Real>& c, const Precond<Real>& P, const tnlb_solver_params& prm, const Real* b,
                        Real* x, tnlb_solve_result* res)
{
   const int64_t n = c.n;
   Work W;
   TNLB_TRY_STATUS(W.alloc());
   DeviceBuffer r, p, Ap, z;
   TNLB_TRY_STATUS(r.alloc(sizeof(Real) * n));
   TNLB_TRY_STATUS(p.alloc(sizeof(Real) * n));
   TNLB_TRY_STATUS(Ap.alloc(sizeof(Real) * n));
   TNLB_TRY_STATUS(z.alloc(sizeof(Real) * n));
   double* sc = W.scratch.as<double>();
   const unsigned G = vec_grid(n);
   double hs[2];
   auto dot = [&](const Real* a, const Real* bb, double* out) -> tnlb_status {
      k_dots<Real><<<G, kRedThreads, 0, c.st>>>(n, a, bb, nullptr, nullptr, W.red(), sc);
      TNLB_CHECK_LAUNCH();
      TNLB_CUDA_TRY(cudaMemcpyAsync(hs, sc, sizeof(hs), cudaMemcpyDeviceToHost, c.st));
      TNLB_CUDA_TRY(cudaStreamSynchronize(c.st));
      *out = hs[0];
      return TNLB_OK;
   };
   int it = 0;
   double residue = 0;
   auto check = [&]() {
      return !(std::isnan(residue) || it > prm.max_iterations ||
               (residue > prm.divergence_residue && it >= prm.min_iterations) ||
               (residue < prm.convergence_residue && it >= prm.min_iterations));
   };
   auto next = [&]() {
      const bool cnt = check();
      it++;
      return cnt;
   };
   double normb;
   TNLB_TRY_STATUS(P.apply(n, b, r.as<Real>(), c.st));
   TNLB_TRY_STATUS(dot(r.as<Real>(), r.as<Real>(), &normb));
   normb = std::sqrt(normb);
   if (normb == 0) {
      TNLB_CUDA_TRY(cudaMemsetAsync(x, 0, sizeof(Real) * n, c.st));
      *res = tnlb_solve_result{1, 0, 0.0, 0, 0};
      return TNLB_OK;
   }
   TNLB_CUDA_TRY(cudaMemcpyAsync(r.ptr, b, sizeof(Real) * n, cudaMemcpyDeviceToDevice, c.st));
   TNLB_TRY_STATUS(c.spmv(x, r.as<Real>(), -1.0, 1.0));
   TNLB_TRY_STATUS(P.apply(n, r.as<Real>(), z.as<Real>(), c.st));
   TNLB_CUDA_TRY(cudaMemcpyAsync(p.ptr, z.ptr, sizeof(Real) * n, cudaMemcpyDeviceToDevice, c.st));
   double s1, s2;
   TNLB_TRY_STATUS(dot(r.as<Real>(), z.as<Real>(), &s1));
   residue = std::sqrt(s1) / normb;
   while (next()) {
      TNLB_TRY_STATUS(c.spmv(p.as<Real>(), Ap.as<Real>()));
      TNLB_TRY_STATUS(dot(Ap.as<Real>(), p.as<Real>(), &s2));
      if (s2 == 0.0) {
         residue = 0;
         break;
      }
      const double alpha = s1 / s2;
      k_axpby<Real><<<G, kRedThreads, 0, c.st>>>(n, (Real)alpha, p.as<Real>(), Real(1), x);
      k_axpby<Real><<<G, kRedThreads, 0, c.st>>>(n, (Real)-alpha, Ap.as<Real>(), Real(1), r.as<Real>());
      TNLB_CHECK_LAUNCH();
      TNLB_TRY_STATUS(P.apply(n, r.as<Real>(), z.as<Real>(), c.st));
      s2 = s1;
      TNLB_TRY_STATUS(dot(r.as<Real>(), z.as<Real>(), &s1));
      const double beta = (s2 == 0.0) ? 0.0 : s1 / s2;
      k_axpby<Real><<<G, kRedThreads, 0, c.st>>>(n, Real(1), z.as<Real>(), (Real)beta, p.as<Real>());
      TNLB_CHECK_LAUNCH();
      residue = std::sqrt(s1) / normb;
   }
   TNLB_CUDA_TRY(cudaStreamSynchronize(c.st));
   res->iterations = it;
   res->residue = residue;
   res->converged = check_convergence(residue, it, prm.max_iterations, prm.min_iterations, prm.convergence_residue,
                                      prm.divergence_residue);
   res->status_detail = 0;
   return TNLB_OK;
}

// ------------------------------------------------------------ BiCGStab

template <typename Real>
tnlb_status bicgstab_solve(const Ctx<Real>& c, const Precond<Real>& P, const tnlb_solver_params& prm, const Real* b,
                           Real* x, tnlb_solve_result* res)
{
   const int64_t n = c.n;
   Work W;
   TNLB_TRY_STATUS(W.alloc());
   DeviceBuffer r, r_ast, p, s, Ap, As, M_tmp;
   for (auto* v : {&r, &r_ast, &p, &s, &Ap, &As, &M_tmp}) TNLB_TRY_STATUS(v->alloc(sizeof(Real) * n));
   double* sc = W.scratch.as<double>();
   const unsigned G = vec_grid(n);
   double hs[2];
   auto dots = [&](const Real* a0, const Real* b0, const Real* a1, const Real* b1) -> tnlb_status {
      k_dots<Real><<<G, kRedThreads, 0, c.st>>>(n, a0, b0, a1, b1, W.red(), sc);
      TNLB_CHECK_LAUNCH();
      TNLB_CUDA_TRY(cudaMemcpyAsync(hs, sc, sizeof(hs), cudaMemcpyDeviceToHost, c.st));
      TNLB_CUDA_TRY(cudaStreamSynchronize(c.st));
      return TNLB_OK;
   };
   const bool pre = P.kind != TNLB_PRECOND_NONE;
   // compute_residue: r = M^-1 (b - A x) (BICGStab.hpp:125-138)
   auto compute_residue = [&](Real* out) -> tnlb_status {
      Real* tgt = pre ? M_tmp.as<Real>() : out;
      TNLB_CUDA_TRY(cudaMemcpyAsync(tgt, b, sizeof(Real) * n, cudaMemcpyDeviceToDevice, c.st));
      TNLB_TRY_STATUS(c.spmv(x, tgt, -1.0, 1.0));
      if (pre) TNLB_TRY_STATUS(P.apply(n, M_tmp.as<Real>(), out, c.st));
      return TNLB_OK;
   };
   // preconditioned_matvec (:141-151)
   auto pmatvec = [&](const Real* src, Real* dst) -> tnlb_status {
      if (!pre) return c.spmv(src, dst);
      TNLB_TRY_STATUS(c.spmv(src, M_tmp.as<Real>()));
      return P.apply(n, M_tmp.as<Real>(), dst, c.st);
   };
   int it = 0;
   double residue = 0;
   auto check = [&]() {
      return !(std::isnan(residue) || it > prm.max_iterations ||
               (residue > prm.divergence_residue && it >= prm.min_iterations) ||
               (residue < prm.convergence_residue && it >= prm.min_iterations));
   };
   double b_norm;
   if (pre) {
      TNLB_TRY_STATUS(P.apply(n, b, M_tmp.as<Real>(), c.st));
      TNLB_TRY_STATUS(dots(M_tmp.as<Real>(), M_tmp.as<Real>(), nullptr, nullptr));
   }
   else
      TNLB_TRY_STATUS(dots(b, b, nullptr, nullptr));
   b_norm = std::sqrt(hs[0]);
   if (b_norm == 0) {
      TNLB_CUDA_TRY(cudaMemsetAsync(x, 0, sizeof(Real) * n, c.st));
      *res = tnlb_solve_result{1, 0, 0.0, 0, 0};
      return TNLB_OK;
   }
   TNLB_TRY_STATUS(compute_residue(r.as<Real>()));
   TNLB_CUDA_TRY(cudaMemcpyAsync(p.ptr, r.ptr, sizeof(Real) * n, cudaMemcpyDeviceToDevice, c.st));
   TNLB_CUDA_TRY(cudaMemcpyAsync(r_ast.ptr, r.ptr, sizeof(Real) * n, cudaMemcpyDeviceToDevice, c.st));
   TNLB_CUDA_TRY(cudaMemsetAsync(s.ptr, 0, sizeof(Real) * n, c.st));
   TNLB_TRY_STATUS(dots(r.as<Real>(), r_ast.as<Real>(), nullptr, nullptr));
   double rho = hs[0], r_ast_sqnorm = hs[0];
   const double eps2 = DBL_EPSILON * DBL_EPSILON;
   const double eps2r = (sizeof(Real) == 4) ? (double)FLT_EPSILON * FLT_EPSILON : eps2;
   residue = std::sqrt(rho) / b_norm;
   while (true) {
      const bool cont = check();
      it++;
      if (!cont) break;
      TNLB_TRY_STATUS(pmatvec(p.as<Real>(), Ap.as<Real>()));
      TNLB_TRY_STATUS(dots(Ap.as<Real>(), r_ast.as<Real>(), nullptr, nullptr));
      const double alpha = rho / hs[0];
      // s = r - alpha Ap
      TNLB_CUDA_TRY(cudaMemcpyAsync(s.ptr, r.ptr, sizeof(Real) * n, cudaMemcpyDeviceToDevice, c.st));
      k_axpby<Real><<<G, kRedThreads, 0, c.st>>>(n, (Real)-alpha, Ap.as<Real>(), Real(1), s.as<Real>());
      TNLB_CHECK_LAUNCH();
      TNLB_TRY_STATUS(pmatvec(s.as<Real>(), As.as<Real>()));
      TNLB_TRY_STATUS(dots(As.as<Real>(), s.as<Real>(), As.as<Real>(), As.as<Real>()));
      const double omega = hs[0] / hs[1];
      k_bicg_xr<Real><<<G, kRedThreads, 0, c.st>>>(n, x, r.as<Real>(), p.as<Real>(), s.as<Real>(), As.as<Real>(),
                                                   r_ast.as<Real>(), (Real)alpha, (Real)omega, W.red(), sc);
      TNLB_CHECK_LAUNCH();
      TNLB_CUDA_TRY(cudaMemcpyAsync(hs, sc, sizeof(hs), cudaMemcpyDeviceToHost, c.st));
      TNLB_CUDA_TRY(cudaStreamSynchronize(c.st));
      const double rho_old = rho;
      rho = hs[0];
      double rnorm2 = hs[1];
      (void)eps2r;
      if (std::fabs(rho) < eps2 * r_ast_sqnorm) {
         TNLB_TRY_STATUS(compute_residue(r.as<Real>()));
         TNLB_CUDA_TRY(cudaMemcpyAsync(r_ast.ptr, r.ptr, sizeof(Real) * n, cudaMemcpyDeviceToDevice, c.st));
         TNLB_TRY_STATUS(dots(r.as<Real>(), r_ast.as<Real>(), nullptr, nullptr));
         r_ast_sqnorm = rho = hs[0];
         rnorm2 = hs[0];
      }
      const double beta = (rho / rho_old) * (alpha / omega);
      k_bicg_p<Real><<<G, kRedThreads, 0, c.st>>>(n, p.as<Real>(), r.as<Real>(), Ap.as<Real>(), (Real)beta,
                                                  (Real)(beta * omega));
      TNLB_CHECK_LAUNCH();
      if (prm.bicgstab_exact_residue) {
         TNLB_TRY_STATUS(compute_residue(s.as<Real>()));
         TNLB_TRY_STATUS(dots(s.as<Real>(), s.as<Real>(), nullptr, nullptr));
         residue = std::sqrt(hs[0]) / b_norm;
      }
      else
         residue = std::sqrt(rnorm2) / b_norm;
   }
   TNLB_CUDA_TRY(cudaStreamSynchronize(c.st));
   res->iterations = it;
   res->residue = residue;
   res->converged = check_convergence(residue, it, prm.max_iterations, prm.min_iterations, prm.convergence_residue,
                                      prm.divergence_residue);
   res->status_detail = 0;
   return TNLB_OK;
}

// --------------------------------------------------------------- GMRES

// Givens rotations on column i of H (leading dimension m + 1) and on s
// (GMRES::apply_givens_rotations, GMRES.hpp:731-770).
void givens_column(int i, int m, double* H, double* s, double* cs, double* sn)
{
   auto rot = [](double& dx, double& dy, double csv, double snv) {
      const double t = csv * dx + snv * dy;
      dy = csv * dy - snv * dx;
      dx = t;
   };
   for (int k = 0; k < i; k++) rot(H[k + i * (m + 1)], H[k + 1 + i * (m + 1)], cs[k], sn[k]);
   if (H[i + 1 + i * (m + 1)] != 0.0) {
      const double dx = H[i + i * (m + 1)], dy = H[i + 1 + i * (m + 1)];
      if (dy == 0.0) {
         cs[i] = 1.0;
         sn[i] = 0.0;
      }
      else if (std::fabs(dy) > std::fabs(dx)) {
         const double t = dx / dy;
         sn[i] = 1.0 / std::sqrt(1.0 + t * t);
         cs[i] = t * sn[i];
      }
      else {
         const double t = dy / dx;
         cs[i] = 1.0 / std::sqrt(1.0 + t * t);
         sn[i] = t * cs[i];
      }
      rot(H[i + i * (m + 1)], H[i + 1 + i * (m + 1)], cs[i], sn[i]);
      rot(s[i], s[i + 1], cs[i], sn[i]);
   }
}

// GMRES with the CWY orthogonalisation (GMRES.hpp:350-423): Householder
// reflections P_i = I - t_i y_i y_i^T kept in compact WY form I - Y T Y^T.
// Y (n x (m_max+1), column-major, zero above the diagonal) stays on the
// device; T, H, s and the upper (m_max+1) x (m_max+1) block of Y (YL) are
// small and live on the host, as in the reference.  The basis vectors are
// not stored: v_i = (I - Y T Y^T) e_i is rebuilt (hauseholder_cwy :572-604),
// and the update adds sum_j y_j v_j the same way (:685-725).  Each cycle
// counts m+1 iterations (i = 0..m) and makes m products.
template <typename Real>
tnlb_status gmres_cwy_solve(const Ctx<Real>& c, const Precond<Real>& P, const tnlb_solver_params& prm, const Real* b,
                            Real* x, tnlb_solve_result* res)
{
   const int64_t n = c.n;
   const int rmin = prm.gmres_restarting_min, rmax = prm.gmres_restarting_max;
   const int dmin = prm.gmres_restarting_step_min, dmax = prm.gmres_restarting_step_max;
   const int L = rmax + 1;
   TNLB_REQUIRE(n >= L, TNLB_ERR_INVALID_ARGUMENT,
                "GMRES CWY needs at least restarting_max + 1 rows (the reference copies that many entries of Y)");
   const int64_t ld = (n + 31) / 32 * 32;
   Work W;
   TNLB_TRY_STATUS(W.alloc());
   DeviceBuffer Yb, z, w, v, r, M_tmp, hdev, cdev, ydev;
   TNLB_TRY_STATUS(Yb.alloc(sizeof(Real) * ld * L));
   TNLB_TRY_STATUS(z.alloc(sizeof(Real) * n));
   TNLB_TRY_STATUS(w.alloc(sizeof(Real) * n));
   TNLB_TRY_STATUS(v.alloc(sizeof(Real) * n));
   TNLB_TRY_STATUS(r.alloc(sizeof(Real) * n));
   TNLB_TRY_STATUS(M_tmp.alloc(sizeof(Real) * n));
   TNLB_TRY_STATUS(hdev.alloc(sizeof(double) * 128));
   TNLB_TRY_STATUS(cdev.alloc(sizeof(double) * 128));
   TNLB_TRY_STATUS(ydev.alloc(sizeof(double) * 128));
   Real* Y = Yb.as<Real>();
   double* sc = W.scratch.as<double>();
   const unsigned G = vec_grid(n);
   const bool pre = P.kind != TNLB_PRECOND_NONE;
   double hs[2];
   auto norm = [&](const Real* a, double* out) -> tnlb_status {
      k_dots<Real><<<G, kRedThreads, 0, c.st>>>(n, a, a, nullptr, nullptr, W.red(), sc);
      TNLB_CHECK_LAUNCH();
      TNLB_CUDA_TRY(cudaMemcpyAsync(hs, sc, sizeof(hs), cudaMemcpyDeviceToHost, c.st));
      TNLB_CUDA_TRY(cudaStreamSynchronize(c.st));
      *out = std::sqrt(hs[0]);
      return TNLB_OK;
   };
   auto compute_residue = [&]() -> tnlb_status {
      Real* tgt = pre ? M_tmp.as<Real>() : r.as<Real>();
      TNLB_CUDA_TRY(cudaMemcpyAsync(tgt, b, sizeof(Real) * n, cudaMemcpyDeviceToDevice, c.st));
      TNLB_TRY_STATUS(c.spmv(x, tgt, -1.0, 1.0));
      if (pre) TNLB_TRY_STATUS(P.apply(n, M_tmp.as<Real>(), r.as<Real>(), c.st));
      return TNLB_OK;
   };
   // Y_cols^T a -> host (Reduction2D in the reference)
   std::vector<double> aux(L + 1);
   auto ytv = [&](int cols, const Real* a) -> tnlb_status {
      k_gmres_vtw<Real><<<G, kRedThreads, 0, c.st>>>(n, ld, cols, Y, a, W.partials.as<double>(),
                                                    W.counter.as<unsigned>() + 1, hdev.as<double>());
      TNLB_CHECK_LAUNCH();
      TNLB_CUDA_TRY(cudaMemcpyAsync(aux.data(), hdev.ptr, sizeof(double) * cols, cudaMemcpyDeviceToHost, c.st));
      return TNLB_OK;
   };
   // out = alpha * Y_cols aux + beta * in (+ e_unit)
   auto gemv = [&](int cols, double alpha, const Real* in, double beta, Real* out, int64_t unit) -> tnlb_status {
      TNLB_CUDA_TRY(cudaMemcpyAsync(cdev.ptr, aux.data(), sizeof(double) * cols, cudaMemcpyHostToDevice, c.st));
      k_gemv_cols<Real><<<G, kRedThreads, 0, c.st>>>(n, ld, cols, Y, cdev.as<double>(), alpha, in, beta, out, unit);
      TNLB_CHECK_LAUNCH();
      return TNLB_OK;
   };
   int it = 0;
   double residue = 0;
   auto check = [&]() {
      return !(std::isnan(residue) || it > prm.max_iterations ||
               (residue > prm.divergence_residue && it >= prm.min_iterations) ||
               (residue < prm.convergence_residue && it >= prm.min_iterations));
   };
   double normb;
   if (pre) {
      TNLB_TRY_STATUS(P.apply(n, b, M_tmp.as<Real>(), c.st));
      TNLB_TRY_STATUS(norm(M_tmp.as<Real>(), &normb));
   }
   else
      TNLB_TRY_STATUS(norm(b, &normb));
   if (normb == 0) {
      TNLB_CUDA_TRY(cudaMemsetAsync(x, 0, sizeof(Real) * n, c.st));
      TNLB_CUDA_TRY(cudaStreamSynchronize(c.st));
      *res = tnlb_solve_result{1, 0, 0.0, 0, 0};
      return TNLB_OK;
   }
   TNLB_TRY_STATUS(compute_residue());
   double beta;
   TNLB_TRY_STATUS(norm(r.as<Real>(), &beta));
   residue = beta / normb;
   std::vector<double> H((size_t)(rmax + 1) * rmax), s(L + 1), cs(L + 1), sn(L + 1), y(L + 1), YL((size_t)L * L),
      T((size_t)L * L);
   std::vector<Real> zh(L), yl(L);
   double beta_ratio = 1;
   const double max_beta_ratio = 0.99, min_beta_ratio = 0.175;
   int restart_cycles = 0;
   int m = rmax;
   while (check()) {
      if (rmax > rmin && restart_cycles > 0) {
         if (beta_ratio > max_beta_ratio)
            m = rmax;
         else if (beta_ratio >= min_beta_ratio) {
            const int step = dmin + (dmax - dmin) / static_cast<float>(rmax - rmin) * (m - rmin);
            if (m - step >= rmin)
               m -= step;
            else
               m = rmax;
         }
      }
      int o_steps = m;
      TNLB_CUDA_TRY(cudaMemcpyAsync(z.ptr, r.ptr, sizeof(Real) * n, cudaMemcpyDeviceToDevice, c.st));
      std::fill(H.begin(), H.end(), 0.0);
      std::fill(s.begin(), s.end(), 0.0);
      std::fill(T.begin(), T.end(), 0.0);
      for (int i = 0; i <= m; i++) {
         const bool cont = check();
         it++;
         if (!cont) break;
         Real* yi = Y + (int64_t)i * ld;
         // hauseholder_generate (GMRES.hpp:468-537)
         k_truncate<Real><<<G, kRedThreads, 0, c.st>>>(n, i, z.as<Real>(), yi);
         TNLB_CHECK_LAUNCH();
         double normz;
         TNLB_TRY_STATUS(norm(yi, &normz));
         TNLB_CUDA_TRY(cudaMemcpyAsync(zh.data(), z.ptr, sizeof(Real) * (i + 1), cudaMemcpyDeviceToHost, c.st));
         TNLB_CUDA_TRY(cudaStreamSynchronize(c.st));
         const double y_ii = (double)zh[i];
         const Real yii_new = (Real)(y_ii > 0.0 ? y_ii + normz : y_ii - normz);
         TNLB_CUDA_TRY(cudaMemcpyAsync(yi + i, &yii_new, sizeof(Real), cudaMemcpyHostToDevice, c.st));
         const double norm_yi_squared = 2 * (normz * normz + std::fabs(y_ii) * normz);
         const double t_i = 2.0 / norm_yi_squared;
         T[i + (size_t)i * L] = t_i;
         if (i > 0) TNLB_TRY_STATUS(ytv(i, yi));
         // the upper block of Y, copied to the host (hauseholder_apply_trunc)
         TNLB_CUDA_TRY(cudaMemcpyAsync(yl.data(), yi, sizeof(Real) * L, cudaMemcpyDeviceToHost, c.st));
         TNLB_CUDA_TRY(cudaStreamSynchronize(c.st));
         if (i > 0)
            for (int k = 0; k < i; k++) {
               double tk = 0.0;
               for (int j = k; j < i; j++) tk -= T[k + (size_t)j * L] * (t_i * aux[j]);
               T[k + (size_t)i * L] = tk;
            }
         for (int k = 0; k < L; k++) YL[(size_t)i * L + k] = (double)yl[k];
         // s = e_1^T P_0 z (i = 0) or H_{i-1} = P_i z: z[0..i] - y_i[0..i]
         double* out = i == 0 ? s.data() : H.data() + (size_t)(i - 1) * (m + 1);
         for (int k = 0; k <= i; k++) out[k] = (double)zh[k] - YL[(size_t)i * L + k] * 1.0;
         // v_i = (I - Y_i T_i Y_i^T) e_i (hauseholder_cwy)
         for (int k = 0; k <= i; k++) aux[k] = YL[i + (size_t)k * L];
         for (int k = 0; k <= i; k++) {
            double a2 = 0.0;
            for (int j = k; j <= i; j++) a2 += T[k + (size_t)j * L] * aux[j];
            aux[k] = a2;
         }
         TNLB_TRY_STATUS(gemv(i + 1, -1.0, nullptr, 0.0, v.as<Real>(), i));
         if (i < m) {
            // w = M^-1 A v_i; z = (I - Y_i T_i^T Y_i^T) w (hauseholder_cwy_transposed)
            if (pre) {
               TNLB_TRY_STATUS(c.spmv(v.as<Real>(), M_tmp.as<Real>()));
               TNLB_TRY_STATUS(P.apply(n, M_tmp.as<Real>(), w.as<Real>(), c.st));
            }
            else
               TNLB_TRY_STATUS(c.spmv(v.as<Real>(), w.as<Real>()));
            TNLB_TRY_STATUS(ytv(i + 1, w.as<Real>()));
            TNLB_CUDA_TRY(cudaStreamSynchronize(c.st));
            for (int k = i; k >= 0; k--) {
               double a2 = 0.0;
               for (int j = 0; j <= k; j++) a2 += T[j + (size_t)k * L] * aux[j];
               aux[k] = a2;
            }
            TNLB_TRY_STATUS(gemv(i + 1, -1.0, w.as<Real>(), 1.0, z.as<Real>(), -1));
         }
         if (i > 0) givens_column(i - 1, m, H.data(), s.data(), cs.data(), sn.data());
         residue = std::fabs(s[i]) / normb;
         if (i > 0 && !check()) {
            o_steps = i - 1;
            break;
         }
      }
      // update (GMRES.hpp:648-725, CWY branch)
      const int k = o_steps < m ? o_steps : m - 1;
      for (int q = 0; q <= m; q++) y[q] = s[q];
      for (int q = k; q >= 0; q--) {
         if (H[q + (size_t)q * (m + 1)] == 0) {
            set_error("GMRES: zero diagonal element of the Hessenberg matrix (breakdown)");
            return TNLB_ERR_BREAKDOWN;
         }
         y[q] /= H[q + (size_t)q * (m + 1)];
         for (int j = q - 1; j >= 0; j--) y[j] -= H[j + (size_t)q * (m + 1)] * y[q];
      }
      for (int j = 0; j <= k; j++) aux[j] = 0;
      for (int j = 0; j <= k; j++)
         for (int q = 0; q <= j; q++) aux[q] += y[j] * YL[j + (size_t)q * L];
      for (int q = 0; q <= k; q++) {
         double a2 = 0.0;
         for (int j = q; j <= k; j++) a2 += T[q + (size_t)j * L] * aux[j];
         aux[q] = a2;
      }
      TNLB_TRY_STATUS(gemv(k + 1, -1.0, x, 1.0, x, -1));
      TNLB_CUDA_TRY(cudaMemcpyAsync(ydev.ptr, y.data(), sizeof(double) * (k + 1), cudaMemcpyHostToDevice, c.st));
      k_add_head<Real><<<1, 128, 0, c.st>>>(k + 1, ydev.as<double>(), x);
      TNLB_CHECK_LAUNCH();
      if (o_steps < m) break;
      TNLB_TRY_STATUS(compute_residue());
      const double beta_old = beta;
      TNLB_TRY_STATUS(norm(r.as<Real>(), &beta));
      residue = beta / normb;
      ++restart_cycles;
      beta_ratio = beta / beta_old;
   }
   TNLB_CUDA_TRY(cudaStreamSynchronize(c.st));
   res->iterations = it;
   res->residue = residue;
   res->converged = check_convergence(residue, it, prm.max_iterations, prm.min_iterations, prm.convergence_residue,
                                      prm.divergence_residue);
   res->status_detail = 0;
   return TNLB_OK;
}

template <typename Real>
tnlb_status gmres_solve(const Ctx<Real>& c, const Precond<Real>& P, const tnlb_solver_params& prm, const Real* b,
                        Real* x, tnlb_solve_result* res, bool flexible = false)
{
   // flexible = right preconditioning with the preconditioned basis kept
   // (FGMRES): w = A M^-1 v_i, x += Z y; residues are unpreconditioned.
   const int64_t n = c.n;
   const int rmin = prm.gmres_restarting_min, rmax = prm.gmres_restarting_max;
   const int dmin = prm.gmres_restarting_step_min, dmax = prm.gmres_restarting_step_max;
   TNLB_REQUIRE(rmin > 0 && rmax > 0 && rmin <= rmax, TNLB_ERR_INVALID_ARGUMENT,
                "Wrong value for the GMRES restarting parameters");
   TNLB_REQUIRE(dmin >= 0 && dmax >= 0 && dmin <= dmax, TNLB_ERR_INVALID_ARGUMENT,
                "Wrong value for the GMRES restarting adjustment parameters");
   TNLB_REQUIRE(rmax <= 64, TNLB_ERR_INVALID_ARGUMENT, "GMRES restarting parameter above 64 is not supported");
   const int variant = prm.gmres_variant;
   TNLB_REQUIRE(variant >= TNLB_GMRES_CGS && variant <= TNLB_GMRES_CWY, TNLB_ERR_INVALID_ARGUMENT,
                "unknown GMRES variant");
   if (variant == TNLB_GMRES_CWY) {
      TNLB_REQUIRE(!flexible, TNLB_ERR_NOT_IMPLEMENTED,
                   "FGMRES keeps its preconditioned basis: use the CGS, CGSR, MGS or MGSR variant");
      return gmres_cwy_solve<Real>(c, P, prm, b, x, res);
   }
   const int m_max = rmax;
   const int64_t ld = (n + 31) / 32 * 32;  // 256-byte aligned columns in FP64
   Work W;
   TNLB_TRY_STATUS(W.alloc());
   DeviceBuffer V, w, r, M_tmp, hdev, ydev;
   TNLB_TRY_STATUS(V.alloc(sizeof(Real) * ld * (m_max + 1)));
   TNLB_TRY_STATUS(w.alloc(sizeof(Real) * n));
   TNLB_TRY_STATUS(r.alloc(sizeof(Real) * n));
   TNLB_TRY_STATUS(M_tmp.alloc(sizeof(Real) * n));
   TNLB_TRY_STATUS(hdev.alloc(sizeof(double) * 128));
   TNLB_TRY_STATUS(ydev.alloc(sizeof(double) * 128));
   DeviceBuffer Z;
   if (flexible) TNLB_TRY_STATUS(Z.alloc(sizeof(Real) * ld * m_max));
   Real* Vp = V.as<Real>();
   double* sc = W.scratch.as<double>();
   const unsigned G = vec_grid(n);
   const bool pre = P.kind != TNLB_PRECOND_NONE && !flexible;
   const bool rightp = P.kind != TNLB_PRECOND_NONE && flexible;
   double hs[2];
   auto norm = [&](const Real* a, double* out) -> tnlb_status {
      k_dots<Real><<<G, kRedThreads, 0, c.st>>>(n, a, a, nullptr, nullptr, W.red(), sc);
      TNLB_CHECK_LAUNCH();
      TNLB_CUDA_TRY(cudaMemcpyAsync(hs, sc, sizeof(hs), cudaMemcpyDeviceToHost, c.st));
      TNLB_CUDA_TRY(cudaStreamSynchronize(c.st));
      *out = std::sqrt(hs[0]);
      return TNLB_OK;
   };
   auto compute_residue = [&]() -> tnlb_status {
      Real* tgt = pre ? M_tmp.as<Real>() : r.as<Real>();
      TNLB_CUDA_TRY(cudaMemcpyAsync(tgt, b, sizeof(Real) * n, cudaMemcpyDeviceToDevice, c.st));
      TNLB_TRY_STATUS(c.spmv(x, tgt, -1.0, 1.0));
      if (pre) TNLB_TRY_STATUS(P.apply(n, M_tmp.as<Real>(), r.as<Real>(), c.st));
      return TNLB_OK;
   };
   int it = 0;
   double residue = 0;
   auto check = [&]() {
      return !(std::isnan(residue) || it > prm.max_iterations ||
               (residue > prm.divergence_residue && it >= prm.min_iterations) ||
               (residue < prm.convergence_residue && it >= prm.min_iterations));
   };
   double normb;
   if (pre) {
      TNLB_TRY_STATUS(P.apply(n, b, M_tmp.as<Real>(), c.st));
      TNLB_TRY_STATUS(norm(M_tmp.as<Real>(), &normb));
   }
   else
      TNLB_TRY_STATUS(norm(b, &normb));
   if (normb == 0) {
      TNLB_CUDA_TRY(cudaMemsetAsync(x, 0, sizeof(Real) * n, c.st));
      *res = tnlb_solve_result{1, 0, 0.0, 0, 0};
      return TNLB_OK;
   }
   TNLB_TRY_STATUS(compute_residue());
   double beta;
   TNLB_TRY_STATUS(norm(r.as<Real>(), &beta));
   residue = beta / normb;
   std::vector<double> H((m_max + 1) * m_max), s(m_max + 1), cs(m_max + 1), sn(m_max + 1), y(m_max + 1);
   double beta_ratio = 1;
   const double max_beta_ratio = 0.99, min_beta_ratio = 0.175;
   int restart_cycles = 0;
   int m = m_max;
   auto rot_apply = [](double& dx, double& dy, double csv, double snv) {
      const double t = csv * dx + snv * dy;
      dy = csv * dy - snv * dx;
      dx = t;
   };
   // x += V y for the first k+1 columns (GMRES::update, GMRES.hpp:648-684)
   auto update = [&](int k) -> tnlb_status {
      for (int i = 0; i <= m; i++) y[i] = s[i];
      for (int i = k; i >= 0; i--) {
         if (H[i + i * (m + 1)] == 0) {
            set_error("GMRES: zero diagonal element of the Hessenberg matrix (breakdown)");
            return TNLB_ERR_BREAKDOWN;
         }
         y[i] /= H[i + i * (m + 1)];
         for (int j = i - 1; j >= 0; j--) y[j] -= H[j + i * (m + 1)] * y[i];
      }
      TNLB_CUDA_TRY(cudaMemcpyAsync(ydev.ptr, y.data(), sizeof(double) * (k + 1), cudaMemcpyHostToDevice, c.st));
      k_gmres_update<Real><<<vec_grid(n), kRedThreads, 0, c.st>>>(n, ld, k + 1, rightp ? Z.as<Real>() : Vp,
                                                                  ydev.as<double>(), x);
      TNLB_CHECK_LAUNCH();
      return TNLB_OK;
   };
   while (check()) {
      if (rmax > rmin && restart_cycles > 0) {
         if (beta_ratio > max_beta_ratio)
            m = rmax;
         else if (beta_ratio >= min_beta_ratio) {
            const int step = dmin + (dmax - dmin) / static_cast<float>(rmax - rmin) * (m - rmin);
            if (m - step >= rmin)
               m -= step;
            else
               m = rmax;
         }
      }
      // orthogonalisation (CGS / CGSR / MGS / MGSR)
      int o_steps = m;
      k_scale<Real><<<vec_grid(n), kRedThreads, 0, c.st>>>(n, (Real)(1.0 / beta), r.as<Real>(), Vp);
      TNLB_CHECK_LAUNCH();
      std::fill(H.begin(), H.end(), 0.0);
      std::fill(s.begin(), s.end(), 0.0);
      s[0] = beta;
      for (int i = 0; i < m; i++) {
         const bool cont = check();
         it++;
         if (!cont) break;
         Real* vi = Vp + (int64_t)i * ld;
         // w = M^-1 A v_i (left), or z_i = M^-1 v_i, w = A z_i (flexible)
         if (rightp) {
            Real* zi = Z.as<Real>() + (int64_t)i * ld;
            TNLB_TRY_STATUS(P.apply(n, vi, zi, c.st));
            TNLB_TRY_STATUS(c.spmv(zi, w.as<Real>()));
         }
         else if (pre) {
            TNLB_TRY_STATUS(c.spmv(vi, M_tmp.as<Real>()));
            TNLB_TRY_STATUS(P.apply(n, M_tmp.as<Real>(), w.as<Real>(), c.st));
         }
         else
            TNLB_TRY_STATUS(c.spmv(vi, w.as<Real>()));
         for (int k = 0; k <= i; k++) H[k + i * (m + 1)] = 0.0;
         const int reorth = (variant == TNLB_GMRES_CGSR || variant == TNLB_GMRES_MGSR) ? 2 : 1;
         double normw = 0;
         std::vector<double> hl(i + 1);
         if (variant == TNLB_GMRES_CGS || variant == TNLB_GMRES_CGSR) {
            for (int l = 0; l < reorth; l++) {
               k_gmres_vtw<Real><<<vec_grid(n), kRedThreads, 0, c.st>>>(
                  n, ld, i + 1, Vp, w.as<Real>(), W.partials.as<double>(), W.counter.as<unsigned>() + 1,
                  hdev.as<double>());
               TNLB_CHECK_LAUNCH();
               const bool last = (l == reorth - 1);
               k_gmres_wmvh<Real><<<vec_grid(n), kRedThreads, 0, c.st>>>(n, ld, i + 1, Vp, hdev.as<double>(),
                                                                       w.as<Real>(), W.red(), last ? sc : nullptr);
               TNLB_CHECK_LAUNCH();
               TNLB_CUDA_TRY(cudaMemcpyAsync(hl.data(), hdev.ptr, sizeof(double) * (i + 1), cudaMemcpyDeviceToHost, c.st));
               if (last) TNLB_CUDA_TRY(cudaMemcpyAsync(hs, sc, sizeof(double), cudaMemcpyDeviceToHost, c.st));
               TNLB_CUDA_TRY(cudaStreamSynchronize(c.st));
               for (int k = 0; k <= i; k++) H[k + i * (m + 1)] += hl[k];
            }
            normw = hs[0];
         }
         else {
            // MGS: H_{k,i} = (w, v_k); w -= H_{k,i} v_k for k = 0..i, `reorth`
            // passes.  Each kernel applies one update and computes the next
            // dot product (or, after the last update, |w|).
            double* hd = hdev.as<double>();  // pass l uses hd[l*64 .. l*64+i]
            k_mgs_step<Real><<<vec_grid(n), kRedThreads, 0, c.st>>>(n, nullptr, nullptr, w.as<Real>(), Vp, W.red(),
                                                                    hd);
            TNLB_CHECK_LAUNCH();
            for (int l = 0; l < reorth; l++) {
               for (int k = 0; k <= i; k++) {
                  const Real* vk = Vp + (int64_t)k * ld;
                  const bool last_k = (k == i), last_l = (l == reorth - 1);
                  const Real* next = !last_k ? Vp + (int64_t)(k + 1) * ld : (!last_l ? Vp : nullptr);
                  double* out = !last_k ? hd + l * 64 + k + 1 : (!last_l ? hd + (l + 1) * 64 : sc);
                  k_mgs_step<Real><<<vec_grid(n), kRedThreads, 0, c.st>>>(n, vk, hd + l * 64 + k, w.as<Real>(), next,
                                                                          W.red(), out);
                  TNLB_CHECK_LAUNCH();
               }
            }
            std::vector<double> hall(2 * 64);
            TNLB_CUDA_TRY(cudaMemcpyAsync(hall.data(), hd, sizeof(double) * 2 * 64, cudaMemcpyDeviceToHost, c.st));
            TNLB_CUDA_TRY(cudaMemcpyAsync(hs, sc, sizeof(double), cudaMemcpyDeviceToHost, c.st));
            TNLB_CUDA_TRY(cudaStreamSynchronize(c.st));
            for (int l = 0; l < reorth; l++)
               for (int k = 0; k <= i; k++) H[k + i * (m + 1)] += hall[l * 64 + k];
            normw = hs[0];
         }
         H[i + 1 + i * (m + 1)] = normw;
         k_scale<Real><<<vec_grid(n), kRedThreads, 0, c.st>>>(n, (Real)(1.0 / normw), w.as<Real>(),
                                                              Vp + (int64_t)(i + 1) * ld);
         TNLB_CHECK_LAUNCH();
         // Givens rotations (GMRES.hpp:731-770)
         for (int k = 0; k < i; k++) rot_apply(H[k + i * (m + 1)], H[k + 1 + i * (m + 1)], cs[k], sn[k]);
         if (H[i + 1 + i * (m + 1)] != 0.0) {
            const double dx = H[i + i * (m + 1)], dy = H[i + 1 + i * (m + 1)];
            if (dy == 0.0) {
               cs[i] = 1.0;
               sn[i] = 0.0;
            }
            else if (std::fabs(dy) > std::fabs(dx)) {
               const double t = dx / dy;
               sn[i] = 1.0 / std::sqrt(1.0 + t * t);
               cs[i] = t * sn[i];
            }
            else {
               const double t = dy / dx;
               cs[i] = 1.0 / std::sqrt(1.0 + t * t);
               sn[i] = t * cs[i];
            }
            rot_apply(H[i + i * (m + 1)], H[i + 1 + i * (m + 1)], cs[i], sn[i]);
            rot_apply(s[i], s[i + 1], cs[i], sn[i]);
         }
         residue = std::fabs(s[i + 1]) / normb;
         if (!check()) {
            o_steps = i;
            break;
         }
      }
      if (o_steps < m) {
         TNLB_TRY_STATUS(update(o_steps));
         break;
      }
      TNLB_TRY_STATUS(update(m - 1));
      TNLB_TRY_STATUS(compute_residue());
      const double beta_old = beta;
      TNLB_TRY_STATUS(norm(r.as<Real>(), &beta));
      residue = beta / normb;
      ++restart_cycles;
      beta_ratio = beta / beta_old;
   }
   TNLB_CUDA_TRY(cudaStreamSynchronize(c.st));
   res->iterations = it;
   res->residue = residue;
   res->converged = check_convergence(residue, it, prm.max_iterations, prm.min_iterations, prm.convergence_residue,
                                      prm.divergence_residue);
   res->status_detail = 0;
   return TNLB_OK;
}

// ------------------------------------------ TFQMR, BiCGStab(ell), IDR(s)

// x_s = x_s - gamma (x_s - x) (residual smoothing of IDR(s))
template <typename Real>
__global__ void k_smooth_x(int64_t n, Real gamma, const Real* __restrict__ x, Real* __restrict__ xs)
{
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
      xs[i] = xs[i] - gamma * (xs[i] - x[i]);
}

// Host-driven vector operations shared by the solvers below: each dot or
// norm is one deterministic grid reduction read back to the host.
template <typename Real>
struct VecOps {
   const Ctx<Real>& c;
   Work& W;
   unsigned G;
   double hs[2];
   VecOps(const Ctx<Real>& c_, Work& W_) : c(c_), W(W_), G(vec_grid(c_.n)) {}
   tnlb_status dot(const Real* a, const Real* b, double* out)
   {
      k_dots<Real><<<G, kRedThreads, 0, c.st>>>(c.n, a, b, nullptr, nullptr, W.red(), W.scratch.as<double>());
      TNLB_CHECK_LAUNCH();
      TNLB_CUDA_TRY(cudaMemcpyAsync(hs, W.scratch.ptr, sizeof(hs), cudaMemcpyDeviceToHost, c.st));
      TNLB_CUDA_TRY(cudaStreamSynchronize(c.st));
      *out = hs[0];
      return TNLB_OK;
   }
   tnlb_status norm(const Real* a, double* out)
   {
      TNLB_TRY_STATUS(dot(a, a, out));
      *out = std::sqrt(*out);
      return TNLB_OK;
   }
   // y = a x + b y
   tnlb_status axpby(double a, const Real* x, double b, Real* y)
   {
      k_axpby<Real><<<G, kRedThreads, 0, c.st>>>(c.n, (Real)a, x, (Real)b, y);
      TNLB_CHECK_LAUNCH();
      return TNLB_OK;
   }
   tnlb_status copy(Real* dst, const Real* src)
   {
      TNLB_CUDA_TRY(cudaMemcpyAsync(dst, src, sizeof(Real) * c.n, cudaMemcpyDeviceToDevice, c.st));
      return TNLB_OK;
   }
};

// The stopping rule of IterativeSolver (IterativeSolver.hpp:98-143) on host
// scalars; next() checks, then counts the iteration, as nextIteration does.
struct HostStop {
   const tnlb_solver_params& prm;
   int it = 0;
   double residue = 0;
   explicit HostStop(const tnlb_solver_params& p) : prm(p) {}
   bool check() const
   {
      return !(std::isnan(residue) || it > prm.max_iterations ||
               (residue > prm.divergence_residue && it >= prm.min_iterations) ||
               (residue < prm.convergence_residue && it >= prm.min_iterations));
   }
   bool next()
   {
      const bool r = check();
      it++;
      return r;
   }
   void finish(tnlb_solve_result* res, bool ok = true) const
   {
      res->iterations = it;
      res->residue = residue;
      res->converged = ok && check_convergence(residue, it, prm.max_iterations, prm.min_iterations,
                                               prm.convergence_residue, prm.divergence_residue);
      res->status_detail = 0;
   }
};

// TFQMR (Solvers/Linear/TFQMR.hpp:12-113): left-preconditioned; the
// stopping residue is the quasi-residual bound tau sqrt(iter+1) / ||M^-1 b||.
template <typename Real>
tnlb_status tfqmr_solve(const Ctx<Real>& c, const Precond<Real>& P, const tnlb_solver_params& prm, const Real* b,
                        Real* x, tnlb_solve_result* res)
{
   const int64_t n = c.n;
   Work W;
   TNLB_TRY_STATUS(W.alloc());
   DeviceBuffer d, r, w, u, v, r_ast, Au, M_tmp;
   for (auto* q : {&d, &r, &w, &u, &v, &r_ast, &Au, &M_tmp}) TNLB_TRY_STATUS(q->alloc(sizeof(Real) * n));
   VecOps<Real> V(c, W);
   const bool pre = P.kind != TNLB_PRECOND_NONE;
   auto pmv = [&](const Real* src, Real* dst) -> tnlb_status {
      if (!pre) return c.spmv(src, dst);
      TNLB_TRY_STATUS(c.spmv(src, M_tmp.as<Real>()));
      return P.apply(n, M_tmp.as<Real>(), dst, c.st);
   };
   HostStop S(prm);
   double b_norm;
   if (pre) {
      TNLB_TRY_STATUS(P.apply(n, b, M_tmp.as<Real>(), c.st));
      TNLB_TRY_STATUS(V.norm(M_tmp.as<Real>(), &b_norm));
      TNLB_TRY_STATUS(V.copy(M_tmp.as<Real>(), b));
      TNLB_TRY_STATUS(c.spmv(x, M_tmp.as<Real>(), -1.0, 1.0));
      TNLB_TRY_STATUS(P.apply(n, M_tmp.as<Real>(), r.as<Real>(), c.st));
   }
   else {
      TNLB_TRY_STATUS(V.norm(b, &b_norm));
      TNLB_TRY_STATUS(V.copy(r.as<Real>(), b));
      TNLB_TRY_STATUS(c.spmv(x, r.as<Real>(), -1.0, 1.0));
   }
   if (b_norm == 0) {
      TNLB_CUDA_TRY(cudaMemsetAsync(x, 0, sizeof(Real) * n, c.st));
      TNLB_CUDA_TRY(cudaStreamSynchronize(c.st));
      *res = tnlb_solve_result{1, 0, 0.0, 0, 0};
      return TNLB_OK;
   }
   TNLB_TRY_STATUS(V.copy(w.as<Real>(), r.as<Real>()));
   TNLB_TRY_STATUS(V.copy(u.as<Real>(), r.as<Real>()));
   TNLB_TRY_STATUS(pmv(u.as<Real>(), Au.as<Real>()));
   TNLB_TRY_STATUS(V.copy(v.as<Real>(), Au.as<Real>()));
   TNLB_CUDA_TRY(cudaMemsetAsync(d.ptr, 0, sizeof(Real) * n, c.st));
   double tau, theta = 0.0, eta = 0.0, rho, alpha = 0.0;
   TNLB_TRY_STATUS(V.norm(r.as<Real>(), &tau));
   TNLB_TRY_STATUS(V.copy(r_ast.as<Real>(), r.as<Real>()));
   TNLB_TRY_STATUS(V.dot(r_ast.as<Real>(), r.as<Real>(), &rho));
   S.residue = tau / b_norm;
   while (S.next()) {
      const int iter = S.it;
      if (iter % 2 == 1) {
         double vr;
         TNLB_TRY_STATUS(V.dot(v.as<Real>(), r_ast.as<Real>(), &vr));
         alpha = rho / vr;
      }
      else
         TNLB_TRY_STATUS(pmv(u.as<Real>(), Au.as<Real>()));
      TNLB_TRY_STATUS(V.axpby(-alpha, Au.as<Real>(), 1.0, w.as<Real>()));
      TNLB_TRY_STATUS(V.axpby(1.0, u.as<Real>(), theta * theta * eta / alpha, d.as<Real>()));
      double w_norm;
      TNLB_TRY_STATUS(V.norm(w.as<Real>(), &w_norm));
      theta = w_norm / tau;
      const double cc = 1.0 / std::sqrt(1.0 + theta * theta);
      tau = tau * theta * cc;
      eta = cc * cc * alpha;
      TNLB_TRY_STATUS(V.axpby(eta, d.as<Real>(), 1.0, x));
      S.residue = tau * std::sqrt((double)(iter + 1)) / b_norm;
      if (iter > prm.min_iterations && S.residue < prm.convergence_residue) break;
      if (iter % 2 == 0) {
         double rho_new;
         TNLB_TRY_STATUS(V.dot(w.as<Real>(), r_ast.as<Real>(), &rho_new));
         const double beta = rho_new / rho;
         rho = rho_new;
         TNLB_TRY_STATUS(V.axpby(1.0, w.as<Real>(), beta, u.as<Real>()));
         TNLB_TRY_STATUS(V.axpby(beta, Au.as<Real>(), beta * beta, v.as<Real>()));
         TNLB_TRY_STATUS(pmv(u.as<Real>(), Au.as<Real>()));
         TNLB_TRY_STATUS(V.axpby(1.0, Au.as<Real>(), 1.0, v.as<Real>()));
      }
      else
         TNLB_TRY_STATUS(V.axpby(-alpha, v.as<Real>(), 1.0, u.as<Real>()));
   }
   TNLB_CUDA_TRY(cudaStreamSynchronize(c.st));
   S.finish(res);
   return TNLB_OK;
}

// BiCGStab(ell) (Solvers/Linear/BICGStabL.hpp:36-242): R and U hold ell+1
// columns (256-byte aligned) on the device; T, sigma and the g vectors are
// small and live on the host, as in the reference.
template <typename Real>
tnlb_status bicgstabl_solve(const Ctx<Real>& c, const Precond<Real>& P, const tnlb_solver_params& prm, const Real* b,
                            Real* x, tnlb_solve_result* res)
{
   const int64_t n = c.n;
   const int ell = prm.bicgstab_ell;
   TNLB_REQUIRE(ell >= 1 && ell <= 32, TNLB_ERR_INVALID_ARGUMENT, "bicgstab-ell must lie in 1..32");
   const int64_t ld = (n + 31) / 32 * 32;
   Work W;
   TNLB_TRY_STATUS(W.alloc());
   DeviceBuffer Rb, Ub, r_ast, M_tmp, res_tmp, cdev;
   TNLB_TRY_STATUS(Rb.alloc(sizeof(Real) * ld * (ell + 1)));
   TNLB_TRY_STATUS(Ub.alloc(sizeof(Real) * ld * (ell + 1)));
   for (auto* q : {&r_ast, &M_tmp, &res_tmp}) TNLB_TRY_STATUS(q->alloc(sizeof(Real) * n));
   TNLB_TRY_STATUS(cdev.alloc(sizeof(double) * 128));
   Real* R = Rb.as<Real>();
   Real* U = Ub.as<Real>();
   auto Rc = [&](int j) { return R + (int64_t)j * ld; };
   auto Uc = [&](int j) { return U + (int64_t)j * ld; };
   VecOps<Real> V(c, W);
   const bool pre = P.kind != TNLB_PRECOND_NONE;
   auto pmv = [&](const Real* src, Real* dst) -> tnlb_status {
      if (!pre) return c.spmv(src, dst);
      TNLB_TRY_STATUS(c.spmv(src, M_tmp.as<Real>()));
      return P.apply(n, M_tmp.as<Real>(), dst, c.st);
   };
   auto compute_residue = [&](Real* out) -> tnlb_status {
      Real* tgt = pre ? M_tmp.as<Real>() : out;
      TNLB_TRY_STATUS(V.copy(tgt, b));
      TNLB_TRY_STATUS(c.spmv(x, tgt, -1.0, 1.0));
      if (pre) TNLB_TRY_STATUS(P.apply(n, M_tmp.as<Real>(), out, c.st));
      return TNLB_OK;
   };
   // out = alpha * Y[:, 0:cols] coef + beta * in
   auto gemv = [&](const Real* Y, int cols, const double* coef, double alpha, const Real* in, double beta,
                   Real* out) -> tnlb_status {
      TNLB_CUDA_TRY(cudaMemcpyAsync(cdev.ptr, coef, sizeof(double) * cols, cudaMemcpyHostToDevice, c.st));
      k_gemv_cols<Real><<<V.G, kRedThreads, 0, c.st>>>(n, ld, cols, Y, cdev.as<double>(), alpha, in, beta, out, -1);
      TNLB_CHECK_LAUNCH();
      return TNLB_OK;
   };
   HostStop S(prm);
   double b_norm;
   if (pre) {
      TNLB_TRY_STATUS(P.apply(n, b, M_tmp.as<Real>(), c.st));
      TNLB_TRY_STATUS(V.norm(M_tmp.as<Real>(), &b_norm));
   }
   else
      TNLB_TRY_STATUS(V.norm(b, &b_norm));
   if (b_norm == 0) {
      TNLB_CUDA_TRY(cudaMemsetAsync(x, 0, sizeof(Real) * n, c.st));
      TNLB_CUDA_TRY(cudaStreamSynchronize(c.st));
      *res = tnlb_solve_result{1, 0, 0.0, 0, 0};
      return TNLB_OK;
   }
   std::vector<double> T((size_t)ell * ell, 0.0), sigma(ell + 1), g0(ell + 1), g1(ell + 1), g2(ell + 1);
   TNLB_TRY_STATUS(compute_residue(Rc(0)));
   TNLB_TRY_STATUS(V.norm(Rc(0), &sigma[0]));
   TNLB_REQUIRE(!std::isnan(sigma[0]), TNLB_ERR_INVALID_ARGUMENT, "BiCGstab(ell): initial residue is NAN");
   TNLB_TRY_STATUS(V.copy(r_ast.as<Real>(), Rc(0)));
   TNLB_TRY_STATUS(V.axpby(0.0, r_ast.as<Real>(), 1.0 / sigma[0], r_ast.as<Real>()));
   TNLB_CUDA_TRY(cudaMemsetAsync(Uc(0), 0, sizeof(Real) * n, c.st));
   double rho_0 = 1.0, rho_1, alpha = 0.0, beta, gamma, omega = 1.0;
   S.residue = sigma[0] / b_norm;
   while (S.check()) {
      rho_0 = -omega * rho_0;
      for (int j = 0; j < ell; j++) {
         S.next();
         TNLB_TRY_STATUS(V.dot(r_ast.as<Real>(), Rc(j), &rho_1));
         beta = alpha * rho_1 / rho_0;
         rho_0 = rho_1;
         for (int q = 0; q <= j; q++) TNLB_TRY_STATUS(V.axpby(1.0, Rc(q), -beta, Uc(q)));
         TNLB_TRY_STATUS(pmv(Uc(j), Uc(j + 1)));
         TNLB_TRY_STATUS(V.dot(r_ast.as<Real>(), Uc(j + 1), &gamma));
         alpha = rho_0 / gamma;
         for (int q = 0; q <= j; q++) TNLB_TRY_STATUS(V.axpby(-alpha, Uc(q + 1), 1.0, Rc(q)));
         TNLB_TRY_STATUS(pmv(Rc(j), Rc(j + 1)));
         TNLB_TRY_STATUS(V.axpby(alpha, Uc(0), 1.0, x));
      }
      for (int j = 1; j <= ell; j++) {
         for (int i = 1; i < j; i++) {
            const int ij = (i - 1) + (j - 1) * ell;
            double d;
            TNLB_TRY_STATUS(V.dot(Rc(i), Rc(j), &d));
            T[ij] = d / sigma[i];
            TNLB_TRY_STATUS(V.axpby(-T[ij], Rc(i), 1.0, Rc(j)));
         }
         TNLB_TRY_STATUS(V.dot(Rc(j), Rc(j), &sigma[j]));
         double d;
         TNLB_TRY_STATUS(V.dot(Rc(0), Rc(j), &d));
         g1[j] = d / sigma[j];
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
      TNLB_TRY_STATUS(gemv(Rc(0), ell, g2.data(), 1.0, x, 1.0, x));
      TNLB_TRY_STATUS(gemv(Rc(1), ell, g1.data() + 1, -1.0, Rc(0), 1.0, Rc(0)));
      TNLB_TRY_STATUS(gemv(Uc(1), ell, g0.data() + 1, -1.0, Uc(0), 1.0, Uc(0)));
      if (prm.bicgstab_exact_residue) {
         TNLB_TRY_STATUS(compute_residue(res_tmp.as<Real>()));
         TNLB_TRY_STATUS(V.norm(res_tmp.as<Real>(), &sigma[0]));
      }
      else
         TNLB_TRY_STATUS(V.norm(Rc(0), &sigma[0]));
      S.residue = sigma[0] / b_norm;
   }
   TNLB_CUDA_TRY(cudaStreamSynchronize(c.st));
   S.finish(res);
   return TNLB_OK;
}

// The shadow space of IDR(s), drawn as IDRs::setSize does
// (Solvers/Linear/IDRs.hpp:270-300): std::mt19937 seeded 0,
// std::normal_distribution(0, 1), s columns of length n; then, for each
// column i and each j < i, P_i = P_i - (P_i, P_j) (the scalar subtracted from
// every entry, as the reference does) and P_i /= ||P_i||.
template <typename Real>
std::vector<Real> idrs_shadow(int64_t n, int s)
{
   std::vector<Real> P((size_t)n * s);
   std::mt19937 rng;
   rng.seed(0);
   std::normal_distribution<Real> dist(0, 1);
   for (auto& p : P) p = dist(rng);
   for (int i = 0; i < s; i++) {
      Real* Pi = P.data() + (size_t)i * n;
      for (int j = 0; j < i; j++) {
         const Real* Pj = P.data() + (size_t)j * n;
         double d = 0;
         for (int64_t q = 0; q < n; q++) d += (double)Pi[q] * (double)Pj[q];
         for (int64_t q = 0; q < n; q++) Pi[q] = (Real)(Pi[q] - d);
      }
      double nn = 0;
      for (int64_t q = 0; q < n; q++) nn += (double)Pi[q] * (double)Pi[q];
      nn = std::sqrt(nn);
      for (int64_t q = 0; q < n; q++) Pi[q] = (Real)(Pi[q] / nn);
   }
   return P;
}

// IDR(s) (Solvers/Linear/IDRs.hpp:50-250): residues unpreconditioned, the
// preconditioner applied to the update directions; P, G and U are n x s on
// the device, M, f and the small LU solves (LUsequential.h) on the host.
template <typename Real>
tnlb_status idrs_solve(const Ctx<Real>& c, const Precond<Real>& Pc, const tnlb_solver_params& prm, const Real* b,
                       Real* x, tnlb_solve_result* res)
{
   const int64_t n = c.n;
   const int s = prm.idr_s;
   TNLB_REQUIRE(s >= 1 && s <= 32, TNLB_ERR_INVALID_ARGUMENT, "idr-s must lie in 1..32");
   const bool smoothing = prm.idr_residual_smoothing != 0;
   const int64_t ld = (n + 31) / 32 * 32;
   Work W;
   TNLB_TRY_STATUS(W.alloc());
   DeviceBuffer Pb, Gb, Ub, r, v, pv, t, x_s, r_s, cdev, hdev;
   for (auto* q : {&Pb, &Gb, &Ub}) TNLB_TRY_STATUS(q->alloc(sizeof(Real) * ld * s));
   for (auto* q : {&r, &v, &pv, &t, &x_s, &r_s}) TNLB_TRY_STATUS(q->alloc(sizeof(Real) * n));
   TNLB_TRY_STATUS(cdev.alloc(sizeof(double) * 128));
   TNLB_TRY_STATUS(hdev.alloc(sizeof(double) * 128));
   Real* Pd = Pb.as<Real>();
   Real* Gd = Gb.as<Real>();
   Real* Ud = Ub.as<Real>();
   auto col = [&](Real* Y, int j) { return Y + (int64_t)j * ld; };
   VecOps<Real> V(c, W);
   const bool pre = Pc.kind != TNLB_PRECOND_NONE;
   {
      const std::vector<Real> Ph = idrs_shadow<Real>(n, s);
      for (int j = 0; j < s; j++)
         TNLB_CUDA_TRY(cudaMemcpyAsync(col(Pd, j), Ph.data() + (size_t)j * n, sizeof(Real) * n,
                                       cudaMemcpyHostToDevice, c.st));
      TNLB_CUDA_TRY(cudaStreamSynchronize(c.st));
   }
   TNLB_CUDA_TRY(cudaMemsetAsync(Gd, 0, sizeof(Real) * ld * s, c.st));
   TNLB_CUDA_TRY(cudaMemsetAsync(Ud, 0, sizeof(Real) * ld * s, c.st));
   // P_[first:first+cnt]^T a -> host
   std::vector<double> hv(s);
   auto ptv = [&](int first, int cnt, const Real* a) -> tnlb_status {
      k_gmres_vtw<Real><<<V.G, kRedThreads, 0, c.st>>>(n, ld, cnt, col(Pd, first), a, W.partials.as<double>(),
                                                      W.counter.as<unsigned>() + 1, hdev.as<double>());
      TNLB_CHECK_LAUNCH();
      TNLB_CUDA_TRY(cudaMemcpyAsync(hv.data(), hdev.ptr, sizeof(double) * cnt, cudaMemcpyDeviceToHost, c.st));
      TNLB_CUDA_TRY(cudaStreamSynchronize(c.st));
      return TNLB_OK;
   };
   auto gemv = [&](const Real* Y, int cols, const double* coef, double alpha, const Real* in, double beta,
                   Real* out) -> tnlb_status {
      TNLB_CUDA_TRY(cudaMemcpyAsync(cdev.ptr, coef, sizeof(double) * cols, cudaMemcpyHostToDevice, c.st));
      k_gemv_cols<Real><<<V.G, kRedThreads, 0, c.st>>>(n, ld, cols, Y, cdev.as<double>(), alpha, in, beta, out, -1);
      TNLB_CHECK_LAUNCH();
      return TNLB_OK;
   };
   // psolve(src, dst) of the reference: M^-1 src, or a copy
   auto psolve = [&](const Real* src, Real* dst) -> tnlb_status {
      if (!pre) return src == dst ? TNLB_OK : V.copy(dst, src);
      TNLB_TRY_STATUS(Pc.apply(n, src, pv.as<Real>(), c.st));
      return V.copy(dst, pv.as<Real>());
   };
   HostStop S(prm);
   double b_norm, r_norm;
   TNLB_TRY_STATUS(V.norm(b, &b_norm));
   if (b_norm == 0) {
      TNLB_CUDA_TRY(cudaMemsetAsync(x, 0, sizeof(Real) * n, c.st));
      TNLB_CUDA_TRY(cudaStreamSynchronize(c.st));
      *res = tnlb_solve_result{1, 0, 0.0, 0, 0};
      return TNLB_OK;
   }
   TNLB_TRY_STATUS(V.copy(r.as<Real>(), b));
   TNLB_TRY_STATUS(c.spmv(x, r.as<Real>(), -1.0, 1.0));
   TNLB_TRY_STATUS(V.norm(r.as<Real>(), &r_norm));
   TNLB_REQUIRE(!std::isnan(r_norm), TNLB_ERR_INVALID_ARGUMENT, "IDR(s): initial residue is NAN");
   const double angle = 0.7;
   double omega = 1.0;
   std::vector<double> M((size_t)s * s, 0.0), f(s), cvec(s), Msub((size_t)s * s);
   for (int i = 0; i < s; i++) M[(size_t)i * s + i] = 1;
   if (smoothing) {
      TNLB_TRY_STATUS(V.copy(x_s.as<Real>(), x));
      TNLB_TRY_STATUS(V.copy(r_s.as<Real>(), r.as<Real>()));
   }
   auto smooth = [&]() -> tnlb_status {
      if (!smoothing) return TNLB_OK;
      TNLB_TRY_STATUS(V.copy(t.as<Real>(), r_s.as<Real>()));
      TNLB_TRY_STATUS(V.axpby(-1.0, r.as<Real>(), 1.0, t.as<Real>()));
      double tr, tt;
      TNLB_TRY_STATUS(V.dot(t.as<Real>(), r_s.as<Real>(), &tr));
      TNLB_TRY_STATUS(V.dot(t.as<Real>(), t.as<Real>(), &tt));
      const double gam = tr / tt;
      TNLB_TRY_STATUS(V.axpby(-gam, t.as<Real>(), 1.0, r_s.as<Real>()));
      k_smooth_x<Real><<<V.G, kRedThreads, 0, c.st>>>(n, (Real)gam, x, x_s.as<Real>());
      TNLB_CHECK_LAUNCH();
      return V.norm(r_s.as<Real>(), &r_norm);
   };
   auto finish_smoothing = [&]() -> tnlb_status { return smoothing ? V.copy(x, x_s.as<Real>()) : TNLB_OK; };
   S.residue = r_norm / b_norm;
   while (S.check()) {
      TNLB_TRY_STATUS(ptv(0, s, r.as<Real>()));
      for (int i = 0; i < s; i++) f[i] = hv[i];
      for (int k = 0; k < s; k++) {
         Real* Uk = col(Ud, k);
         Real* Gk = col(Gd, k);
         const int m = s - k;
         // c = M[k:s, k:s]^-1 f[k:s] (LU without pivoting)
         for (int i = 0; i < m; i++)
            for (int j = 0; j < m; j++) Msub[(size_t)i * s + j] = M[(size_t)(i + k) * s + (j + k)];
         for (int kk = 0; kk < m; kk++) {
            const double pivot = Msub[(size_t)kk * s + kk];
            for (int j = kk + 1; j < m; j++) {
               const double factor = Msub[(size_t)j * s + kk] / pivot;
               Msub[(size_t)j * s + kk] = factor;
               for (int i = kk + 1; i < m; i++) Msub[(size_t)j * s + i] -= factor * Msub[(size_t)kk * s + i];
            }
         }
         for (int i = 0; i < m; i++) cvec[i] = f[k + i];
         for (int kk = 1; kk < m; kk++)
            for (int j = 0; j < kk; j++) cvec[kk] -= Msub[(size_t)kk * s + j] * cvec[j];
         for (int kk = m - 1; kk >= 0; kk--) {
            for (int j = m - 1; j > kk; j--) cvec[kk] -= Msub[(size_t)kk * s + j] * cvec[j];
            cvec[kk] /= Msub[(size_t)kk * s + kk];
         }
         // v = M^-1 (r - G[:, k:s] c); U_k = U[:, k:s] c + omega v; G_k = A U_k
         TNLB_TRY_STATUS(gemv(Gk, m, cvec.data(), -1.0, r.as<Real>(), 1.0, v.as<Real>()));
         TNLB_TRY_STATUS(psolve(v.as<Real>(), v.as<Real>()));
         TNLB_TRY_STATUS(gemv(Uk, m, cvec.data(), 1.0, nullptr, 0.0, Uk));
         TNLB_TRY_STATUS(V.axpby(omega, v.as<Real>(), 1.0, Uk));
         TNLB_TRY_STATUS(c.spmv(Uk, Gk));
         for (int i = 0; i < k; i++) {
            double pg;
            TNLB_TRY_STATUS(V.dot(col(Pd, i), Gk, &pg));
            const double al = pg / M[(size_t)i * s + i];
            TNLB_TRY_STATUS(V.axpby(-al, col(Ud, i), 1.0, Uk));
            TNLB_TRY_STATUS(V.axpby(-al, col(Gd, i), 1.0, Gk));
         }
         TNLB_TRY_STATUS(ptv(k, m, Gk));
         for (int i = k; i < s; i++) M[(size_t)i * s + k] = hv[i - k];
         if (M[(size_t)k * s + k] == 0) {
            TNLB_CUDA_TRY(cudaStreamSynchronize(c.st));
            S.finish(res, false);
            return TNLB_OK;
         }
         const double beta = f[k] / M[(size_t)k * s + k];
         TNLB_TRY_STATUS(V.axpby(beta, Uk, 1.0, x));
         TNLB_TRY_STATUS(V.axpby(-beta, Gk, 1.0, r.as<Real>()));
         TNLB_TRY_STATUS(V.norm(r.as<Real>(), &r_norm));
         TNLB_TRY_STATUS(smooth());
         S.residue = r_norm / b_norm;
         if (!S.next()) {
            TNLB_TRY_STATUS(finish_smoothing());
            TNLB_CUDA_TRY(cudaStreamSynchronize(c.st));
            S.finish(res);
            return TNLB_OK;
         }
         for (int i = k + 1; i < s; i++) f[i] = f[i] - beta * M[(size_t)i * s + k];
      }
      TNLB_TRY_STATUS(psolve(r.as<Real>(), v.as<Real>()));
      TNLB_TRY_STATUS(c.spmv(v.as<Real>(), t.as<Real>()));
      double t_norm, tr;
      TNLB_TRY_STATUS(V.norm(t.as<Real>(), &t_norm));
      TNLB_TRY_STATUS(V.dot(t.as<Real>(), r.as<Real>(), &tr));
      const double rho = std::fabs(tr / (t_norm * r_norm));
      omega = tr / (t_norm * t_norm);
      if (rho < angle) omega = omega * angle / rho;
      if (omega == 0) {
         TNLB_CUDA_TRY(cudaStreamSynchronize(c.st));
         S.finish(res, false);
         return TNLB_OK;
      }
      TNLB_TRY_STATUS(V.axpby(omega, v.as<Real>(), 1.0, x));
      TNLB_TRY_STATUS(V.axpby(-omega, t.as<Real>(), 1.0, r.as<Real>()));
      TNLB_TRY_STATUS(V.norm(r.as<Real>(), &r_norm));
      TNLB_TRY_STATUS(smooth());
      S.residue = r_norm / b_norm;
      S.next();
   }
   TNLB_TRY_STATUS(finish_smoothing());
   TNLB_CUDA_TRY(cudaStreamSynchronize(c.st));
   S.finish(res);
   return TNLB_OK;
}

template <typename Real>
tnlb_status solve_t(tnlb_solver_kind solver, const tnlb_precond* pobj, const tnlb_solver_params& prm,
                    const tnlb_segments* seg, tnlb_real real, const int32_t* cols, const Real* vals, const Real* b,
                    Real* x, cudaStream_t st, tnlb_solve_result* res)
{
   Ctx<Real> c{seg, real, cols, vals, seg->n, st};
   const Precond<Real> P = view<Real>(pobj);
   switch (solver) {
      case TNLB_SOLVER_CG:
         if (P.kind == TNLB_PRECOND_ILU0 || P.kind == TNLB_PRECOND_ILUT) return pcg_general<Real>(c, P, prm, b, x, res);
         return cg_solve<Real>(c, P, prm, b, x, res);
      case TNLB_SOLVER_BICGSTAB: return bicgstab_solve<Real>(c, P, prm, b, x, res);
      case TNLB_SOLVER_GMRES: return gmres_solve<Real>(c, P, prm, b, x, res);
      case TNLB_SOLVER_FGMRES: return gmres_solve<Real>(c, P, prm, b, x, res, true);
      case TNLB_SOLVER_TFQMR: return tfqmr_solve<Real>(c, P, prm, b, x, res);
      case TNLB_SOLVER_BICGSTABL: return bicgstabl_solve<Real>(c, P, prm, b, x, res);
      case TNLB_SOLVER_IDRS: return idrs_solve<Real>(c, P, prm, b, x, res);
   }
   set_error("unknown solver");
   return TNLB_ERR_INVALID_ARGUMENT;
}

template <typename Real>
__global__ void __launch_bounds__(kRedThreads) k_resid_norms(int64_t n, const Real* __restrict__ b,
                                                             const Real* __restrict__ ax, RedWork w,
                                                             double* __restrict__ out)
{
   double a0 = 0, a1 = 0;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
      const double d = (double)b[i] - (double)ax[i];
      a0 += d * d;
      a1 += (double)b[i] * (double)b[i];
   }
   double v[2] = {a0, a1};
   if (publish_and_arrive<2>(v, w)) {
      double t[2];
      gather_totals<2>(t, w);
      if (threadIdx.x == 0) {
         out[0] = t[0];
         out[1] = t[1];
      }
   }
}

// r32 = (float)((b - ax) * scale): the unit-norm FP32 residual of the refinement
__global__ void k_resid_to_f32(int64_t n, const double* __restrict__ b, const double* __restrict__ ax, double scale,
                               float* __restrict__ r32)
{
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
      r32[i] = (float)((b[i] - ax[i]) * scale);
}

}  // namespace

tnlb_status true_residual(const tnlb_segments* seg, tnlb_real real, const int32_t* cols, const void* vals,
                          const void* b, const void* x, cudaStream_t st, double* out)
{
   const int64_t n = seg->n;
   const size_t rs = real == TNLB_F64 ? 8 : 4;
   DeviceBuffer ax;
   Work W;
   TNLB_TRY_STATUS(W.alloc());
   TNLB_TRY_STATUS(ax.alloc(rs * (n > 0 ? n : 1)));
   TNLB_TRY_STATUS(spmv_dispatch(seg, real, cols, vals, x, ax.ptr, 1.0, 0.0, st));
   if (real == TNLB_F64)
      k_resid_norms<double><<<vec_grid(n), kRedThreads, 0, st>>>(n, (const double*)b, ax.as<double>(), W.red(),
                                                                  W.scratch.as<double>());
   else
      k_resid_norms<float><<<vec_grid(n), kRedThreads, 0, st>>>(n, (const float*)b, ax.as<float>(), W.red(),
                                                                 W.scratch.as<double>());
   TNLB_CHECK_LAUNCH();
   double h[2];
   TNLB_CUDA_TRY(cudaMemcpyAsync(h, W.scratch.ptr, sizeof(h), cudaMemcpyDeviceToHost, st));
   TNLB_CUDA_TRY(cudaStreamSynchronize(st));
   *out = std::sqrt(h[0]) / std::sqrt(h[1]);
   return TNLB_OK;
}

tnlb_status precond_create(int kind, const tnlb_segments* seg, tnlb_real real, const int32_t* cols, const void* vals,
                           cudaStream_t st, tnlb_precond** out)
{
   TNLB_REQUIRE(seg->n > 0, TNLB_ERR_INVALID_ARGUMENT, "Preconditioner::update: the matrix is empty");
   auto* P = new tnlb_precond();
   P->kind = kind;
   P->real = real;
   P->n = seg->n;
   tnlb_status s = TNLB_OK;
   if (kind == TNLB_PRECOND_JACOBI) {
      s = P->diag.alloc((real == TNLB_F64 ? 8 : 4) * (size_t)seg->n);
      if (s == TNLB_OK) {
         if (real == TNLB_F64)
            k_diag<double><<<grid_for(seg->n, 256), 256, 0, st>>>(view_of(seg), cols, (const double*)vals,
                                                                 P->diag.as<double>());
         else
            k_diag<float><<<grid_for(seg->n, 256), 256, 0, st>>>(view_of(seg), cols, (const float*)vals,
                                                                P->diag.as<float>());
         if (cudaGetLastError() != cudaSuccess) {
            set_error("Jacobi setup launch failed");
            s = TNLB_ERR_CUDA;
         }
      }
   }
   else if (kind == TNLB_PRECOND_ILU0)
      s = ilu0_create(seg, real, cols, vals, st, &P->ilu);
   else if (kind == TNLB_PRECOND_FSAI)
      s = fsai_create(seg, real, cols, vals, true, st, &P->fsai);
   else if (kind == TNLB_PRECOND_FSAI2) {
      s = fsai_create(seg, real, cols, vals, true, st, &P->fsai, true);
      P->kind = TNLB_PRECOND_FSAI;  // applied the same way: z = G_U (G_L r)
   }
   if (s != TNLB_OK) {
      delete P;
      return s;
   }
   *out = P;
   return TNLB_OK;
}

tnlb_status solve(tnlb_solver_kind solver, const tnlb_precond* P, const tnlb_solver_params& prm,
                  const tnlb_segments* seg, tnlb_real real, const int32_t* cols, const void* vals, const void* b,
                  void* x, cudaStream_t st, tnlb_solve_result* res)
{
   TNLB_REQUIRE(!P || P->real == real, TNLB_ERR_INVALID_ARGUMENT, "preconditioner real type differs from the matrix");
   TNLB_REQUIRE(!P || P->n == seg->n, TNLB_ERR_INVALID_ARGUMENT, "preconditioner size differs from the matrix");
   if (real == TNLB_F64)
      return solve_t<double>(solver, P, prm, seg, real, cols, (const double*)vals, (const double*)b, (double*)x, st,
                             res);
   return solve_t<float>(solver, P, prm, seg, real, cols, (const float*)vals, (const float*)b, (float*)x, st, res);
}

tnlb_status precond_apply(const tnlb_precond* P, const void* b, void* x, cudaStream_t st)
{
   if (P->real == TNLB_F64)
      TNLB_TRY_STATUS(view<double>(P).apply(P->n, (const double*)b, (double*)x, st));
   else
      TNLB_TRY_STATUS(view<float>(P).apply(P->n, (const float*)b, (float*)x, st));
   TNLB_CUDA_TRY(cudaStreamSynchronize(st));
   return TNLB_OK;
}

// FP32 inner Krylov solve inside FP64 iterative refinement.
tnlb_status solve_mixed_cg(const tnlb_segments* seg, const int32_t* cols, const double* vals, const double* b,
                           double* x, const tnlb_solver_params& prm, double inner_tol, int32_t max_outer,
                           cudaStream_t st, tnlb_solve_result* res, int32_t* inner_total, int32_t* outer,
                           int inner_kind, const tnlb_precond* inner_precond, int inner_solver)
{
   const int64_t n = seg->n;
   DeviceBuffer v32, r64, r32, d32, d64;
   TNLB_TRY_STATUS(v32.alloc(sizeof(float) * (seg->storage > 0 ? seg->storage : 1)));
   TNLB_TRY_STATUS(r64.alloc(sizeof(double) * n));
   TNLB_TRY_STATUS(r32.alloc(sizeof(float) * n));
   TNLB_TRY_STATUS(d32.alloc(sizeof(float) * n));
   k_convert<float, double><<<grid_for(seg->storage, 256 * 8), 256, 0, st>>>(seg->storage, vals, v32.as<float>());
   TNLB_CHECK_LAUNCH();
   Ctx<float> c32{seg, TNLB_F32, cols, v32.as<float>(), n, st};
   tnlb_precond* own = nullptr;
   if (!inner_precond) TNLB_TRY_STATUS(precond_create(inner_kind, seg, TNLB_F32, cols, v32.ptr, st, &own));
   struct Guard {
      tnlb_precond* p;
      ~Guard() { delete p; }
   } guard{own};
   const tnlb_precond* pobj = inner_precond ? inner_precond : own;
   TNLB_REQUIRE(pobj->real == TNLB_F32, TNLB_ERR_INVALID_ARGUMENT, "the inner preconditioner must be FP32");
   const Precond<float> P = view<float>(pobj);
   tnlb_solver_params ip = prm;
   ip.convergence_residue = inner_tol;
   *inner_total = 0;
   *outer = 0;
   double resid = 0;
   Work W;
   TNLB_TRY_STATUS(W.alloc());
   for (int o = 0; o <= max_outer; o++) {
      // A x in FP64; the residual norm computed as tnlb_true_residual does
      TNLB_TRY_STATUS(spmv_dispatch(seg, TNLB_F64, cols, vals, x, r64.ptr, 1.0, 0.0, st));
      k_resid_norms<double><<<vec_grid(n), kRedThreads, 0, st>>>(n, b, r64.as<double>(), W.red(),
                                                                  W.scratch.as<double>());
      TNLB_CHECK_LAUNCH();
      double h[2];
      TNLB_CUDA_TRY(cudaMemcpyAsync(h, W.scratch.ptr, sizeof(h), cudaMemcpyDeviceToHost, st));
      TNLB_CUDA_TRY(cudaStreamSynchronize(st));
      const double rn = std::sqrt(h[0]), bn = std::sqrt(h[1]);
      resid = bn > 0 ? rn / bn : 0.0;
      if (bn == 0 || resid < prm.convergence_residue || o == max_outer) break;
      // unit-norm FP32 residual, FP32 correction
      k_resid_to_f32<<<vec_grid(n), kRedThreads, 0, st>>>(n, b, r64.as<double>(), 1.0 / rn, r32.as<float>());
      TNLB_CUDA_TRY(cudaMemsetAsync(d32.ptr, 0, sizeof(float) * n, st));
      TNLB_CHECK_LAUNCH();
      tnlb_solve_result ir{};
      TNLB_TRY_STATUS(solve_t<float>((tnlb_solver_kind)inner_solver, pobj, ip, seg, TNLB_F32, cols, v32.as<float>(),
                                     r32.as<float>(), d32.as<float>(), st, &ir));
      *inner_total += ir.iterations;
      (*outer)++;
      // x += rn * d
      k_axpby_mixed<<<vec_grid(n), kRedThreads, 0, st>>>(n, rn, d32.as<float>(), x);
      TNLB_CHECK_LAUNCH();
   }
   res->iterations = *inner_total;
   res->residue = resid;
   res->converged = resid < prm.convergence_residue;
   res->status_detail = 0;
   return TNLB_OK;
}

namespace {

// State of the reliable-update PCG (solve_mixed_reliable).  `halt` stops the
// rest of a CUDA-graph batch: 1 a reliable update is due (the recursive
// |r|^2 below trig2, or the iteration force_at reached), 2 breakdown
// ((p, A p) zero or not finite), 3 the iteration limit.
struct RuState {
   double rz;     // (r, z) of the iteration whose alpha was formed last
   double alpha;
   double trig2;  // |r|^2 of the recursion below which an update is due
   double rr;     // |r|^2 after the last update of r
   int32_t it, halt, maxit, force_at;
   int32_t loops, pad;  // batches run by the device-side loop since k_ru_set
};

// Iterations after which an update is due whatever the recursive residual,
// so that the true residual of a recursion that stops falling is checked.
constexpr int32_t kRuForceEvery = 4096;

// (a, b) into *out, for matrices the fused product does not cover.
template <typename VT>
__global__ void __launch_bounds__(kRedThreads) k_ru_dot(int64_t n, const VT* __restrict__ a, const VT* __restrict__ b,
                                                        RedWork w, double* __restrict__ out,
                                                        const int32_t* __restrict__ skip)
{
   if (skip && *skip) return;
   double acc = 0;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
      acc += (double)a[i] * (double)b[i];
   double v[1] = {acc};
   if (publish_and_arrive<1>(v, w)) {
      double t[1];
      gather_totals<1>(t, w);
      if (threadIdx.x == 0) *out = t[0];
   }
}

// alpha = (r, z) / (p, A p) (a zero or non-finite (p, A p) is a breakdown:
// alpha 0, halt 2); xc += alpha p; r -= alpha Ap; |r|^2; and for Jacobi
// (mode 1) z = r / d with (r, z), for no preconditioner (mode 0)
// (r, z) = |r|^2, into *rz_cur.  Every block reads *rz_cur before the last
// block overwrites it; the last block keeps the old value in S->rz for
// beta, counts the iteration and raises `halt` when an update is due.
// Four consecutive entries of a 16-byte-aligned vector (the solver's own
// buffers): one float4 or two double2 accesses.
__device__ __forceinline__ void ld4(const float* p, float (&v)[4])
{
   const float4 t = *reinterpret_cast<const float4*>(p);
   v[0] = t.x;
   v[1] = t.y;
   v[2] = t.z;
   v[3] = t.w;
}
__device__ __forceinline__ void ld4(const double* p, double (&v)[4])
{
   const double2 a = *reinterpret_cast<const double2*>(p), b = *reinterpret_cast<const double2*>(p + 2);
   v[0] = a.x;
   v[1] = a.y;
   v[2] = b.x;
   v[3] = b.y;
}
__device__ __forceinline__ void st4(float* p, const float (&v)[4])
{
   *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
__device__ __forceinline__ void st4(double* p, const double (&v)[4])
{
   *reinterpret_cast<double2*>(p) = make_double2(v[0], v[1]);
   *reinterpret_cast<double2*>(p + 2) = make_double2(v[2], v[3]);
}

// One entry of k_ru_update.  The correction xc is FP64 for either vector
// type: summed in FP32, the small late steps of a long run between updates
// lose their low bits, and on high-contrast matrices that cost up to 1.7x
// the iterations (an emulation of the iteration on a 512^2 GRF problem:
// 10473 against 6258 with xc in FP64, 5785 all in FP64).  The product of
// the FP32 alpha and p is exact in FP64.
template <typename VT>
__device__ __forceinline__ void ru_entry(VT alpha, double& xc, VT& r, VT p, VT ap, float d, VT& z, int mode,
                                         double& rr, double& rzn)
{
   xc += (double)alpha * (double)p;
   r = r - alpha * ap;
   rr += (double)r * (double)r;
   if (mode == 1) {
      z = r / (VT)d;
      rzn += (double)r * (double)z;
   }
}

template <typename VT>
__global__ void __launch_bounds__(kRedThreads) k_ru_update(int64_t n, double* __restrict__ xc, VT* __restrict__ r,
                                                           const VT* __restrict__ p, const VT* __restrict__ Ap,
                                                           const float* __restrict__ d, VT* __restrict__ z, int mode,
                                                           RedWork w, RuState* S, double* __restrict__ rz_cur,
                                                           const double* __restrict__ pap)
{
   if (S->halt) return;
   const double rz = *rz_cur, t = *pap;
   const bool ok = t != 0.0 && isfinite(t);
   const VT alpha = ok ? (VT)(rz / t) : VT(0);
   double rr = 0, rzn = 0;
   const int64_t stride = (int64_t)gridDim.x * blockDim.x, tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   // four entries per thread and pass (16-byte loads), then the tail
   for (int64_t q = tid; q < n / 4; q += stride) {
      const int64_t i = 4 * q;
      double xv[4];
      VT rv[4], pv[4], av[4], zv[4];
      float dv[4] = {1.0f, 1.0f, 1.0f, 1.0f};
      ld4(xc + i, xv);
      ld4(r + i, rv);
      ld4(p + i, pv);
      ld4(Ap + i, av);
      if (mode == 1) ld4(d + i, dv);
#pragma unroll
      for (int k = 0; k < 4; k++) ru_entry(alpha, xv[k], rv[k], pv[k], av[k], dv[k], zv[k], mode, rr, rzn);
      st4(xc + i, xv);
      st4(r + i, rv);
      if (mode == 1) st4(z + i, zv);
   }
   for (int64_t i = 4 * (n / 4) + tid; i < n; i += stride) {
      double xv = xc[i];
      VT rv = r[i], zv = VT(0);
      ru_entry(alpha, xv, rv, p[i], Ap[i], mode == 1 ? d[i] : 1.0f, zv, mode, rr, rzn);
      xc[i] = xv;
      r[i] = rv;
      if (mode == 1) z[i] = zv;
   }
   double v[2] = {rr, rzn};
   if (publish_and_arrive<2>(v, w)) {
      double tt[2];
      gather_totals<2>(tt, w);
      if (threadIdx.x == 0) {
         S->rz = rz;
         S->alpha = (double)alpha;
         S->it++;
         S->rr = tt[0];
         if (mode != 2) *rz_cur = mode == 0 ? tt[0] : tt[1];
         if (!ok || !isfinite(tt[0]))
            S->halt = 2;
         else if (tt[0] < S->trig2 || S->it >= S->force_at)
            S->halt = 1;
         else if (S->it >= S->maxit)
            S->halt = 3;
      }
   }
}

// r - alpha Ap: one expression for the stored residual and for the copies
// of it that k_ru_g_update gathers, so that both round alike.
__device__ __forceinline__ float ru_rnext(float r, float alpha, float ap) { return r - alpha * ap; }

// The input of k_ru_g_update's product: r - alpha Ap at a column, or at four
// (16-byte-aligned) consecutive columns.
struct RuNextInput {
   const float* __restrict__ r;
   const float* __restrict__ Ap;
   float alpha;
   __device__ __forceinline__ float operator()(int32_t c) const
   {
      return ru_rnext(__ldg(r + c), alpha, __ldg(Ap + c));
   }
   __device__ __forceinline__ void quad(int32_t c, float (&o)[4]) const
   {
      float a[4], b[4];
      ld_quad(r + c, a);
      ld_quad(Ap + c, b);
#pragma unroll
      for (int k = 0; k < 4; k++) o[k] = ru_rnext(a[k], alpha, b[k]);
   }
};

// k_ru_update fused into the first FSAI factor product, on a compact copy
// of G (compact.cu): alpha = (r, z) / (p, A p) as k_ru_update
// forms it; rn = r - alpha Ap into the other residual buffer; t = G rn, each
// gathered rn[c] recomputed from r and Ap; |rn|^2 and (t, t) = (rn, M rn)
// reduced together.  The last block keeps k_ru_update's books and stores
// (t, t) as the new (r, z).  xc += alpha p is left to k_ru_gt_xpby, which
// reads p anyway -- or, when this iteration raises `halt`, to the fold of
// the reliable update (k_ru_fold_p).
template <typename Rows>
__global__ void __launch_bounds__(kRedThreads, Rows::kMinBlocks)
   k_ru_g_update(Rows G, const float* __restrict__ r, const float* __restrict__ Ap, float* __restrict__ rn,
                 float* __restrict__ t, int32_t n, RedWork w, RuState* S, double* __restrict__ rz_cur,
                 const double* __restrict__ pap)
{
   if (S->halt) return;
   const double rz = *rz_cur, tp = *pap;
   const bool ok = tp != 0.0 && isfinite(tp);
   const float alpha = ok ? (float)(rz / tp) : 0.0f;
   const RuNextInput rv{r, Ap, alpha};
   double rr = 0, tt = 0;
#pragma unroll 1
   for (int64_t base = G.first(); base < n; base += G.step()) {
      G.prefetch(base + G.step(), n);
      float s[Rows::kR];
      G.rows(base, n, rv, s);
      if constexpr (Rows::kQuad) {
         if (base + 3 < n) {
            float v[4];
            rv.quad((int32_t)base, v);
            *reinterpret_cast<float4*>(rn + base) = make_float4(v[0], v[1], v[2], v[3]);
            *reinterpret_cast<float4*>(t + base) = make_float4(s[0], s[1], s[2], s[3]);
#pragma unroll
            for (int k = 0; k < 4; k++) {
               rr += (double)v[k] * (double)v[k];
               tt += (double)s[k] * (double)s[k];
            }
            continue;
         }
      }
#pragma unroll
      for (int k = 0; k < Rows::kR; k++) {
         const int64_t i = G.row(base, k);
         if (i < n) {
            const float v = rv((int32_t)i);
            rn[i] = v;
            t[i] = s[k];
            rr += (double)v * (double)v;
            tt += (double)s[k] * (double)s[k];
         }
      }
   }
   double v[2] = {rr, tt};
   if (publish_and_arrive<2>(v, w)) {
      double tot[2];
      gather_totals<2>(tot, w);
      if (threadIdx.x == 0) {
         S->rz = rz;
         S->alpha = (double)alpha;
         S->it++;
         S->rr = tot[0];
         *rz_cur = tot[1];
         if (!ok || !isfinite(tot[0]))
            S->halt = 2;
         else if (tot[0] < S->trig2 || S->it >= S->force_at)
            S->halt = 1;
         else if (S->it >= S->maxit)
            S->halt = 3;
      }
   }
}

// p = G^T t + beta p (beta = (r, z)_new / (r, z)_old) on the compact copy of
// G^T, and xc += alpha p with the p that alpha was formed for.
template <typename Rows>
__global__ void __launch_bounds__(kRedThreads, Rows::kMinBlocks)
   k_ru_gt_xpby(Rows GT, const float* __restrict__ t, float* __restrict__ p, double* __restrict__ xc, int32_t n,
                const double* __restrict__ rz_cur, const RuState* S)
{
   if (S->halt) return;
   const float beta = (float)(*rz_cur / S->rz);
   const float alpha = (float)S->alpha;
   const PlainInput tv{t};
#pragma unroll 1
   for (int64_t base = GT.first(); base < n; base += GT.step()) {
      GT.prefetch(base + GT.step(), n);
      float s[Rows::kR];
      GT.rows(base, n, tv, s);
      if constexpr (Rows::kQuad) {
         if (base + 3 < n) {
            float4* pp = reinterpret_cast<float4*>(p + base);
            const float4 po = *pp;
            double xo[4];
            ld4(xc + base, xo);
            xo[0] += (double)alpha * (double)po.x;
            xo[1] += (double)alpha * (double)po.y;
            xo[2] += (double)alpha * (double)po.z;
            xo[3] += (double)alpha * (double)po.w;
            st4(xc + base, xo);
            *pp = make_float4(s[0] + beta * po.x, s[1] + beta * po.y, s[2] + beta * po.z, s[3] + beta * po.w);
            continue;
         }
      }
#pragma unroll
      for (int k = 0; k < Rows::kR; k++) {
         const int64_t i = GT.row(base, k);
         if (i < n) {
            const float po = p[i];
            xc[i] += (double)alpha * (double)po;
            p[i] = s[k] + beta * po;
         }
      }
   }
}

template <typename Rows>
void launch_ru_g_update(const Rows& G, const float* r, const float* Ap, float* rn, float* t, int32_t n, RedWork w,
                        RuState* S, double* rz_cur, const double* pap, cudaStream_t st)
{
   auto* k = k_ru_g_update<Rows>;
   const unsigned g = resident_grid((const void*)k, kRedThreads, n, Rows::kR);
   k<<<g, kRedThreads, 0, st>>>(G, r, Ap, rn, t, n, w, S, rz_cur, pap);
}

template <typename Rows>
void launch_ru_gt_xpby(const Rows& GT, const float* t, float* p, double* xc, int32_t n, const double* rz_cur,
                       const RuState* S, cudaStream_t st)
{
   auto* k = k_ru_gt_xpby<Rows>;
   const unsigned g = resident_grid((const void*)k, kRedThreads, n, Rows::kR);
   k<<<g, kRedThreads, 0, st>>>(GT, t, p, xc, n, rz_cur, S);
}

// k_ru_g_update on a diagonal copy of G with r and Ap staged by bulk copies
// (band.cuh): each gathered r - alpha Ap formed by ru_rnext from the staged
// entries, the row sums in the order of DiaRows / DiaRow1.  The own row's
// new residual comes from the band of offset 0.  A wait that gave up makes
// the block's sums NaN, which the last block turns into a breakdown.
template <typename TV, int D>
__global__ void __launch_bounds__(kBandBlock)
   k_band_g_update(const TV* __restrict__ vals, int64_t pitch, DiaOffsets o, BandPlan P, const float* __restrict__ r,
                   const float* __restrict__ Ap, float* __restrict__ rn, float* __restrict__ t, int32_t n,
                   int64_t npad, RedWork w, RuState* S, double* __restrict__ rz_cur, const double* __restrict__ pap)
{
   if (band_block_flag(&S->halt)) return;
   extern __shared__ __align__(128) unsigned char smem[];
   __shared__ __align__(8) uint64_t full[kBandStages], empty[kBandStages];
   const double rz = *rz_cur, tp = *pap;
   const bool okp = tp != 0.0 && isfinite(tp);
   const float alpha = okp ? (float)(rz / tp) : 0.0f;
   const float* const bin[2] = {r, Ap};
   const float* const oin[1] = {nullptr};
   const double* const din[1] = {nullptr};
   double rr = 0, tt = 0;
   const bool ok = band_loop<TV, D, 2, 0, 0>(smem, full, empty, P, vals, pitch, bin, oin, din, n, npad,
                                          [&](int64_t i0, const unsigned char* st) {
      const BandPtrs<TV, D, 2> B(st, P, o, i0, n);
      auto rows = [&](auto check) {
         constexpr bool C = decltype(check)::value;
#pragma unroll
         for (int q = 0; q < kBandRows; q++) {
            const int rl = q * kBandThreads;
            const int64_t i = i0 + threadIdx.x + rl;
            if (C && i >= n) break;
            float v[D], x[D];
#pragma unroll
            for (int j = 0; j < D; j++) {
               bool in = true;
               if (C) {
                  const int64_t c = i + o.o[j];
                  in = c >= 0 && c < n;
               }
               v[j] = in ? rel_to_f(B.v[j * kBandT + rl]) : 0.0f;
               x[j] = in ? ru_rnext(B.x[0][j][rl], alpha, B.x[1][j][rl]) : 0.0f;
            }
            float s = 0.0f;
#pragma unroll
            for (int j = 0; j < D; j++) s += v[j] * x[j];
            const float rv = ru_rnext(B.self[0][rl], alpha, B.self[1][rl]);
            rn[i] = rv;
            t[i] = s;
            rr += (double)rv * (double)rv;
            tt += (double)s * (double)s;
         }
      };
      if (B.interior)
         rows(std::false_type{});
      else
         rows(std::true_type{});
   });
   if (!ok) rr = __longlong_as_double(0x7ff8000000000000ll);
   double v[2] = {rr, tt};
   if (band_publish<2>(v, w)) {
      double tot[2];
      band_totals<2>(tot, w);
      if (threadIdx.x == 0) {
         S->rz = rz;
         S->alpha = (double)alpha;
         S->it++;
         S->rr = tot[0];
         *rz_cur = tot[1];
         if (!okp || !isfinite(tot[0]))
            S->halt = 2;
         else if (tot[0] < S->trig2 || S->it >= S->force_at)
            S->halt = 1;
         else if (S->it >= S->maxit)
            S->halt = 3;
      }
   }
}

// k_ru_gt_xpby on a diagonal copy of G^T: t staged by bands, the tile's own
// p and FP64 xc by bulk copies.  A wait that gave up raises a breakdown.
template <typename TV, int D>
__global__ void __launch_bounds__(kBandBlock)
   k_band_gt_xpby(const TV* __restrict__ vals, int64_t pitch, DiaOffsets o, BandPlan P, const float* __restrict__ t,
                  float* __restrict__ p, double* __restrict__ xc, int32_t n, int64_t npad,
                  const double* __restrict__ rz_cur, RuState* S)
{
   if (band_block_flag(&S->halt)) return;
   extern __shared__ __align__(128) unsigned char smem[];
   __shared__ __align__(8) uint64_t full[kBandStages], empty[kBandStages];
   const float beta = (float)(*rz_cur / S->rz);
   const float alpha = (float)S->alpha;
   const float* const bin[1] = {t};
   const float* const oin[1] = {p};
   const double* const din[1] = {xc};
   const bool ok = band_loop<TV, D, 1, 1, 1>(smem, full, empty, P, vals, pitch, bin, oin, din, n, npad,
                                          [&](int64_t i0, const unsigned char* st) {
      const BandPtrs<TV, D, 1> B(st, P, o, i0, n);
      auto rows = [&](auto check) {
         constexpr bool C = decltype(check)::value;
#pragma unroll
         for (int q = 0; q < kBandRows; q++) {
            const int rl = q * kBandThreads;
            const int64_t i = i0 + threadIdx.x + rl;
            if (C && i >= n) break;
            float v[D], x[D];
#pragma unroll
            for (int j = 0; j < D; j++) {
               bool in = true;
               if (C) {
                  const int64_t c = i + o.o[j];
                  in = c >= 0 && c < n;
               }
               v[j] = in ? rel_to_f(B.v[j * kBandT + rl]) : 0.0f;
               x[j] = in ? B.x[0][j][rl] : 0.0f;
            }
            float s = 0.0f;
#pragma unroll
            for (int j = 0; j < D; j++) s += v[j] * x[j];
            const float po = B.own[0][rl];
            xc[i] = B.ownd[rl] + (double)alpha * (double)po;
            p[i] = s + beta * po;
         }
      };
      if (B.interior)
         rows(std::false_type{});
      else
         rows(std::true_type{});
   });
   if (!ok && threadIdx.x == 0) S->halt = 2;
}

// The banded forms of launch_ru_g_update / launch_ru_gt_xpby on a
// band-capable diagonal copy (compact_band_capable) with FP16 values.
void launch_band_g_update(const CompactCopy& G, const float* r, const float* Ap, float* rn, float* t, int32_t n,
                          RedWork w, RuState* S, double* rz_cur, const double* pap, cudaStream_t st)
{
   const BandPlan P = band_plan(G.diag, G.width, (int)sizeof(__half), 2, 0);
   DiaOffsets o{};
   for (int j = 0; j < 8; j++) o.o[j] = G.diag[j];
   const int64_t npad = ((int64_t)n + 3) / 4 * 4;
   const size_t smem = (size_t)P.stages * P.bytes;
   TNLB_DIA_WIDTH(G.width, {
      auto* k = k_band_g_update<__half, D>;
      const unsigned grid = band_grid((const void*)k, smem, n, kRedMaxBlocks);
      k<<<grid, kBandBlock, smem, st>>>(G.vals.as<__half>(), G.pitch, o, P, r, Ap, rn, t, n, npad, w, S, rz_cur,
                                           pap);
   });
}

void launch_band_gt_xpby(const CompactCopy& GT, const float* t, float* p, double* xc, int32_t n, const double* rz_cur,
                         RuState* S, cudaStream_t st)
{
   const BandPlan P = band_plan(GT.diag, GT.width, (int)sizeof(__half), 1, 1, 1);
   DiaOffsets o{};
   for (int j = 0; j < 8; j++) o.o[j] = GT.diag[j];
   const int64_t npad = ((int64_t)n + 3) / 4 * 4;
   const size_t smem = (size_t)P.stages * P.bytes;
   TNLB_DIA_WIDTH(GT.width, {
      auto* k = k_band_gt_xpby<__half, D>;
      const unsigned grid = band_grid((const void*)k, smem, n, kRedMaxBlocks);
      k<<<grid, kBandBlock, smem, st>>>(GT.vals.as<__half>(), GT.pitch, o, P, t, p, xc, n, npad, rz_cur, S);
   });
}

// x += xc + alpha p, the step k_ru_gt_xpby skips when the iteration that
// formed alpha raised `halt` (alpha is 0 before the first iteration); xc = 0.
template <typename VT>
__global__ void k_ru_fold_p(int64_t n, double* __restrict__ xc, const VT* __restrict__ p, const RuState* S,
                            double* __restrict__ x)
{
   const VT alpha = (VT)S->alpha;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
      double xv = xc[i];
      xv += (double)alpha * (double)p[i];
      x[i] += xv;
      xc[i] = 0.0;
   }
}

// z and (r, z) from r alone (after a reliable update): mode 1 Jacobi, mode 0 none.
template <typename VT>
__global__ void __launch_bounds__(kRedThreads) k_ru_precond(int64_t n, const VT* __restrict__ r,
                                                            const float* __restrict__ d, VT* __restrict__ z, int mode,
                                                            RedWork w, double* __restrict__ rz_out)
{
   double rz = 0;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
      const VT ri = r[i];
      const VT zi = mode == 1 ? ri / (VT)d[i] : ri;
      if (mode == 1) z[i] = zi;
      rz += (double)ri * (double)zi;
   }
   double v[1] = {rz};
   if (publish_and_arrive<1>(v, w)) {
      double t[1];
      gather_totals<1>(t, w);
      if (threadIdx.x == 0) *rz_out = t[0];
   }
}

// p = z + beta p with beta = (r, z)_new / (r, z)_old.
template <typename VT>
__global__ void k_ru_p(int64_t n, VT* __restrict__ p, const VT* __restrict__ z, const double* __restrict__ rz_cur,
                       const RuState* S)
{
   if (S->halt) return;
   const VT beta = (VT)(*rz_cur / S->rz);
   const int64_t stride = (int64_t)gridDim.x * blockDim.x, tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
   for (int64_t q = tid; q < n / 4; q += stride) {
      VT pv[4], zv[4];
      ld4(p + 4 * q, pv);
      ld4(z + 4 * q, zv);
#pragma unroll
      for (int k = 0; k < 4; k++) pv[k] = zv[k] + beta * pv[k];
      st4(p + 4 * q, pv);
   }
   for (int64_t i = 4 * (n / 4) + tid; i < n; i += stride) p[i] = z[i] + beta * p[i];
}

// x += xc; xc = 0.
__global__ void k_ru_fold(int64_t n, double* __restrict__ xc, double* __restrict__ x)
{
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
      x[i] += xc[i];
      xc[i] = 0.0;
   }
}

// r = (VT)(b - ax) and the sums |b - ax|^2, |b|^2 (in the order
// k_resid_norms uses, so the residual equals tnlb_true_residual's).
template <typename VT>
__global__ void __launch_bounds__(kRedThreads) k_ru_resid(int64_t n, const double* __restrict__ b,
                                                          const double* __restrict__ ax, VT* __restrict__ r, RedWork w,
                                                          double* __restrict__ out)
{
   double a0 = 0, a1 = 0;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
      const double di = (double)b[i] - (double)ax[i];
      r[i] = (VT)di;
      a0 += di * di;
      a1 += (double)b[i] * (double)b[i];
   }
   double v[2] = {a0, a1};
   if (publish_and_arrive<2>(v, w)) {
      double t[2];
      gather_totals<2>(t, w);
      if (threadIdx.x == 0) {
         out[0] = t[0];
         out[1] = t[1];
      }
   }
}

__global__ void k_ru_set(RuState* S, double trig2)
{
   if (threadIdx.x != 0) return;
   S->trig2 = trig2;
   S->force_at = S->it + kRuForceEvery;
   S->halt = 0;
   S->loops = 0;
}

// Last node of the batch body under a conditional WHILE node: run the body
// again until the state halts (an update is due, a breakdown, the iteration
// limit), and at most `cap` times per launch whatever the state holds.
__global__ void k_ru_continue(cudaGraphConditionalHandle loop, RuState* S, int32_t cap)
{
   if (threadIdx.x != 0) return;
   const int32_t l = ++S->loops;
   cudaGraphSetConditional(loop, S->halt == 0 && l < cap ? 1u : 0u);
}

// The solver body for vectors of type VT (float: FP32 vectors; double: FP64
// vectors with the FP32 values); see solve_mixed_reliable.
template <typename VT>
tnlb_status reliable_t(const tnlb_segments* seg, const int32_t* cols, const double* vals, const double* b, double* x,
                       const tnlb_solver_params& prm, double delta, cudaStream_t st, tnlb_solve_result* res,
                       int32_t* updates, int inner_kind, const tnlb_precond* inner_precond)
{
   constexpr tnlb_real kVec = sizeof(VT) == 8 ? TNLB_F64 : TNLB_F32;
   const int64_t n = seg->n;
   // vectors hold a multiple of 4 entries: the bulk copies of the banded
   // kernels (band.cuh) read whole 16-byte groups
   const int64_t npad = (n + 3) / 4 * 4;
   DeviceBuffer v32, ax, r, z, p, Ap, xc, scal;
   TNLB_TRY_STATUS(v32.alloc(sizeof(float) * (seg->storage > 0 ? seg->storage : 1)));
   TNLB_TRY_STATUS(ax.alloc(sizeof(double) * n));
   TNLB_TRY_STATUS(r.alloc(sizeof(VT) * npad));
   TNLB_TRY_STATUS(z.alloc(sizeof(VT) * npad));
   TNLB_TRY_STATUS(p.alloc(sizeof(VT) * npad));
   TNLB_TRY_STATUS(Ap.alloc(sizeof(VT) * npad));
   TNLB_TRY_STATUS(xc.alloc(sizeof(double) * npad));  // the correction is FP64 (ru_entry)
   TNLB_TRY_STATUS(scal.alloc(sizeof(double) * 4));  // [0] (p, Ap), [1] (r, z), [2..3] residual sums
   k_convert<float, double><<<grid_for(seg->storage, 256 * 8), 256, 0, st>>>(seg->storage, vals, v32.as<float>());
   TNLB_CHECK_LAUNCH();
   tnlb_precond* own = nullptr;
   if (!inner_precond && inner_kind != TNLB_PRECOND_NONE)
      TNLB_TRY_STATUS(precond_create(inner_kind, seg, TNLB_F32, cols, v32.ptr, st, &own));
   struct Guard {
      tnlb_precond* p;
      ~Guard() { delete p; }
   } guard{own};
   const tnlb_precond* pobj = inner_precond ? inner_precond : own;
   TNLB_REQUIRE(!pobj || pobj->real == TNLB_F32, TNLB_ERR_INVALID_ARGUMENT, "the inner preconditioner must be FP32");
   TNLB_REQUIRE(!pobj || pobj->n == n, TNLB_ERR_INVALID_ARGUMENT, "preconditioner size differs from the matrix");
   TNLB_REQUIRE(!pobj || pobj->kind == TNLB_PRECOND_JACOBI || pobj->kind == TNLB_PRECOND_FSAI,
                TNLB_ERR_INVALID_ARGUMENT, "solve_mixed_reliable: the preconditioner must be Jacobi or FSAI");
   TNLB_REQUIRE(!pobj || pobj->kind != TNLB_PRECOND_FSAI || !fsai_two_factor(pobj->fsai), TNLB_ERR_INVALID_ARGUMENT,
                "solve_mixed_reliable: a two-factor FSAI is not symmetric");
   const int mode = !pobj ? 0 : pobj->kind == TNLB_PRECOND_JACOBI ? 1 : 2;
   const float* d = mode == 1 ? pobj->diag.as<float>() : nullptr;
   VT* zp = mode == 0 ? r.as<VT>() : z.as<VT>();
   const bool fused_a = spmv_dot_fusable(seg);
   const bool fused_m = mode == 2 && fsai_dot_fusable(pobj->fsai);
   TNLB_REQUIRE(mode != 2 || fused_m || kVec == TNLB_F32, TNLB_ERR_INVALID_ARGUMENT,
                "solve_mixed_reliable: FP64 vectors need an FSAI whose factors hold at most 16 entries per row");
   Work W;  // reductions of the vector kernels
   TNLB_TRY_STATUS(W.alloc());
   Work WA, WM;  // reductions of the fused products
   TNLB_TRY_STATUS(WA.alloc());
   TNLB_TRY_STATUS(WM.alloc());
   RuState* S = reinterpret_cast<RuState*>(W.S());
   static_assert(sizeof(RuState) <= sizeof(DevState), "RuState must fit the state buffer");
   double* pap = scal.as<double>();
   double* rz_cur = pap + 1;
   double* rsum = pap + 2;
   const int32_t* halt = &S->halt;
   const unsigned G = vec_grid(n);
   // grids of the per-iteration vector kernels: resident blocks only
   const unsigned Gu = resident_grid((const void*)k_ru_update<VT>, kRedThreads, n, 4);
   const unsigned Gp = resident_grid((const void*)k_ru_p<VT>, kRedThreads, n, 4);
   const unsigned Gd = resident_grid((const void*)k_ru_dot<VT>, kRedThreads, n, 4);
   const float* v32f = v32.as<float>();

   // FP32 vectors on stencil-like matrices: compact copies of A (FP32
   // values) and of the FSAI factors (FP16 values: M = G^T G stays symmetric
   // positive definite), by diagonal or with 16-bit column offsets
   // (compact.cu), which the FP32 products read instead of the 8-byte
   // entries
   CompactCopy cA, cG, cGT;
   const bool compact_dia = prm.reliable_layout != 1;
   if (kVec == TNLB_F32) {
      if (fused_a)
         TNLB_TRY_STATUS(compact_build(seg, cols, v32f, false, 1.0f, compact_dia, st, &cA,
                                       prm.reliable_operator == 0 ? vals : nullptr));
      if (fused_m) {
         // G and G^T in FP16 times one power of two (PCG's iterates do not
         // change when M is scaled), so that no entry overflows
         const FsaiView fv = fsai_view(pobj->fsai);
         float gs = 1.0f;
         TNLB_TRY_STATUS(half_scale((const float*)fv.gvals, fv.g->elements, st, &gs));
         TNLB_TRY_STATUS(compact_build(fv.g, fv.gcols, (const float*)fv.gvals, true, gs, compact_dia, st, &cG));
         if (cG.kind != CompactCopy::kNone)
            TNLB_TRY_STATUS(
               compact_build(fv.gt, fv.gtcols, (const float*)fv.gtvals, true, gs, compact_dia, st, &cGT));
      }
   }
   const bool cmp_a = cA.kind != CompactCopy::kNone;
   const bool cmp_m = cG.kind != CompactCopy::kNone && cGT.kind != CompactCopy::kNone;
   // FSAI factor copies of more than 5 diagonals stage their products'
   // operands by bulk copies (band.cuh): on the 2048^2 diffusion matrix
   // the iteration with the 7-diagonal level-1 factors took 99.7 against
   // 149.4 us.  Up to 5 diagonals the four-row register form (DiaRows)
   // measured as fast (3-diagonal factors: 87.6 against 88.1 us), and for
   // A (FP32 values) the register forms were faster: 788 against 901 ms on
   // the 256^3 7-point Jacobi solve.
   auto banded = [&](const CompactCopy& C) {
      return prm.reliable_layout == 0 && C.kind == CompactCopy::kDia && C.width > 5 && compact_band_capable(C);
   };
   const bool band_g = cmp_m && banded(cG), band_gt = cmp_m && banded(cGT);
   // with the compact FSAI copies the update of xc and r goes into the two
   // factor products (k_ru_g_update, k_ru_gt_xpby); the new residual goes
   // to the other of two buffers, iteration by iteration, and t = G r to a
   // buffer of its own
   const bool fused_u = cmp_m;
   DeviceBuffer r2, tb;
   if (fused_u) {
      TNLB_TRY_STATUS(r2.alloc(sizeof(float) * npad));
      TNLB_TRY_STATUS(tb.alloc(sizeof(float) * npad));
   }
   float* tvec = fused_u ? tb.as<float>() : mode == 2 ? (float*)fsai_view(pobj->fsai).tmp : nullptr;
   TNLB_REQUIRE(!fused_u || aligned16(tvec), TNLB_ERR_INVALID_ARGUMENT,
                "solve_mixed_reliable: the FSAI work vector must be 16-byte aligned");

   // z = M^-1 r, (r, z) into rz_cur and p = z + beta p (beta = (r, z) /
   // S->rz); a short-row symmetric FSAI does it in two fused products
   // (t = G r with (t, t) = (r, z); p = G^T t + beta p), z never stored
   auto precondition = [&](cudaStream_t s, const int32_t* skip) -> tnlb_status {
      if (cmp_m) {
         TNLB_TRY_STATUS(compact_spmv_dot(cG, (const float*)r.ptr, tvec, WM.partials.as<double>(),
                                          WM.counter.as<unsigned>(), rz_cur, s, skip, true));
         return compact_spmv_xpby(cGT, tvec, (float*)p.ptr, rz_cur, &S->rz, s, skip);
      }
      if (fused_m)
         return fsai_apply_dot_xpby(pobj->fsai, kVec, r.ptr, p.ptr, WM.partials.as<double>(),
                                    WM.counter.as<unsigned>(), rz_cur, &S->rz, s, skip);
      if (mode == 2) {
         TNLB_TRY_STATUS(fsai_apply(pobj->fsai, r.ptr, z.ptr, s, skip));
         k_ru_dot<VT><<<Gd, kRedThreads, 0, s>>>(n, r.as<VT>(), z.as<VT>(), WM.red(), rz_cur, skip);
      }
      k_ru_p<VT><<<Gp, kRedThreads, 0, s>>>(n, p.as<VT>(), zp, rz_cur, S);
      TNLB_CHECK_LAUNCH();
      return TNLB_OK;
   };
   auto iteration = [&](cudaStream_t s, int k) -> tnlb_status {
      if (cmp_a)
         TNLB_TRY_STATUS(compact_spmv_dot(cA, (const float*)p.ptr, (float*)Ap.ptr, WA.partials.as<double>(),
                                          WA.counter.as<unsigned>(), pap, s, halt, false));
      else if (fused_a)
         TNLB_TRY_STATUS(spmv_dot_mixed(seg, TNLB_F32, kVec, kVec, cols, v32f, p.ptr, Ap.ptr,
                                        WA.partials.as<double>(), WA.counter.as<unsigned>(), pap, s, halt, false));
      else {
         // FP32 vectors: the FP32 values; FP64 vectors: the caller's FP64 values
         if (kVec == TNLB_F32)
            TNLB_TRY_STATUS(spmv_dispatch(seg, TNLB_F32, cols, v32f, p.ptr, Ap.ptr, 1.0, 0.0, s, halt));
         else
            TNLB_TRY_STATUS(spmv_dispatch(seg, TNLB_F64, cols, vals, p.ptr, Ap.ptr, 1.0, 0.0, s, halt));
         k_ru_dot<VT><<<Gd, kRedThreads, 0, s>>>(n, p.as<VT>(), Ap.as<VT>(), WA.red(), pap, halt);
      }
      if (fused_u) {
         // even iterations r -> r2, odd ones r2 -> r: a batch (even) ends in r
         const float* rin = (const float*)(k & 1 ? r2.ptr : r.ptr);
         float* rout = (float*)(k & 1 ? r.ptr : r2.ptr);
         if (band_g)
            launch_band_g_update(cG, rin, (const float*)Ap.ptr, rout, tvec, (int32_t)n, W.red(), S, rz_cur, pap, s);
         else
            TNLB_COMPACT_ROWS(cG, __half,
                              launch_ru_g_update(rows_, rin, (const float*)Ap.ptr, rout, tvec, (int32_t)n, W.red(), S,
                                                 rz_cur, pap, s));
         TNLB_CHECK_LAUNCH();
         if (band_gt)
            launch_band_gt_xpby(cGT, tvec, (float*)p.ptr, xc.as<double>(), (int32_t)n, rz_cur, S, s);
         else
            TNLB_COMPACT_ROWS(cGT, __half,
                              launch_ru_gt_xpby(rows_, tvec, (float*)p.ptr, xc.as<double>(), (int32_t)n, rz_cur, S, s));
         TNLB_CHECK_LAUNCH();
         return TNLB_OK;
      }
      k_ru_update<VT><<<Gu, kRedThreads, 0, s>>>(n, xc.as<double>(), r.as<VT>(), p.as<VT>(), Ap.as<VT>(), d, z.as<VT>(),
                                                 mode, W.red(), S, rz_cur, pap);
      TNLB_CHECK_LAUNCH();
      return precondition(s, halt);
   };

   // initial state: it = 0, halt set until the first residual is in
   RuState s0{};
   s0.rz = 1.0;
   s0.maxit = prm.max_iterations;
   s0.halt = 1;
   TNLB_CUDA_TRY(cudaMemcpyAsync(S, &s0, sizeof(s0), cudaMemcpyHostToDevice, st));
   TNLB_CUDA_TRY(cudaMemsetAsync(p.ptr, 0, sizeof(VT) * n, st));
   TNLB_CUDA_TRY(cudaMemsetAsync(xc.ptr, 0, sizeof(double) * n, st));

   // CUDA graph of the iterations between updates, captured once on a side
   // stream
   const int kBatch = n < (1 << 22) ? 32 : 16;
   cudaStream_t cs;
   TNLB_CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
   struct StreamGuard {
      cudaStream_t s;
      ~StreamGuard()
      {
         cudaStreamSynchronize(s);
         cudaStreamDestroy(s);
      }
   } sguard{cs};
   cudaEvent_t ev;
   TNLB_CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
   TNLB_CUDA_TRY(cudaEventRecord(ev, st));
   TNLB_CUDA_TRY(cudaStreamWaitEvent(cs, ev, 0));
   cudaEventDestroy(ev);
   cudaGraph_t graph = nullptr;
   cudaGraphExec_t exec = nullptr;
   // The device repeats the batch and k_ru_continue until the state halts,
   // with no host round trip between batches: the state halts at the latest
   // kRuForceEvery iterations after k_ru_set, within kCap bodies. Otherwise
   // the batch alone is relaunched by the host; where its capture fails too,
   // the iterations are launched directly.
   const int32_t kCap = kRuForceEvery / kBatch + 2;
   const bool device_loop = build_iteration_graph(
      cs,
      [&](cudaStream_t s) {
         tnlb_status rc = TNLB_OK;
         for (int k = 0; k < kBatch && rc == TNLB_OK; k++) rc = iteration(s, k);
         return rc;
      },
      [&](cudaGraphConditionalHandle loop, cudaStream_t s) { k_ru_continue<<<1, 32, 0, s>>>(loop, S, kCap); },
      &graph, &exec);
   struct GraphGuard {  // released after the stream has drained
      cudaStream_t s;
      cudaGraph_t g;
      cudaGraphExec_t e;
      ~GraphGuard()
      {
         cudaStreamSynchronize(s);
         if (e) cudaGraphExecDestroy(e);
         if (g) cudaGraphDestroy(g);
      }
   } gguard{cs, graph, exec};
   // pinned copy of the state for reads that do not stall the stream
   struct Pinned {  // released after the stream has drained
      cudaStream_t s;
      RuState* p = nullptr;
      ~Pinned()
      {
         cudaStreamSynchronize(s);
         if (p) cudaFreeHost(p);
      }
   } hstate{cs};
   TNLB_CUDA_TRY(cudaMallocHost(&hstate.p, sizeof(RuState)));
   cudaEvent_t copied;
   TNLB_CUDA_TRY(cudaEventCreateWithFlags(&copied, cudaEventDisableTiming));
   struct EventGuard {
      cudaEvent_t e;
      ~EventGuard() { cudaEventDestroy(e); }
   } eguard{copied};
   auto launch_batch = [&]() -> tnlb_status {
      if (exec) {
         TNLB_CUDA_TRY(cudaGraphLaunch(exec, cs));
         return TNLB_OK;
      }
      for (int k = 0; k < kBatch; k++) TNLB_TRY_STATUS(iteration(cs, k));
      return TNLB_OK;
   };

   // The FP32 iteration has stalled when the true residual at the updates
   // has not halved within the last max(kStallWindow, iterations to the
   // last halving) iterations, or when it broke down or went non-finite;
   // the solve then finishes with FP64 Jacobi PCG from the x of the lowest
   // true residual so far (xbest).
   constexpr int32_t kStallWindow = 16384;
   DeviceBuffer xbest;
   TNLB_TRY_STATUS(xbest.alloc(sizeof(double) * n));
   double best = HUGE_VAL, lowest = HUGE_VAL;
   int32_t it_best = 0;
   bool stalled = false;

   *updates = 0;
   double resid = 0.0, bn = 0.0;
   RuState h{};
   bool converged = false;
   for (;;) {
      // reliable update: x += xc, r = b - A x in FP64, r = (VT) r
      if (fused_u)
         k_ru_fold_p<VT><<<G, kRedThreads, 0, cs>>>(n, xc.as<double>(), p.as<VT>(), S, x);
      else
         k_ru_fold<<<G, kRedThreads, 0, cs>>>(n, xc.as<double>(), x);
      TNLB_CHECK_LAUNCH();
      TNLB_TRY_STATUS(spmv_dispatch(seg, TNLB_F64, cols, vals, x, ax.ptr, 1.0, 0.0, cs));
      k_ru_resid<VT><<<G, kRedThreads, 0, cs>>>(n, b, ax.as<double>(), r.as<VT>(), W.red(), rsum);
      TNLB_CHECK_LAUNCH();
      double hs[2];
      TNLB_CUDA_TRY(cudaMemcpyAsync(hs, rsum, sizeof(hs), cudaMemcpyDeviceToHost, cs));
      TNLB_CUDA_TRY(cudaMemcpyAsync(&h, S, sizeof(h), cudaMemcpyDeviceToHost, cs));
      TNLB_CUDA_TRY(cudaStreamSynchronize(cs));
      const double rn = std::sqrt(hs[0]);
      bn = std::sqrt(hs[1]);
      resid = bn > 0 ? rn / bn : 0.0;
      if (bn == 0 || resid < prm.convergence_residue) {
         converged = true;
         break;
      }
      if (!std::isfinite(resid)) {
         stalled = true;
         break;
      }
      if (resid < lowest) {
         lowest = resid;
         TNLB_CUDA_TRY(cudaMemcpyAsync(xbest.ptr, x, sizeof(double) * n, cudaMemcpyDeviceToDevice, cs));
      }
      if (h.halt == 2) {
         stalled = true;
         break;
      }
      if (h.it >= prm.max_iterations) break;
      if (resid < 0.5 * best) {
         best = resid;
         it_best = h.it;
      }
      else if (h.it - it_best > std::max(kStallWindow, it_best)) {
         stalled = true;
         break;
      }
      if (h.it > 0) (*updates)++;
      const double t1 = delta * rn, t2 = prm.convergence_residue * bn;
      k_ru_set<<<1, 32, 0, cs>>>(S, t1 > t2 ? t1 * t1 : t2 * t2);
      // z = M^-1 r, (r, z), p = z + beta p with the kept direction
      if (mode != 2) {
         k_ru_precond<VT><<<G, kRedThreads, 0, cs>>>(n, r.as<VT>(), d, z.as<VT>(), mode, W.red(), rz_cur);
         TNLB_CHECK_LAUNCH();
      }
      TNLB_TRY_STATUS(precondition(cs, halt));
      if (device_loop) {
         // iterations until an update is due, looped on the device; the
         // next update reads the state it halted in
         TNLB_CUDA_TRY(cudaGraphLaunch(exec, cs));
         continue;
      }
      // iterations until an update is due, one batch queued ahead of the
      // host's check of the state (a batch after the halt skips itself)
      TNLB_TRY_STATUS(launch_batch());
      TNLB_CUDA_TRY(cudaMemcpyAsync(hstate.p, S, sizeof(RuState), cudaMemcpyDeviceToHost, cs));
      TNLB_CUDA_TRY(cudaEventRecord(copied, cs));
      for (;;) {
         TNLB_TRY_STATUS(launch_batch());
         TNLB_CUDA_TRY(cudaEventSynchronize(copied));
         h = *hstate.p;
         if (h.halt) break;
         TNLB_CUDA_TRY(cudaMemcpyAsync(hstate.p, S, sizeof(RuState), cudaMemcpyDeviceToHost, cs));
         TNLB_CUDA_TRY(cudaEventRecord(copied, cs));
      }
   }
   TNLB_CUDA_TRY(cudaStreamSynchronize(cs));
   const int32_t fp32_its = h.it;
   int32_t fb_its = 0;
   const bool fall_back = stalled && fp32_its < prm.max_iterations;
   const bool restore = stalled && lowest < HUGE_VAL && !(resid <= lowest);
   if (restore) {
      TNLB_CUDA_TRY(cudaMemcpyAsync(x, xbest.ptr, sizeof(double) * n, cudaMemcpyDeviceToDevice, cs));
      resid = lowest;
   }
   if (fall_back) {
      tnlb_precond* jac = nullptr;
      TNLB_TRY_STATUS(precond_create(TNLB_PRECOND_JACOBI, seg, TNLB_F64, cols, vals, cs, &jac));
      struct JGuard {
         tnlb_precond* p;
         ~JGuard() { delete p; }
      } jguard{jac};
      // CG stops on sqrt((r, M^-1 r)) / ||M^-1 b||, which on a badly scaled
      // matrix lies orders of magnitude away from the true residual: each
      // run that ends above the tolerance is followed by one from its x
      // with the stopping residue scaled by the gap it showed
      tnlb_solver_params p64 = prm;
      p64.min_iterations = 0;
      double tau = 0.5 * prm.convergence_residue;
      const Ctx<double> c64{seg, TNLB_F64, cols, vals, n, cs};
      for (int run = 0; run < 8 && fp32_its + fb_its < prm.max_iterations; run++) {
         p64.max_iterations = prm.max_iterations - fp32_its - fb_its;
         p64.convergence_residue = tau;
         tnlb_solve_result r64{};
         TNLB_TRY_STATUS(cg_solve<double>(c64, view<double>(jac), p64, b, x, &r64));
         fb_its += r64.iterations;
         TNLB_TRY_STATUS(true_residual(seg, TNLB_F64, cols, vals, b, x, cs, &resid));
         if (bn == 0 || resid < prm.convergence_residue || !std::isfinite(resid)) break;
         tau *= 0.5 * prm.convergence_residue / resid;
      }
      converged = bn == 0 || resid < prm.convergence_residue;
   }
   TNLB_CUDA_TRY(cudaStreamSynchronize(cs));
   res->iterations = fp32_its + fb_its;
   res->residue = resid;
   res->converged = converged ? 1 : 0;
   res->status_detail = fall_back ? 2 : stalled ? 1 : 0;
   res->fallback_iterations = fb_its;
   return TNLB_OK;
}

}  // namespace

// Mixed-precision PCG with reliable updates (G. L. G. Sleijpen, H. A. van der
// Vorst, "Reliable updated residuals in hybrid Bi-CG methods", Computing 56
// (1996); M. A. Clark et al., "Solving lattice QCD systems of equations using
// mixed precision solvers on GPUs", Comput. Phys. Commun. 181 (2010)).  CG
// iterates on an FP32 copy of the values (FP32 preconditioner), with FP32 or
// FP64 vectors and FP64 dot products; its correction xc is folded into the
// FP64 x and the residual replaced by the FP64 b - A x whenever the
// recursive |r| has fallen below max(delta |r_last update|, tol |b|).  The
// search direction p is kept across an update (beta = (r, z)_new /
// (r, z)_old), so the Krylov space is not restarted as it is by iterative
// refinement.
tnlb_status solve_mixed_reliable(const tnlb_segments* seg, const int32_t* cols, const double* vals, const double* b,
                                 double* x, const tnlb_solver_params& prm, double delta, tnlb_real vectors,
                                 cudaStream_t st, tnlb_solve_result* res, int32_t* updates, int inner_kind,
                                 const tnlb_precond* inner_precond)
{
   TNLB_REQUIRE(seg->n > 0, TNLB_ERR_INVALID_ARGUMENT, "solve_mixed_reliable: the matrix is empty");
   TNLB_REQUIRE(delta > 0.0 && delta < 1.0, TNLB_ERR_INVALID_ARGUMENT, "solve_mixed_reliable: delta must lie in (0, 1)");
   if (vectors == TNLB_F64)
      return reliable_t<double>(seg, cols, vals, b, x, prm, delta, st, res, updates, inner_kind, inner_precond);
   return reliable_t<float>(seg, cols, vals, b, x, prm, delta, st, res, updates, inner_kind, inner_precond);
}

}  // namespace tnlb

tnlb_precond::~tnlb_precond()
{
   if (ilu) tnlb::ilu0_destroy(ilu);
   if (fsai) tnlb::fsai_destroy(fsai);
}
