// ilut.cu -- ILUT preconditioner (Preconditioners/ILUT.h, ILUT.hpp:27-258).
//
// The reference has ILUT on the host only ("ILUT is not implemented for
// CUDA", ILUT.h:148-170).  Here the factorisation runs on the host -- its
// dropping makes the pattern of row i depend on the values of the rows
// before it, a sequential walk over the rows -- and the factors are applied
// on the GPU by the level-scheduled, software-pipelined triangular solves of
// ILU(0) (ilu0.cu).
//
// Factorisation of row i, as ILUT.hpp:96-250 does it (dual threshold,
// Y. Saad, "Iterative Methods for Sparse Linear Systems", 2nd ed., 10.4):
//   w = A_i (dense work row), W = the set of its column indexes;
//   tau_i = tau * ||A_i||_2 (sum of squares in stored order);
//   for k in W, k < i, in ascending order (W grows while walked):
//      w_k = w_k / a_kk (the diagonal of A, 0 if absent); w_k = 0 if |w_k| < tau_i;
//      if w_k != 0: w_j -= w_k * U_kj for the stored U_k entries, W += {j};
//   the entries with |w_j| >= tau_i go to a max-heap by |w_j| for L (j < i)
//   or U (j >= i), pushed in ascending j; up to nL_i + p (nU_i + p) largest
//   are popped -- the loop runs while the pop count is below both the
//   capacity and the remaining heap size, so at most half the candidates
//   (rounded up) are kept, as the reference's loop does;
//   the kept entries, sorted by column, are row i of L and of U (the first
//   U entry is the pivot of the back substitution, TriangularSolve.h:81-101).
// nL_i / nU_i are the stored entries of A_i left of / from the diagonal.
// The heaps are std::make_heap / std::pop_heap, as in the reference, so
// equal magnitudes are chosen in the same order.
#include <algorithm>
#include <cmath>
#include <set>
#include <vector>

#include "internal.cuh"
#include "segview.cuh"

namespace tnlb {

namespace {

template <typename Real>
struct Cand {
   int32_t col;
   Real val;
   Real mag;
};

template <typename Real>
void ilut_host(int32_t n, const std::vector<int32_t>& rp, const std::vector<int32_t>& cols,
               const std::vector<Real>& vals, int32_t p, Real tau, std::vector<int32_t>& frp,
               std::vector<int32_t>& fcols, std::vector<Real>& fvals)
{
   // U rows as they are produced (columns ascending, values)
   std::vector<std::vector<int32_t>> ucol(n);
   std::vector<std::vector<Real>> uval(n);
   std::vector<Real> diag(n, Real(0));
   std::vector<int32_t> ncapL(n), ncapU(n);
   for (int32_t i = 0; i < n; i++) {
      int32_t nl = 0, nu = 0;
      for (int32_t q = rp[i]; q < rp[i + 1]; q++) {
         const int32_t c = cols[q];
         if (c < 0) continue;
         if (c < i)
            nl++;
         else if (c < n)
            nu++;
         if (c == i) diag[i] = vals[q];  // getElement(i, i): the stored entry, else 0
      }
      ncapL[i] = nl + p;
      ncapU[i] = nu + p;
   }
   std::vector<Real> w(n, Real(0));
   auto by_mag = [](const Cand<Real>& a, const Cand<Real>& b) { return a.mag < b.mag; };
   auto by_col = [](const Cand<Real>& a, const Cand<Real>& b) { return a.col < b.col; };
   std::vector<Cand<Real>> heapL, heapU, keepL, keepU;
   frp.assign((size_t)n + 1, 0);
   fcols.clear();
   fvals.clear();
   for (int32_t i = 0; i < n; i++) {
      std::set<int32_t> W;
      Real norm = 0;
      for (int32_t q = rp[i]; q < rp[i + 1]; q++) {
         const int32_t c = cols[q];
         if (c < 0) break;  // padding ends a row
         w[c] = vals[q];
         norm += w[c] * w[c];
         W.insert(c);
      }
      const Real tau_i = tau * std::sqrt(norm);
      for (auto it = W.begin(); it != W.end() && *it < i; ++it) {
         const int32_t k = *it;
         Real wk = w[k] / diag[k];
         if (std::abs(wk) < tau_i) wk = Real(0);
         w[k] = wk;
         if (wk != Real(0))
            for (size_t e = 0; e < ucol[k].size(); e++) {
               const int32_t j = ucol[k][e];
               w[j] -= wk * uval[k][e];
               W.insert(j);
            }
      }
      for (const int32_t j : W) {
         const Real m = std::abs(w[j]);
         if (m < tau_i) continue;
         (j < i ? heapL : heapU).push_back(Cand<Real>{j, w[j], m});
      }
      std::make_heap(heapL.begin(), heapL.end(), by_mag);
      std::make_heap(heapU.begin(), heapU.end(), by_mag);
      for (int32_t c = 0; c < ncapL[i] && c < (int32_t)heapL.size(); c++) {
         std::pop_heap(heapL.begin(), heapL.end(), by_mag);
         keepL.push_back(heapL.back());
         heapL.pop_back();
      }
      for (int32_t c = 0; c < ncapU[i] && c < (int32_t)heapU.size(); c++) {
         std::pop_heap(heapU.begin(), heapU.end(), by_mag);
         keepU.push_back(heapU.back());
         heapU.pop_back();
      }
      std::sort(keepL.begin(), keepL.end(), by_col);
      std::sort(keepU.begin(), keepU.end(), by_col);
      for (const auto& e : keepL) {
         fcols.push_back(e.col);
         fvals.push_back(e.val);
      }
      for (const auto& e : keepU) {
         fcols.push_back(e.col);
         fvals.push_back(e.val);
         ucol[i].push_back(e.col);
         uval[i].push_back(e.val);
      }
      frp[i + 1] = (int32_t)fcols.size();
      for (const int32_t j : W) w[j] = Real(0);
      heapL.clear();
      heapU.clear();
      keepL.clear();
      keepU.clear();
   }
}

template <typename Real>
tnlb_status ilut_create_t(const tnlb_segments* seg, tnlb_real real, const int32_t* cols, const Real* vals, int32_t p,
                          double tau, cudaStream_t st, void** out)
{
   const int32_t n = seg->n;
   DeviceBuffer drp, dc, dv;
   TNLB_TRY_STATUS(gather_csr(view_of(seg), real, cols, vals, drp, dc, dv, st));
   std::vector<int32_t> rp((size_t)n + 1);
   TNLB_CUDA_TRY(cudaMemcpyAsync(rp.data(), drp.ptr, sizeof(int32_t) * ((size_t)n + 1), cudaMemcpyDeviceToHost, st));
   TNLB_CUDA_TRY(cudaStreamSynchronize(st));
   const size_t nnz = (size_t)rp[n];
   std::vector<int32_t> hc(nnz);
   std::vector<Real> hv(nnz);
   if (nnz) {
      TNLB_CUDA_TRY(cudaMemcpyAsync(hc.data(), dc.ptr, sizeof(int32_t) * nnz, cudaMemcpyDeviceToHost, st));
      TNLB_CUDA_TRY(cudaMemcpyAsync(hv.data(), dv.ptr, sizeof(Real) * nnz, cudaMemcpyDeviceToHost, st));
   }
   TNLB_CUDA_TRY(cudaStreamSynchronize(st));
   std::vector<int32_t> frp, fc;
   std::vector<Real> fv;
   ilut_host<Real>(n, rp, hc, hv, p, (Real)tau, frp, fc, fv);
   return ilu_from_factors(real, n, frp, fc, fv.data(), st, out);
}

}  // namespace

tnlb_status ilut_create(const tnlb_segments* seg, tnlb_real real, const int32_t* cols, const void* vals, int32_t p,
                        double tau, cudaStream_t st, void** out)
{
   TNLB_REQUIRE(seg->n > 0, TNLB_ERR_INVALID_ARGUMENT, "ILUT::update: the matrix is empty");
   TNLB_REQUIRE(p >= 0, TNLB_ERR_INVALID_ARGUMENT, "ILUT: ilut-p must be non-negative");
   if (real == TNLB_F64) return ilut_create_t<double>(seg, real, cols, (const double*)vals, p, tau, st, out);
   return ilut_create_t<float>(seg, real, cols, (const float*)vals, p, tau, st, out);
}

}  // namespace tnlb
