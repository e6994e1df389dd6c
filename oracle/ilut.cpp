// ilut.cpp -- TEST INFRASTRUCTURE: restatement of the reference's ILUT
// factorisation (Solvers/Linear/Preconditioners/ILUT.hpp:27-258) for the
// tests; the product never loads it.
//
// Row i: w = A_i, W = its columns, tau_i = tau * sqrt(sum of w_j^2 in stored
// order); for k in W (ascending, W growing) with k < i: w_k /= a_kk (A's
// diagonal), dropped below tau_i, and if nonzero w -= w_k * U_k over U_k's
// stored entries (W extended); candidates |w_j| >= tau_i pushed in
// ascending j into max-heaps by magnitude for L (j < i) and U (j >= i),
// std::make_heap, then std::pop_heap while the pop count is below both
// (stored entries of A_i on that side) + p and the remaining heap size;
// the popped entries sorted by column form the rows of L and U.  The same
// standard-library heap routines as the reference, hence the same choice
// among equal magnitudes.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <set>
#include <vector>

namespace {

struct Entry {
   int32_t col;
   double val, mag;
};

}  // namespace

extern "C" {

// Factors as one CSR: row i holds its L entries then its U entries (columns
// ascending within each part, the first U entry the pivot).  A first call
// with null outputs returns the number of entries; rowptr has n + 1 slots.
long orc_ilut_factor(int32_t n, const int32_t* rowptr, const int32_t* cols, const double* vals, int32_t p, double tau,
                     int32_t* frowptr, int32_t* fcols, double* fvals)
{
   std::vector<std::vector<int32_t>> ucol(n);
   std::vector<std::vector<double>> uval(n);
   std::vector<double> diag(n, 0.0), w(n, 0.0);
   std::vector<int32_t> capL(n), capU(n);
   for (int32_t i = 0; i < n; i++) {
      int32_t l = 0, u = 0;
      for (int32_t q = rowptr[i]; q < rowptr[i + 1]; q++) {
         const int32_t c = cols[q];
         if (c < 0) continue;
         if (c < i) l++;
         else if (c < n) u++;
         if (c == i) diag[i] = vals[q];
      }
      capL[i] = l + p;
      capU[i] = u + p;
   }
   auto mag_less = [](const Entry& a, const Entry& b) { return a.mag < b.mag; };
   auto col_less = [](const Entry& a, const Entry& b) { return a.col < b.col; };
   long total = 0;
   if (frowptr) frowptr[0] = 0;
   for (int32_t i = 0; i < n; i++) {
      std::set<int32_t> W;
      double s = 0.0;
      for (int32_t q = rowptr[i]; q < rowptr[i + 1]; q++) {
         if (cols[q] < 0) break;
         w[cols[q]] = vals[q];
         s += w[cols[q]] * w[cols[q]];
         W.insert(cols[q]);
      }
      const double thr = tau * std::sqrt(s);
      for (auto it = W.begin(); it != W.end(); ++it) {
         const int32_t k = *it;
         if (k >= i) break;
         double f = w[k] / diag[k];
         if (std::fabs(f) < thr) f = 0.0;
         w[k] = f;
         if (f == 0.0) continue;
         for (size_t e = 0; e < ucol[k].size(); e++) {
            w[ucol[k][e]] -= f * uval[k][e];
            W.insert(ucol[k][e]);
         }
      }
      std::vector<Entry> hl, hu, kl, ku;
      for (int32_t j : W) {
         const double m = std::fabs(w[j]);
         if (m < thr) continue;
         if (j < i) hl.push_back({j, w[j], m});
         else hu.push_back({j, w[j], m});
      }
      std::make_heap(hl.begin(), hl.end(), mag_less);
      std::make_heap(hu.begin(), hu.end(), mag_less);
      for (int32_t c = 0; c < capL[i] && c < (int32_t)hl.size(); c++) {
         std::pop_heap(hl.begin(), hl.end(), mag_less);
         kl.push_back(hl.back());
         hl.pop_back();
      }
      for (int32_t c = 0; c < capU[i] && c < (int32_t)hu.size(); c++) {
         std::pop_heap(hu.begin(), hu.end(), mag_less);
         ku.push_back(hu.back());
         hu.pop_back();
      }
      std::sort(kl.begin(), kl.end(), col_less);
      std::sort(ku.begin(), ku.end(), col_less);
      for (const Entry& e : ku) {
         ucol[i].push_back(e.col);
         uval[i].push_back(e.val);
      }
      if (fcols)
         for (const auto* part : {&kl, &ku})
            for (const Entry& e : *part) {
               fcols[total] = e.col;
               fvals[total] = e.val;
               total++;
            }
      else
         total += (long)(kl.size() + ku.size());
      if (frowptr) frowptr[i + 1] = (int32_t)total;
      for (int32_t j : W) w[j] = 0.0;
   }
   return total;
}

// x = U^-1 L^-1 b for such factors (unit L; U divided by its first entry,
// 0 when a row of U is empty), in column order, without fused multiply-adds.
void orc_lu_apply(int32_t n, const int32_t* frowptr, const int32_t* fcols, const double* fvals, const double* b,
                  double* x)
{
   std::vector<int32_t> us(n);
   for (int32_t i = 0; i < n; i++) {
      int32_t q = frowptr[i];
      while (q < frowptr[i + 1] && fcols[q] < i) q++;
      us[i] = q;
   }
   for (int32_t i = 0; i < n; i++) {
      double xi = b[i];
      for (int32_t q = frowptr[i]; q < us[i]; q++) xi -= fvals[q] * x[fcols[q]];
      x[i] = xi;
   }
   for (int32_t i = n - 1; i >= 0; i--) {
      double xi = x[i];
      for (int32_t q = us[i] + 1; q < frowptr[i + 1]; q++) xi -= fvals[q] * x[fcols[q]];
      x[i] = xi / (us[i] < frowptr[i + 1] ? fvals[us[i]] : 0.0);
   }
}

}  // extern "C"
