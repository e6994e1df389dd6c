// idrs_shadow.cpp -- test infrastructure (part of the oracle): the shadow
// space of IDR(s) drawn as IDRs::setSize does (Solvers/Linear/IDRs.hpp:270-300):
// std::mt19937 seeded 0, std::normal_distribution<double>(0, 1), s columns of
// length n in column-major order, then for each column i and each j < i the
// reference's update P_i = P_i - (P_i, P_j) (the scalar (P_i, P_j) subtracted
// from every entry) and P_i /= ||P_i||.  The draws depend on the C++ standard
// library, so this uses the same one as the reference build.
#include <cmath>
#include <cstdint>
#include <random>

extern "C" void orc_idrs_shadow(int32_t n, int32_t s, double* P)
{
   std::mt19937 rng;
   rng.seed(0);
   std::normal_distribution<double> dist(0, 1);
   for (int64_t i = 0; i < (int64_t)n * s; i++) P[i] = dist(rng);
   for (int i = 0; i < s; i++) {
      double* Pi = P + (int64_t)i * n;
      for (int j = 0; j < i; j++) {
         const double* Pj = P + (int64_t)j * n;
         double d = 0;
         for (int32_t q = 0; q < n; q++) d += Pi[q] * Pj[q];
         for (int32_t q = 0; q < n; q++) Pi[q] = Pi[q] - d;
      }
      double nn = 0;
      for (int32_t q = 0; q < n; q++) nn += Pi[q] * Pi[q];
      nn = std::sqrt(nn);
      for (int32_t q = 0; q < n; q++) Pi[q] = Pi[q] / nn;
   }
}
