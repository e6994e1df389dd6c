// Device-side assembly through the C++ drop-in layer: the 2D Laplace
// operator of the reference's sparse set-up benchmark
// (Documentation/UsersGuide/Matrices/SparseMatrixSetup_Benchmark.cpp) written
// by SparseMatrix::forElements with a device lambda, and by the library's
// compiled assembler (tnlb_matrix_assemble_laplace_2d) into a SlicedEllpack
// matrix; both checked against a host-built CSR of the same operator by a
// product with a known vector.  Prints "OK" on success.
#include <cmath>
#include <cstdio>
#include <vector>

#include "tnlb/tnlb.hpp"

using namespace TNL;
using Csr = Matrices::SparseMatrix<double, Devices::Cuda, int, Matrices::GeneralMatrix, Algorithms::Segments::CSR>;
using Sell =
   Matrices::SparseMatrix<double, Devices::Cuda, int, Matrices::GeneralMatrix, Algorithms::Segments::SlicedEllpack>;

int main()
{
   const int N = 37, n = N * N;
   // host reference: identity rows on the boundary, (1, 1, -4, 1, 1) inside
   std::vector<int> rp(1, 0), cols;
   std::vector<double> vals;
   for (int r = 0; r < n; r++) {
      const int i = r % N, j = r / N;
      if (i == 0 || j == 0 || i == N - 1 || j == N - 1) {
         cols.push_back(r);
         vals.push_back(1.0);
      }
      else {
         const int c[5] = {r - N, r - 1, r, r + 1, r + N};
         const double v[5] = {1.0, 1.0, -4.0, 1.0, 1.0};
         for (int k = 0; k < 5; k++) {
            cols.push_back(c[k]);
            vals.push_back(v[k]);
         }
      }
      rp.push_back((int)cols.size());
   }
   std::vector<double> x(n), yref(n, 0.0);
   for (int r = 0; r < n; r++) x[r] = std::sin(0.37 * r) + 0.1;
   for (int r = 0; r < n; r++)
      for (int k = rp[r]; k < rp[r + 1]; k++) yref[r] += vals[k] * x[cols[k]];
   Containers::Vector<double> dx(n), dy(n);
   dx.copyFromHost(x.data());
   std::vector<double> y(n);
   auto check = [&](const char* what) {
      dy.copyToHost(y.data());
      for (int r = 0; r < n; r++)
         if (std::fabs(y[r] - yref[r]) > 1e-12 * (1.0 + std::fabs(yref[r]))) {
            std::printf("FAIL %s row %d: %g != %g\n", what, r, y[r], yref[r]);
            return false;
         }
      return true;
   };

   // forElements with a device lambda on a CSR matrix of capacity 5 per row
   Csr A(n, n);
   A.setRowCapacities(std::vector<int>(n, 5));
   A.forAllElements([=] __host__ __device__(int row, int local, int& column, double& value) {
      const int i = row % N, j = row / N;
      if (i == 0 || j == 0 || i == N - 1 || j == N - 1) {
         if (local == 0) {
            column = row;
            value = 1.0;
         }
         return;  // the other slots stay padding
      }
      const int c[5] = {row - N, row - 1, row, row + 1, row + N};
      const double v[5] = {1.0, 1.0, -4.0, 1.0, 1.0};
      column = c[local];
      value = v[local];
   });
   A.vectorProduct(dx, dy);
   if (!check("forElements")) return 1;

   // the library's assembler into SlicedEllpack storage
   Sell B(n, n);
   B.setRowCapacities(std::vector<int>(n, 5));
   tnlb::check(tnlb_matrix_assemble_laplace_2d(B.segments(), TNLB_F64, N, B.getColumnIndexes().getData(),
                                               B.getValues().getData(), nullptr));
   B.vectorProduct(dx, dy);
   if (!check("assemble_laplace_2d")) return 1;

   // a non-CSR matrix refuses forElements (its rows are not contiguous)
   bool refused = false;
   try {
      B.forAllElements([] __host__ __device__(int, int, int&, double&) {});
   }
   catch (const std::invalid_argument&) {
      refused = true;
   }
   if (!refused) {
      std::printf("FAIL forElements on SlicedEllpack did not raise\n");
      return 1;
   }
   std::printf("OK\n");
   return 0;
}
