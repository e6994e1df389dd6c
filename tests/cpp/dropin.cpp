// Drop-in check of include/tnlb/tnlb.hpp: code written against the
// reference's API (SparseMatrix, vectorProduct, CG + Diagonal) runs on the
// GPU through libtnlb200.so.  Prints "OK <iterations> <residue>" on success.
#include <cmath>
#include <cstdio>
#include <memory>

#include "tnlb/tnlb.hpp"

using namespace TNL;

int main()
{
   using Matrix = Matrices::SparseMatrix<double, Devices::Cuda, int, Matrices::GeneralMatrix,
                                         Algorithms::Segments::SlicedEllpack>;
   const int N = 64, n = N * N;
   std::vector<int> rp{0}, cols;
   std::vector<double> vals;
   for (int i = 0; i < n; i++) {
      const int iy = i / N, ix = i % N;
      auto add = [&](int c, double v) {
         cols.push_back(c);
         vals.push_back(v);
      };
      if (iy > 0) add(i - N, -1);
      if (ix > 0) add(i - 1, -1);
      add(i, 4);
      if (ix < N - 1) add(i + 1, -1);
      if (iy < N - 1) add(i + N, -1);
      rp.push_back((int)cols.size());
   }
   auto A = std::make_shared<Matrix>();
   A->setFromCSR(n, n, rp, cols, vals);
   // known answer: A * 1 = 4 - (number of neighbours)
   Containers::Vector<double> x(n, 1.0), y(n, -7.0);
   A->vectorProduct(x, y);
   std::vector<double> h = y.toHost();
   for (int i = 0; i < n; i++) {
      const int iy = i / N, ix = i % N;
      const int nb = (iy > 0) + (ix > 0) + (ix < N - 1) + (iy < N - 1);
      if (h[i] != 4.0 - nb) {
         std::printf("FAIL spmv row %d: %g\n", i, h[i]);
         return 1;
      }
   }
   // size mismatch -> std::invalid_argument, as in the reference
   try {
      Containers::Vector<double> bad(n + 1, 1.0);
      A->vectorProduct(bad, y);
      std::printf("FAIL no exception\n");
      return 1;
   }
   catch (const std::invalid_argument&) {
   }
   // getTransposition of the (symmetric-valued) Laplacian gives it back
   {
      Matrices::SparseMatrix<double, Devices::Cuda, int, Matrices::GeneralMatrix, Algorithms::Segments::CSR> T;
      T.getTransposition(*A, 2.0);
      std::vector<int> trp, tcols;
      std::vector<double> tvals;
      T.toHostCSR(trp, tcols, tvals);
      if (T.getRows() != n || trp != rp || tcols != cols) {
         std::printf("FAIL transposition pattern\n");
         return 1;
      }
      for (size_t k = 0; k < vals.size(); k++)
         if (tvals[k] != 2.0 * vals[k]) {
            std::printf("FAIL transposition value %zu\n", k);
            return 1;
         }
   }
   // save / load round trip through TNL's binary file, and the type check
   {
      const std::string path = "dropin_matrix.tnl";
      A->save(path);
      Matrix B;
      B.load(path);
      Containers::Vector<double> yb(n, 0.0);
      B.vectorProduct(x, yb);
      A->vectorProduct(x, y);
      if (yb.toHost() != y.toHost()) {
         std::printf("FAIL load product\n");
         return 1;
      }
      try {
         Matrices::SparseMatrix<float, Devices::Cuda, int, Matrices::GeneralMatrix, Algorithms::Segments::SlicedEllpack>
            C;
         C.load(path);
         std::printf("FAIL load of another type\n");
         return 1;
      }
      catch (const std::runtime_error&) {
      }
      std::remove(path.c_str());
   }
   // CG + Jacobi
   Solvers::Linear::CG<Matrix> solver;
   solver.setMatrix(A);
   auto P = std::make_shared<Solvers::Linear::Preconditioners::Diagonal<Matrix>>();
   P->update(A);
   solver.setPreconditioner(P);
   solver.setConvergenceResidue(1e-8);
   Containers::Vector<double> b(n, 1.0), sol(n, 0.0);
   const bool ok = solver.solve(b, sol);
   double tr = 0;
   tnlb::check(tnlb_true_residual(A->segments(), TNLB_F64, A->getColumnIndexes().getData(), A->getValues().getData(),
                                  b.getData(), sol.getData(), nullptr, &tr));
   if (!ok || tr > 1e-7) {
      std::printf("FAIL solve ok=%d residue=%g true=%g\n", ok, solver.getResidue(), tr);
      return 1;
   }
   std::printf("OK %d %.3e\n", solver.getIterations(), tr);
   return 0;
}
