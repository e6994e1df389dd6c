// ref_cuda.cu -- a thin C-ABI driver over the REFERENCE's own CUDA backend:
// TNL's SparseMatrix< Real, Devices::Cuda, int, GeneralMatrix, Segments >::
// vectorProduct, compiled from its headers for sm_100a into
// oracle/_ref/libtnlref_cuda.so by oracle/Makefile (target ref_cuda), with
// the reference's own CUDA flags (--extended-lambda --expt-relaxed-constexpr
// --default-stream per-thread, cmake/cuda_flags.cmake).
//
// TEST INFRASTRUCTURE.  No algorithm lives here: the matrix is built by the
// reference's Host CSR and copied to the device by the reference's
// cross-format, cross-device operator=; every product is the reference's
// vectorProduct under its default LaunchConfiguration and under each entry
// of its reductionLaunchConfigurations list
// (Algorithms/Segments/ReductionLaunchConfigurations.h:26-145).  It gives
// the secondary GPU comparison: the reference's CUDA SpMV timed on the same
// B200 as the library's kernels.  The product never loads it.
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include <TNL/Algorithms/Segments/CSR.h>
#include <TNL/Algorithms/Segments/ReductionLaunchConfigurations.h>
#include <TNL/Algorithms/Segments/SlicedEllpack.h>
#include <TNL/Containers/Vector.h>
#include <TNL/Matrices/SparseMatrix.h>

using namespace TNL;
namespace Seg = TNL::Algorithms::Segments;

template< typename D, typename I, typename A >
using SellC = Seg::SlicedEllpack< D, I, A, Seg::ColumnMajorOrder, 32 >;

template< typename Real, typename Device, template< typename, typename, typename > class S >
using Mat = Matrices::SparseMatrix< Real, Device, int, Matrices::GeneralMatrix, S >;

namespace {

// Host CSR matrix from plain arrays, through setRowCapacities.
template< typename Real >
void
makeHostCSR( Mat< Real, Devices::Host, Seg::CSR >& A, int n, int ncols, const int* rowptr, const int* cols,
             const Real* vals )
{
   A.setDimensions( n, ncols );
   Containers::Vector< int, Devices::Host, int > caps( n );
   for( int i = 0; i < n; i++ )
      caps[ i ] = rowptr[ i + 1 ] - rowptr[ i ];
   A.setRowCapacities( caps );
   auto v = A.getValues().getView();
   auto c = A.getColumnIndexes().getView();
   for( int j = 0; j < rowptr[ n ]; j++ ) {
      v[ j ] = vals[ j ];
      c[ j ] = cols[ j ];
   }
}

// Mean milliseconds of one synchronous vectorProduct call (CUDA events on
// the per-thread default stream around `reps` back-to-back calls).
template< typename M, typename V, typename F >
double
timeCalls( M& D, V& xv, V& yv, int reps, F&& call )
{
   call( D, xv, yv );
   cudaDeviceSynchronize();
   cudaEvent_t e0, e1;
   cudaEventCreate( &e0 );
   cudaEventCreate( &e1 );
   cudaEventRecord( e0, cudaStreamPerThread );
   for( int r = 0; r < reps; r++ )
      call( D, xv, yv );
   cudaEventRecord( e1, cudaStreamPerThread );
   cudaEventSynchronize( e1 );
   float ms = 0;
   cudaEventElapsedTime( &ms, e0, e1 );
   cudaEventDestroy( e0 );
   cudaEventDestroy( e1 );
   return ms / reps;
}

template< typename Real, template< typename, typename, typename > class S >
int
spmvCuda( int n, int ncols, const int* rowptr, const int* cols, const Real* vals, const Real* x, Real* y, int reps,
          double* msDefault, double* msBest, char* bestName, int bestNameLen, double* msAll, int maxAll )
{
   Mat< Real, Devices::Host, Seg::CSR > H;
   makeHostCSR( H, n, ncols, rowptr, cols, vals );
   Mat< Real, Devices::Host, S > HS;
   HS = H;
   Mat< Real, Devices::Cuda, S > D;
   D = HS;
   Containers::Vector< Real, Devices::Cuda, int > xv( ncols ), yv( n );
   {
      Containers::Vector< Real, Devices::Host, int > xh( ncols );
      for( int i = 0; i < ncols; i++ )
         xh[ i ] = x[ i ];
      xv = xh;
   }
   *msDefault = timeCalls( D,
                           xv,
                           yv,
                           reps,
                           []( auto& A, auto& xx, auto& yy )
                           {
                              A.vectorProduct( xx, yy );
                           } );
   {
      Containers::Vector< Real, Devices::Host, int > yh( n );
      yh = yv;
      for( int i = 0; i < n; i++ )
         y[ i ] = yh[ i ];
   }
   *msBest = *msDefault;
   std::string best = "default";
   int k = 0;
   for( const auto& [ cfg, name ] : Seg::reductionLaunchConfigurations( D.getSegments() ) ) {
      // a configuration the reference refuses for this matrix (e.g. more
      // threads than its index type counts) is recorded as -1
      double ms = -1;
      try {
         ms = timeCalls( D,
                         xv,
                         yv,
                         reps,
                         [ &cfg = cfg ]( auto& A, auto& xx, auto& yy )
                         {
                            A.vectorProduct( xx, yy, 1, 0, 0, 0, cfg );
                         } );
      }
      catch( const std::exception& ) {
         ms = -1;
      }
      if( k < maxAll )
         msAll[ k ] = ms;
      k++;
      if( ms >= 0 && ms < *msBest ) {
         *msBest = ms;
         best = name;
      }
   }
   if( bestName && bestNameLen > 0 ) {
      std::strncpy( bestName, best.c_str(), bestNameLen - 1 );
      bestName[ bestNameLen - 1 ] = 0;
   }
   return k;
}

}  // namespace

extern "C" {

// fmt 0: CSR, 2: SlicedEllpack (column-major, slice 32).  x, y in host
// memory; y receives the default-configuration product.  Returns the number
// of launch configurations tried (their times in msAll, -1 for one the
// reference refused), or -1 on an error (message in err).
int
ref_cuda_spmv( int fmt, int real64, int n, int ncols, const int* rowptr, const int* cols, const void* vals,
               const void* x, void* y, int reps, double* msDefault, double* msBest, char* bestName, int bestNameLen,
               double* msAll, int maxAll, char* err, int errLen )
{
   try {
      if( real64 ) {
         if( fmt == 0 )
            return spmvCuda< double, Seg::CSR >( n, ncols, rowptr, cols, (const double*) vals, (const double*) x,
                                                 (double*) y, reps, msDefault, msBest, bestName, bestNameLen, msAll,
                                                 maxAll );
         return spmvCuda< double, SellC >( n, ncols, rowptr, cols, (const double*) vals, (const double*) x,
                                           (double*) y, reps, msDefault, msBest, bestName, bestNameLen, msAll,
                                           maxAll );
      }
      if( fmt == 0 )
         return spmvCuda< float, Seg::CSR >( n, ncols, rowptr, cols, (const float*) vals, (const float*) x,
                                             (float*) y, reps, msDefault, msBest, bestName, bestNameLen, msAll,
                                             maxAll );
      return spmvCuda< float, SellC >( n, ncols, rowptr, cols, (const float*) vals, (const float*) x, (float*) y, reps,
                                       msDefault, msBest, bestName, bestNameLen, msAll, maxAll );
   }
   catch( const std::exception& e ) {
      if( err && errLen > 0 ) {
         std::strncpy( err, e.what(), errLen - 1 );
         err[ errLen - 1 ] = 0;
      }
      return -1;
   }
}

}  // extern "C"
