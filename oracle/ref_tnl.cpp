// ref_tnl.cpp -- a thin C-ABI driver over the REFERENCE's own Host (OpenMP)
// implementation, compiled from its headers into oracle/_ref/libtnlref.so by
// oracle/Makefile.
//
// TEST INFRASTRUCTURE.  This file contains no algorithm: every call below
// goes to TNL's own templates (setSegmentsSizes, operator= across formats,
// vectorProduct, CG/BICGStab/GMRES solve with Diagonal/ILU0).  It exists to
// (1) pin the C restatement in tnl_oracle.c against the reference itself on
// the same seeded inputs, and (2) time the reference's CPU path as the
// baseline arm of bench.py.  The product never loads it.
#include <chrono>
#include <cstdint>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <vector>
#ifdef _OPENMP
   #include <omp.h>
#endif

#include <TNL/Algorithms/Segments/AdaptiveCSR.h>
#include <TNL/Algorithms/Segments/BiEllpack.h>
#include <TNL/Algorithms/Segments/CSR.h>
#include <TNL/Algorithms/Segments/ChunkedEllpack.h>
#include <TNL/Algorithms/Segments/Ellpack.h>
#include <TNL/Algorithms/Segments/SlicedEllpack.h>
#include <TNL/Config/ParameterContainer.h>
#include <TNL/Containers/Vector.h>
#include <TNL/Matrices/MatrixReader.h>
#include <TNL/Matrices/MatrixWriter.h>
#include <TNL/Matrices/SparseMatrix.h>
#include <TNL/Solvers/Linear/BICGStab.h>
#include <TNL/Solvers/Linear/BICGStabL.h>
#include <TNL/Solvers/Linear/IDRs.h>
#include <TNL/Solvers/Linear/TFQMR.h>
#include <TNL/Solvers/Linear/CG.h>
#include <TNL/Solvers/Linear/GMRES.h>
#include <TNL/Solvers/Linear/Preconditioners/Diagonal.h>
#include <TNL/Solvers/Linear/Preconditioners/ILU0.h>
#include <TNL/Solvers/Linear/Preconditioners/ILUT.h>

using namespace TNL;
namespace Seg = TNL::Algorithms::Segments;
using Host = Devices::Host;
using IVec = Containers::Vector< int, Host, int >;

template< typename D, typename I, typename A >
using EllR = Seg::Ellpack< D, I, A, Seg::RowMajorOrder, 32 >;
template< typename D, typename I, typename A >
using EllC = Seg::Ellpack< D, I, A, Seg::ColumnMajorOrder, 32 >;
template< typename D, typename I, typename A >
using SellR = Seg::SlicedEllpack< D, I, A, Seg::RowMajorOrder, 32 >;
template< typename D, typename I, typename A >
using SellC = Seg::SlicedEllpack< D, I, A, Seg::ColumnMajorOrder, 32 >;
template< typename D, typename I, typename A >
using ChellR = Seg::ChunkedEllpack< D, I, A, Seg::RowMajorOrder >;
template< typename D, typename I, typename A >
using ChellC = Seg::ChunkedEllpack< D, I, A, Seg::ColumnMajorOrder >;
template< typename D, typename I, typename A >
using BiellR = Seg::BiEllpack< D, I, A, Seg::RowMajorOrder, 32 >;
template< typename D, typename I, typename A >
using BiellC = Seg::BiEllpack< D, I, A, Seg::ColumnMajorOrder, 32 >;

template< typename Real, template< typename, typename, typename > class S >
using Mat = Matrices::SparseMatrix< Real, Host, int, Matrices::GeneralMatrix, S >;

// ILUT's factors are protected members; a derived class exposes them.
template< typename M >
struct ILUTAccess : public Solvers::Linear::Preconditioners::ILUT< M >
{
   using Base = Solvers::Linear::Preconditioners::ILUT< M >;
   using Base::L;
   using Base::U;
};

// ILUT parameters of the solver driver (precond 3): ilut-p, ilut-threshold.
static int g_ilutP = 0;
static double g_ilutTau = 1e-4;

template< typename M >
static void
setupILUT( Solvers::Linear::Preconditioners::ILUT< M >& P, int p, double tau )
{
   Config::ParameterContainer prm;
   prm.addParameter< int >( "ilut-p", p );
   prm.addParameter< double >( "ilut-threshold", tau );
   P.setup( prm );
}

static IVec
toVec( const int* p, int n )
{
   IVec v( n );
   for( int i = 0; i < n; i++ )
      v[ i ] = p[ i ];
   return v;
}

template< typename V >
static void
copyOut( const V& v, int* out )
{
   if( out )
      for( int i = 0; i < v.getSize(); i++ )
         out[ i ] = v[ i ];
}

enum { F_CSR = 0, F_ELL = 1, F_SELL = 2, F_CHELL = 3, F_BIELL = 4, F_ACSR = 5 };

extern "C" {

// ---------------------------------------------------------------- builders
int
ref_csr_build( const int* sizes, int n, int* offsets )
{
   Seg::CSR< Host, int > s;
   s.setSegmentsSizes( toVec( sizes, n ) );
   copyOut( s.getOffsets(), offsets );
   return 0;
}

int
ref_ellpack_build( const int* sizes, int n, int colmajor, int* segmentSize, int* alignedSize )
{
   try {
      if( colmajor ) {
         EllC< Host, int, Allocators::Host< int > > s;
         s.setSegmentsSizes( toVec( sizes, n ) );
         *segmentSize = s.getSegmentSize( 0 );
         *alignedSize = s.getAlignedSize();
      }
      else {
         EllR< Host, int, Allocators::Host< int > > s;
         s.setSegmentsSizes( toVec( sizes, n ) );
         *segmentSize = s.getSegmentSize( 0 );
         *alignedSize = s.getAlignedSize();
      }
   }
   catch( const std::overflow_error& ) {
      return 2;
   }
   return 0;
}

long
ref_sell_build( const int* sizes, int n, int* sliceOffsets, int* sliceSegmentSizes )
{
   SellC< Host, int, Allocators::Host< int > > s;
   s.setSegmentsSizes( toVec( sizes, n ) );
   IVec a;
   a = s.getSliceOffsetsView();
   copyOut( a, sliceOffsets );
   a = s.getSliceSegmentSizesView();
   copyOut( a, sliceSegmentSizes );
   return s.getStorageSize();
}

// Returns the number of slices; outputs may be null (count only).
int
ref_chell_build( const int* sizes,
                 int n,
                 int* sliceSize,
                 int* sliceChunkSize,
                 int* sliceFirst,
                 int* slicePointer,
                 int* segmentToChunk,
                 int* segmentToSlice,
                 int* segmentPointers,
                 int* chunksToSegments,
                 int* storageSize )
{
   ChellC< Host, int, Allocators::Host< int > > s;
   s.setSegmentsSizes( toVec( sizes, n ) );
   const int ns = s.getNumberOfSlices();
   if( sliceSize ) {
      auto slices = s.getSlicesView();
      for( int i = 0; i < ns; i++ ) {
         sliceSize[ i ] = slices[ i ].size;
         sliceChunkSize[ i ] = slices[ i ].chunkSize;
         sliceFirst[ i ] = slices[ i ].firstSegment;
         slicePointer[ i ] = slices[ i ].pointer;
      }
      IVec a;
      a = s.getSegmentToChunkMappingView();
      copyOut( a, segmentToChunk );
      a = s.getSegmentToSliceMappingView();
      copyOut( a, segmentToSlice );
      a = s.getSegmentPointersView();
      copyOut( a, segmentPointers );
      a = s.getChunksToSegmentsMappingView();
      copyOut( a, chunksToSegments );
      *storageSize = s.getStorageSize();
   }
   return ns;
}

long
ref_biell_build( const int* sizes, int n, int* perm, int* groupPointers )
{
   BiellC< Host, int, Allocators::Host< int > > s;
   s.setSegmentsSizes( toVec( sizes, n ) );
   IVec a;
   a = s.getSegmentsPermutationView();
   copyOut( a, perm );
   a = s.getGroupPointersView();
   copyOut( a, groupPointers );
   return s.getStorageSize();
}

// AdaptiveCSR descriptors for value size 2^sizeLog; outputs may be null.
// The reference leaves some fields uninitialised: blockSize/segmentsInBlock
// of LONG and closing descriptors (one-index constructor) and warpsCount of
// STREAM/VECTOR descriptors (the five-argument constructor); those fields
// are reported as 0.
long
ref_acsr_blocks( const int* sizes,
                 int n,
                 int sizeLog,
                 unsigned char* type,
                 int* first,
                 int* blockSize,
                 int* segsInBlock,
                 unsigned char* warpIdx,
                 unsigned char* warpsCount )
{
   Seg::AdaptiveCSR< Host, int > s;
   try {
      s.setSegmentsSizes( toVec( sizes, n ) );
   }
   catch( const std::exception& ) {
      // LONG blocks query the CUDA warp size (AdaptiveCSR.hpp:211-213), which
      // a build without a GPU backend cannot do.
      return -1;
   }
   const auto& blocks = s.getBlocks()[ sizeLog ];
   const long cnt = blocks.getSize();
   if( type )
      for( long i = 0; i < cnt; i++ ) {
         const auto& b = blocks[ i ];
         type[ i ] = (unsigned char) b.getType();
         first[ i ] = b.getFirstSegment();
         const bool closing = ( i == cnt - 1 );
         const bool full = ! closing && b.getType() != Seg::detail::Type::LONG;
         blockSize[ i ] = full ? b.getSize() : 0;
         segsInBlock[ i ] = full ? b.getSegmentsInBlock() : 0;
         warpIdx[ i ] = b.getWarpIdx();
         warpsCount[ i ] = ( closing || b.getType() == Seg::detail::Type::LONG ) ? b.getWarpsCount() : 0;
      }
   return cnt;
}

}  // extern "C"

// ------------------------------------------------------ matrices from CSR
template< typename Real >
static void
makeCSR( Mat< Real, Seg::CSR >& A, int n, int ncols, const int* rowptr, const int* cols, const Real* vals )
{
   A.setDimensions( n, ncols );
   IVec caps( n );
   for( int i = 0; i < n; i++ )
      caps[ i ] = rowptr[ i + 1 ] - rowptr[ i ];
   A.setRowCapacities( caps );
   auto v = A.getValues().getView();
   auto c = A.getColumnIndexes().getView();
   const int nnz = rowptr[ n ];
   for( int j = 0; j < nnz; j++ ) {
      v[ j ] = vals[ j ];
      c[ j ] = cols[ j ];
   }
}

template< typename Real, template< typename, typename, typename > class S, typename F >
static long
withFormat( int n, int ncols, const int* rowptr, const int* cols, const Real* vals, F&& f )
{
   Mat< Real, Seg::CSR > csr;
   makeCSR( csr, n, ncols, rowptr, cols, vals );
   Mat< Real, S > A;
   A = csr;
   return f( A );
}

template< typename Real, typename F >
static long
dispatch( int fmt, int colmajor, int n, int ncols, const int* rowptr, const int* cols, const Real* vals, F&& f )
{
   switch( fmt ) {
      case F_CSR:
         {
            Mat< Real, Seg::CSR > csr;
            makeCSR( csr, n, ncols, rowptr, cols, vals );
            return f( csr );
         }
      case F_ELL:
         return colmajor ? withFormat< Real, EllC >( n, ncols, rowptr, cols, vals, f )
                         : withFormat< Real, EllR >( n, ncols, rowptr, cols, vals, f );
      case F_SELL:
         return colmajor ? withFormat< Real, SellC >( n, ncols, rowptr, cols, vals, f )
                         : withFormat< Real, SellR >( n, ncols, rowptr, cols, vals, f );
      case F_CHELL:
         return colmajor ? withFormat< Real, ChellC >( n, ncols, rowptr, cols, vals, f )
                         : withFormat< Real, ChellR >( n, ncols, rowptr, cols, vals, f );
      case F_BIELL:
         return colmajor ? withFormat< Real, BiellC >( n, ncols, rowptr, cols, vals, f )
                         : withFormat< Real, BiellR >( n, ncols, rowptr, cols, vals, f );
      case F_ACSR:
         return withFormat< Real, Seg::AdaptiveCSR >( n, ncols, rowptr, cols, vals, f );
   }
   return -1;
}

template< typename Real >
static long
fillImpl( int fmt, int colmajor, int n, int ncols, const int* rowptr, const int* cols, const Real* vals, int* outCols,
          Real* outVals )
{
   try {
      return dispatch< Real >( fmt,
                               colmajor,
                               n,
                               ncols,
                               rowptr,
                               cols,
                               vals,
                               [ & ]( auto& A ) -> long
                               {
                                  const long storage = A.getValues().getSize();
                                  if( outCols )
                                     for( long g = 0; g < storage; g++ ) {
                                        outCols[ g ] = A.getColumnIndexes()[ g ];
                                        outVals[ g ] = A.getValues()[ g ];
                                     }
                                  return storage;
                               } );
   }
   catch( const std::overflow_error& ) {
      return -2;
   }
}

template< typename Real >
static double
spmvImpl( int fmt, int colmajor, int n, int ncols, const int* rowptr, const int* cols, const Real* vals, const Real* x,
          Real* y, double alpha, double beta, int begin, int end, int reps )
{
   double best = -1;
   dispatch< Real >( fmt,
                     colmajor,
                     n,
                     ncols,
                     rowptr,
                     cols,
                     vals,
                     [ & ]( auto& A ) -> long
                     {
                        Containers::Vector< Real, Host, int > xv( ncols ), yv( n );
                        for( int i = 0; i < ncols; i++ )
                           xv[ i ] = x[ i ];
                        for( int r = 0; r < reps; r++ ) {
                           for( int i = 0; i < n; i++ )
                              yv[ i ] = y[ i ];
                           auto t0 = std::chrono::steady_clock::now();
                           A.vectorProduct( xv, yv, (Real) alpha, (Real) beta, begin, end );
                           auto t1 = std::chrono::steady_clock::now();
                           const double dt = std::chrono::duration< double >( t1 - t0 ).count();
                           if( best < 0 || dt < best )
                              best = dt;
                        }
                        for( int i = 0; i < n; i++ )
                           y[ i ] = yv[ i ];
                        return 0;
                     } );
   return best;
}

extern "C" {

// Fill the format's value/column arrays through the reference's cross-format
// operator= from a CSR matrix.  Returns the storage size (outputs may be null),
// or -2 when the reference throws std::overflow_error.
long
ref_fill_f64( int fmt, int colmajor, int n, int ncols, const int* rowptr, const int* cols, const double* vals, int* outCols,
              double* outVals )
{
   return fillImpl< double >( fmt, colmajor, n, ncols, rowptr, cols, vals, outCols, outVals );
}

long
ref_fill_f32( int fmt, int colmajor, int n, int ncols, const int* rowptr, const int* cols, const float* vals, int* outCols,
              float* outVals )
{
   return fillImpl< float >( fmt, colmajor, n, ncols, rowptr, cols, vals, outCols, outVals );
}

// y = alpha*A*x + beta*y via SparseMatrix::vectorProduct, repeated `reps`
// times from the same input y; returns the best single-call time in seconds.
double
ref_spmv_f64( int fmt, int colmajor, int n, int ncols, const int* rowptr, const int* cols, const double* vals,
              const double* x, double* y, double alpha, double beta, int begin, int end, int reps )
{
   return spmvImpl< double >( fmt, colmajor, n, ncols, rowptr, cols, vals, x, y, alpha, beta, begin, end, reps );
}

double
ref_spmv_f32( int fmt, int colmajor, int n, int ncols, const int* rowptr, const int* cols, const float* vals,
              const float* x, float* y, double alpha, double beta, int begin, int end, int reps )
{
   return spmvImpl< float >( fmt, colmajor, n, ncols, rowptr, cols, vals, x, y, alpha, beta, begin, end, reps );
}

// vectorProduct of a symmetric CSR matrix (only the stored triangle given in
// rowptr/cols/vals) and transposedVectorProduct of a general CSR matrix,
// through the reference's Host code.  y is in/out.
void
ref_spmv_symmetric_f64( int n, const int* rowptr, const int* cols, const double* vals, const double* x, double* y,
                        double alpha, double beta, int begin, int end )
{
   using SM = Matrices::SparseMatrix< double, Host, int, Matrices::SymmetricMatrix, Seg::CSR >;
   SM A;
   A.setDimensions( n, n );
   IVec caps( n );
   for( int i = 0; i < n; i++ )
      caps[ i ] = rowptr[ i + 1 ] - rowptr[ i ];
   A.setRowCapacities( caps );
   auto v = A.getValues().getView();
   auto c = A.getColumnIndexes().getView();
   for( int j = 0; j < rowptr[ n ]; j++ ) {
      v[ j ] = vals[ j ];
      c[ j ] = cols[ j ];
   }
   Containers::Vector< double, Host, int > xv( n ), yv( n );
   for( int i = 0; i < n; i++ ) {
      xv[ i ] = x[ i ];
      yv[ i ] = y[ i ];
   }
   A.vectorProduct( xv, yv, alpha, beta, begin, end );
   for( int i = 0; i < n; i++ )
      y[ i ] = yv[ i ];
}

void
ref_spmv_transposed_f64( int n, int ncols, const int* rowptr, const int* cols, const double* vals, const double* x,
                         double* y, double alpha, double beta, int begin, int end )
{
   Mat< double, Seg::CSR > A;
   makeCSR( A, n, ncols, rowptr, cols, vals );
   Containers::Vector< double, Host, int > xv( n ), yv( ncols );
   for( int i = 0; i < n; i++ )
      xv[ i ] = x[ i ];
   for( int i = 0; i < ncols; i++ )
      yv[ i ] = y[ i ];
   A.transposedVectorProduct( xv, yv, alpha, beta, begin, end );
   for( int i = 0; i < ncols; i++ )
      y[ i ] = yv[ i ];
}

// SparseMatrix::getTransposition of a CSR matrix into a CSR matrix:
// B = mult * A^T (B has ncols rows); writes B's row pointer (ncols + 1),
// columns and values (B's storage, padding included).  Returns B's storage
// size.  Outputs may be null on a first, sizing call.
long
ref_transpose_f64( int n, int ncols, const int* rowptr, const int* cols, const double* vals, double mult, int* trowptr,
                   int* tcols, double* tvals )
{
   Mat< double, Seg::CSR > A, B;
   makeCSR( A, n, ncols, rowptr, cols, vals );
   B.getTransposition( A, mult );
   const auto& off = B.getSegments().getOffsets();
   const long storage = off[ ncols ];
   if( trowptr )
      for( int i = 0; i <= ncols; i++ )
         trowptr[ i ] = off[ i ];
   if( tcols && tvals )
      for( long j = 0; j < storage; j++ ) {
         tcols[ j ] = B.getColumnIndexes()[ j ];
         tvals[ j ] = B.getValues()[ j ];
      }
   return storage;
}

// SparseMatrix::save of a matrix of format `fmt` (organization per
// `colmajor`) built from CSR by the cross-format operator=, with FP64
// (real64 != 0) or FP32 values.  Returns 0, or -1 on an exception.
int
ref_save( int fmt, int colmajor, int real64, int n, int ncols, const int* rowptr, const int* cols, const double* vals,
          const char* path )
{
   try {
      if( real64 )
         return (int) dispatch< double >( fmt, colmajor, n, ncols, rowptr, cols, vals,
                                          [ & ]( auto& A ) -> long
                                          {
                                             A.save( path );
                                             return 0;
                                          } );
      std::vector< float > v32( rowptr[ n ] );
      for( int k = 0; k < rowptr[ n ]; k++ )
         v32[ k ] = (float) vals[ k ];
      return (int) dispatch< float >( fmt, colmajor, n, ncols, rowptr, cols, v32.data(),
                                      [ & ]( auto& A ) -> long
                                      {
                                         A.save( path );
                                         return 0;
                                      } );
   }
   catch( ... ) {
      return -1;
   }
}

// MatrixReader::readMtx into a general (symmetric == 0) or SymmetricMatrix
// CSR matrix on the host.  First call with null arrays returns the sizes in
// rows/columns/nnz; the second fills rowptr/cols/vals.  Returns 0, or -1
// with the exception's message in `err` (size errLen).
int
ref_mtx_read( const char* path, int symmetric, int* rows, int* columns, long* nnz, int* rowptr, int* cols, double* vals,
              char* err, int errLen )
{
   auto out = [ & ]( auto& A ) -> int
   {
      *rows = A.getRows();
      *columns = A.getColumns();
      const auto& off = A.getSegments().getOffsets();
      *nnz = off[ A.getRows() ];
      if( rowptr ) {
         for( int i = 0; i <= A.getRows(); i++ )
            rowptr[ i ] = off[ i ];
         for( long k = 0; k < *nnz; k++ ) {
            cols[ k ] = A.getColumnIndexes()[ k ];
            vals[ k ] = A.getValues()[ k ];
         }
      }
      return 0;
   };
   try {
      if( symmetric ) {
         Matrices::SparseMatrix< double, Host, int, Matrices::SymmetricMatrix, Seg::CSR > A;
         Matrices::MatrixReader< decltype( A ) >::readMtx( path, A );
         return out( A );
      }
      Mat< double, Seg::CSR > A;
      Matrices::MatrixReader< decltype( A ) >::readMtx( path, A );
      return out( A );
   }
   catch( const std::exception& e ) {
      std::strncpy( err, e.what(), errLen - 1 );
      err[ errLen - 1 ] = 0;
      return -1;
   }
}

// MatrixWriter::writeMtx of a general CSR matrix given by host arrays.
void
ref_mtx_write( const char* path, int n, int ncols, const int* rowptr, const int* cols, const double* vals )
{
   Mat< double, Seg::CSR > A;
   makeCSR( A, n, ncols, rowptr, cols, vals );
   Matrices::MatrixWriter< decltype( A ) >::writeMtx( path, A );
}

// Solve A x = b with TNL's CG (solver 0), BICGStab (1) or GMRES (2), with no
// preconditioner (0), Diagonal (1) or ILU0 (2).  gmresVariant: 2 MGS, 3 MGSR,
// 4 CWY.  x holds the initial guess on entry.  Returns 1 if solve() returned
// true, else 0; iterations, residue and wall seconds are written out.
int
ref_solve( int solver,
           int precond,
           int n,
           const int* rowptr,
           const int* cols,
           const double* vals,
           const double* b,
           double* x,
           double tol,
           int maxIterations,
           int gmresRestart,
           int gmresVariant,
           int bicgstabExact,
           int* iterations,
           double* residue,
           double* seconds )
{
   using M = Mat< double, Seg::CSR >;
   auto A = std::make_shared< M >();
   makeCSR( *A, n, n, rowptr, cols, vals );
   Containers::Vector< double, Host, int > bv( n ), xv( n );
   for( int i = 0; i < n; i++ ) {
      bv[ i ] = b[ i ];
      xv[ i ] = x[ i ];
   }
   auto run = [ & ]( auto& S ) -> int
   {
      S.setMatrix( A );
      S.setConvergenceResidue( tol );
      S.setMaxIterations( maxIterations );
      using P = typename std::remove_reference_t< decltype( S ) >::PreconditionerType;
      (void) sizeof( P* );
      std::shared_ptr< Solvers::Linear::Preconditioners::Diagonal< M > > jac;
      std::shared_ptr< Solvers::Linear::Preconditioners::ILU0< M > > ilu;
      std::shared_ptr< Solvers::Linear::Preconditioners::ILUT< M > > ilut;
      auto t0 = std::chrono::steady_clock::now();
      if( precond == 3 ) {
         ilut = std::make_shared< Solvers::Linear::Preconditioners::ILUT< M > >();
         setupILUT( *ilut, g_ilutP, g_ilutTau );
         ilut->update( A );
         S.setPreconditioner( ilut );
      }
      if( precond == 1 ) {
         jac = std::make_shared< Solvers::Linear::Preconditioners::Diagonal< M > >();
         jac->update( A );
         S.setPreconditioner( jac );
      }
      else if( precond == 2 ) {
         ilu = std::make_shared< Solvers::Linear::Preconditioners::ILU0< M > >();
         ilu->update( A );
         S.setPreconditioner( ilu );
      }
      const bool ok = S.solve( bv, xv );
      auto t1 = std::chrono::steady_clock::now();
      *seconds = std::chrono::duration< double >( t1 - t0 ).count();
      *iterations = S.getIterations();
      *residue = S.getResidue();
      return ok ? 1 : 0;
   };
   int ok = 0;
   if( solver == 0 ) {
      Solvers::Linear::CG< M > S;
      ok = run( S );
   }
   else if( solver == 1 ) {
      Solvers::Linear::BICGStab< M > S;
      Config::ParameterContainer p;
      p.addParameter< bool >( "bicgstab-exact-residue", bicgstabExact != 0 );
      S.setup( p );
      ok = run( S );
   }
   else {
      Solvers::Linear::GMRES< M > S;
      Config::ParameterContainer p;
      const char* names[] = { "CGS", "CGSR", "MGS", "MGSR", "CWY" };
      p.addParameter< String >( "gmres-variant", names[ gmresVariant ] );
      p.addParameter< int >( "gmres-restarting-min", gmresRestart );
      p.addParameter< int >( "gmres-restarting-max", gmresRestart );
      S.setup( p );
      ok = run( S );
   }
   for( int i = 0; i < n; i++ )
      x[ i ] = xv[ i ];
   return ok;
}

// Solve A x = b with TNL's TFQMR (solver 3), BICGStabL (4: param = ell,
// flag = bicgstab-exact-residue) or IDRs (5: param = s, flag =
// idr-residual-smoothing), with no preconditioner (0), Diagonal (1) or
// ILU0 (2).  Returns 1 if solve() returned true, 0 if false, -2 if it threw.
int
ref_solve_ext( int solver,
               int precond,
               int n,
               const int* rowptr,
               const int* cols,
               const double* vals,
               const double* b,
               double* x,
               double tol,
               int maxIterations,
               int param,
               int flag,
               int* iterations,
               double* residue,
               double* seconds )
{
   using M = Mat< double, Seg::CSR >;
   auto A = std::make_shared< M >();
   makeCSR( *A, n, n, rowptr, cols, vals );
   Containers::Vector< double, Host, int > bv( n ), xv( n );
   for( int i = 0; i < n; i++ ) {
      bv[ i ] = b[ i ];
      xv[ i ] = x[ i ];
   }
   auto run = [ & ]( auto& S ) -> int
   {
      S.setMatrix( A );
      S.setConvergenceResidue( tol );
      S.setMaxIterations( maxIterations );
      std::shared_ptr< Solvers::Linear::Preconditioners::Diagonal< M > > jac;
      std::shared_ptr< Solvers::Linear::Preconditioners::ILU0< M > > ilu;
      auto t0 = std::chrono::steady_clock::now();
      if( precond == 1 ) {
         jac = std::make_shared< Solvers::Linear::Preconditioners::Diagonal< M > >();
         jac->update( A );
         S.setPreconditioner( jac );
      }
      else if( precond == 2 ) {
         ilu = std::make_shared< Solvers::Linear::Preconditioners::ILU0< M > >();
         ilu->update( A );
         S.setPreconditioner( ilu );
      }
      int ok;
      try {
         ok = S.solve( bv, xv ) ? 1 : 0;
      }
      catch( const std::exception& ) {
         ok = -2;
      }
      auto t1 = std::chrono::steady_clock::now();
      *seconds = std::chrono::duration< double >( t1 - t0 ).count();
      *iterations = S.getIterations();
      *residue = S.getResidue();
      return ok;
   };
   int ok = 0;
   if( solver == 3 ) {
      Solvers::Linear::TFQMR< M > S;
      ok = run( S );
   }
   else if( solver == 4 ) {
      Solvers::Linear::BICGStabL< M > S;
      Config::ParameterContainer p;
      p.addParameter< int >( "bicgstab-ell", param );
      p.addParameter< bool >( "bicgstab-exact-residue", flag != 0 );
      S.setup( p );
      ok = run( S );
   }
   else {
      Solvers::Linear::IDRs< M > S;
      Config::ParameterContainer p;
      p.addParameter< int >( "idr-s", param );
      p.addParameter< bool >( "idr-residual-smoothing", flag != 0 );
      S.setup( p );
      ok = run( S );
   }
   for( int i = 0; i < n; i++ )
      x[ i ] = xv[ i ];
   return ok;
}

// Apply the preconditioner once: x = M^{-1} b (1 = Diagonal, 2 = ILU0).
int
ref_prec_apply( int n, const int* rowptr, const int* cols, const double* vals, int kind, const double* b, double* x )
{
   using M = Mat< double, Seg::CSR >;
   auto A = std::make_shared< M >();
   makeCSR( *A, n, n, rowptr, cols, vals );
   Containers::Vector< double, Host, int > bv( n ), xv( n );
   for( int i = 0; i < n; i++ )
      bv[ i ] = b[ i ];
   if( kind == 1 ) {
      Solvers::Linear::Preconditioners::Diagonal< M > P;
      P.update( A );
      P.solve( bv, xv );
   }
   else {
      Solvers::Linear::Preconditioners::ILU0< M > P;
      P.update( A );
      P.solve( bv, xv );
   }
   for( int i = 0; i < n; i++ )
      x[ i ] = xv[ i ];
   return 0;
}

void
ref_set_ilut( int p, double tau )
{
   g_ilutP = p;
   g_ilutTau = tau;
}

// ILUT::update on a CSR matrix: the factors L (unit lower, rows in order)
// and U (rows stored reversed: row N-1-i holds row i, its first entry the
// pivot), both CSR with their padding.  A first call with null outputs
// returns the sizes in lnnz / unnz.  Returns 0, or -1 on an exception.
int
ref_ilut_factor( int n, const int* rowptr, const int* cols, const double* vals, int p, double tau, long* lnnz,
                 long* unnz, int* lrp, int* lc, double* lv, int* urp, int* uc, double* uv )
{
   try {
      using M = Mat< double, Seg::CSR >;
      auto A = std::make_shared< M >();
      makeCSR( *A, n, n, rowptr, cols, vals );
      ILUTAccess< M > P;
      setupILUT( P, p, tau );
      P.update( A );
      const auto& lo = P.L.getSegments().getOffsets();
      const auto& uo = P.U.getSegments().getOffsets();
      *lnnz = lo[ n ];
      *unnz = uo[ n ];
      if( lrp ) {
         for( int i = 0; i <= n; i++ ) {
            lrp[ i ] = lo[ i ];
            urp[ i ] = uo[ i ];
         }
         for( long k = 0; k < *lnnz; k++ ) {
            lc[ k ] = P.L.getColumnIndexes()[ k ];
            lv[ k ] = P.L.getValues()[ k ];
         }
         for( long k = 0; k < *unnz; k++ ) {
            uc[ k ] = P.U.getColumnIndexes()[ k ];
            uv[ k ] = P.U.getValues()[ k ];
         }
      }
      return 0;
   }
   catch( ... ) {
      return -1;
   }
}

// ILUT::update then ILUT::solve once: x = M^{-1} b.
int
ref_ilut_apply( int n, const int* rowptr, const int* cols, const double* vals, int p, double tau, const double* b,
                double* x )
{
   try {
      using M = Mat< double, Seg::CSR >;
      auto A = std::make_shared< M >();
      makeCSR( *A, n, n, rowptr, cols, vals );
      Solvers::Linear::Preconditioners::ILUT< M > P;
      setupILUT( P, p, tau );
      P.update( A );
      Containers::Vector< double, Host, int > bv( n ), xv( n );
      for( int i = 0; i < n; i++ )
         bv[ i ] = b[ i ];
      P.solve( bv, xv );
      for( int i = 0; i < n; i++ )
         x[ i ] = xv[ i ];
      return 0;
   }
   catch( ... ) {
      return -1;
   }
}

void
ref_set_threads( int n )
{
#ifdef _OPENMP
   omp_set_num_threads( n );
#endif
}

int
ref_omp_threads()
{
#ifdef _OPENMP
   return omp_get_max_threads();
#else
   return 1;
#endif
}

}  // extern "C"
