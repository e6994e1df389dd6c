// tnlb.hpp -- C++ drop-in layer over libtnlb200.so (include/tnlb200.h).
//
// Mirrors the reference's API for the SpMV / Krylov path so that calling
// code changes only its includes and namespace:
//   TNL::Matrices::SparseMatrix< Real, Devices::Cuda, int, GeneralMatrix, Segments >
//        setDimensions, setRowCapacities, setFromCSR (the cross-format
//        operator= from a CSR matrix), forElements / forAllElements (device
//        lambdas, CSR storage; CUDA translation units only), vectorProduct,
//        transposedVectorProduct, getTransposition,
//        getRows, getColumns; MatrixType GeneralMatrix or SymmetricMatrix
//        (Matrices/SparseMatrix.h:41-57, SparseMatrixBase.h:1020-1035);
//   TNL::Algorithms::Segments::{CSR, Ellpack, SlicedEllpack, ChunkedEllpack,
//        BiEllpack, AdaptiveCSR}, LaunchConfiguration, ElementsOrganization;
//   TNL::Solvers::Linear::{CG, BICGStab, GMRES, TFQMR, BICGStabL, IDRs} (+ FGMRES) with setMatrix,
//        setPreconditioner, setup, setConvergenceResidue, setMaxIterations,
//        solve, getIterations, getResidue (Solvers/Linear/LinearSolver.h);
//   TNL::Solvers::Linear::Preconditioners::{Diagonal, ILU0} (+ FSAI) with
//        update and solve (Preconditioners/Preconditioner.h:96-110).
// Errors raise the reference's exception types: std::invalid_argument,
// std::overflow_error, tnlb::BackendRuntimeError (Backend/Macros.h:14-24).
// vectorProduct is synchronous on return, like the reference
// (Algorithms/Segments/detail/ReducingOperations_CSR.h:327).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "../tnlb200.h"

namespace tnlb {

class BackendRuntimeError : public std::runtime_error {
public:
   using std::runtime_error::runtime_error;
};

inline void check(tnlb_status s)
{
   if (s == TNLB_OK) return;
   const std::string msg = tnlb_last_error();
   switch (s) {
      case TNLB_ERR_INVALID_ARGUMENT: throw std::invalid_argument(msg);
      case TNLB_ERR_OVERFLOW: throw std::overflow_error(msg);
      case TNLB_ERR_NOT_IMPLEMENTED: throw std::logic_error("not implemented: " + msg);
      case TNLB_ERR_OUT_OF_MEMORY: throw std::bad_alloc();
      case TNLB_ERR_IO: throw std::runtime_error(msg);
      default: throw BackendRuntimeError(msg);
   }
}

inline void cuda_check(cudaError_t e)
{
   if (e != cudaSuccess) throw BackendRuntimeError(cudaGetErrorString(e));
}

template <typename Real>
constexpr tnlb_real real_code()
{
   static_assert(std::is_same<Real, double>::value || std::is_same<Real, float>::value, "FP64 or FP32 values");
   return std::is_same<Real, double>::value ? TNLB_F64 : TNLB_F32;
}

}  // namespace tnlb

namespace TNL {

namespace Devices {
struct Cuda {};
}  // namespace Devices

namespace Containers {

// Device vector (Containers/Vector.h subset): owns cudaMalloc'd memory.
template <typename Real, typename Device = Devices::Cuda, typename Index = int>
class Vector {
public:
   Vector() = default;
   explicit Vector(Index size) { setSize(size); }
   Vector(Index size, Real value)
   {
      setSize(size);
      setValue(value);
   }
   Vector(const Vector&) = delete;
   Vector& operator=(const Vector&) = delete;
   Vector(Vector&& o) noexcept : data_(o.data_), size_(o.size_)
   {
      o.data_ = nullptr;
      o.size_ = 0;
   }
   ~Vector() { reset(); }
   void reset()
   {
      if (data_) cudaFree(data_);
      data_ = nullptr;
      size_ = 0;
   }
   void setSize(Index size)
   {
      if (size == size_) return;
      reset();
      if (size > 0) tnlb::cuda_check(cudaMalloc(&data_, sizeof(Real) * (size_t)size));
      size_ = size;
   }
   void setValue(Real v)
   {
      std::vector<Real> h(size_, v);
      copyFromHost(h.data());
   }
   void copyFromHost(const Real* h)
   {
      if (size_) tnlb::cuda_check(cudaMemcpy(data_, h, sizeof(Real) * size_, cudaMemcpyHostToDevice));
   }
   void copyToHost(Real* h) const
   {
      if (size_) tnlb::cuda_check(cudaMemcpy(h, data_, sizeof(Real) * size_, cudaMemcpyDeviceToHost));
   }
   std::vector<Real> toHost() const
   {
      std::vector<Real> h(size_);
      copyToHost(h.data());
      return h;
   }
   Real getElement(Index i) const
   {
      Real v;
      tnlb::cuda_check(cudaMemcpy(&v, data_ + i, sizeof(Real), cudaMemcpyDeviceToHost));
      return v;
   }
   Index getSize() const { return size_; }
   Real* getData() { return data_; }
   const Real* getData() const { return data_; }

private:
   Real* data_ = nullptr;
   Index size_ = 0;
};

}  // namespace Containers

namespace Algorithms {
namespace Segments {

enum ElementsOrganization { ColumnMajorOrder = 0, RowMajorOrder = 1 };

// Segment formats (Algorithms/Segments/*.h); the template signature matches
// the reference's Segments< Device, Index, IndexAllocator > parameter.
template <typename Device, typename Index, typename IndexAllocator = void>
struct CSR {
   static constexpr tnlb_format format = TNLB_CSR;
};
template <typename Device, typename Index, typename IndexAllocator = void>
struct Ellpack {
   static constexpr tnlb_format format = TNLB_ELLPACK;
};
template <typename Device, typename Index, typename IndexAllocator = void>
struct SlicedEllpack {
   static constexpr tnlb_format format = TNLB_SLICED_ELLPACK;
};
template <typename Device, typename Index, typename IndexAllocator = void>
struct ChunkedEllpack {
   static constexpr tnlb_format format = TNLB_CHUNKED_ELLPACK;
};
template <typename Device, typename Index, typename IndexAllocator = void>
struct BiEllpack {
   static constexpr tnlb_format format = TNLB_BIELLPACK;
};
template <typename Device, typename Index, typename IndexAllocator = void>
struct AdaptiveCSR {
   static constexpr tnlb_format format = TNLB_ADAPTIVE_CSR;
};

enum class ThreadsToSegmentsMapping : std::uint8_t { Fixed, Warp, Block, BlockMerged, DynamicGrouping };

// Segments::LaunchConfiguration (Algorithms/Segments/LaunchConfiguration.h:18-86).
struct LaunchConfiguration {
   LaunchConfiguration() = default;
   LaunchConfiguration(ThreadsToSegmentsMapping m, int tps) : mapping(m) { setThreadsPerSegmentCount(tps); }
   void setThreadsPerSegmentCount(int tps)
   {
      if (tps > 0 && (tps & (tps - 1)) == 0)
         threadsPerSegmentCount = tps;
      else
         throw std::invalid_argument("Threads per segment count must be a positive power of two.");
   }
   ThreadsToSegmentsMapping mapping = ThreadsToSegmentsMapping::DynamicGrouping;
   int threadsPerSegmentCount = 1;
   tnlb_kernel kernel() const
   {
      switch (mapping) {
         case ThreadsToSegmentsMapping::Fixed: return threadsPerSegmentCount == 1 ? TNLB_KERNEL_SCALAR : TNLB_KERNEL_VECTOR;
         case ThreadsToSegmentsMapping::Warp:
         case ThreadsToSegmentsMapping::Block: return TNLB_KERNEL_VECTOR;
         default: return TNLB_KERNEL_DEFAULT;
      }
   }
   int tps() const
   {
      if (mapping == ThreadsToSegmentsMapping::Warp) return 32;
      if (mapping == ThreadsToSegmentsMapping::Fixed || mapping == ThreadsToSegmentsMapping::Block)
         return threadsPerSegmentCount;
      return 0;
   }
};

}  // namespace Segments
}  // namespace Algorithms

namespace Matrices {

struct GeneralMatrix {};
// MatrixType SymmetricMatrix (Matrices/MatrixType.h:48): one triangle stored.
struct SymmetricMatrix {};

#ifdef __CUDACC__
namespace detail {
// One thread per row of CSR storage: f(rowIdx, localIdx, columnIdx&, value&)
// on each of the row's slots (SparseMatrixBase::forElements).
template <typename Index, typename Real, typename F>
__global__ void for_elements_csr(const Index* __restrict__ offsets, Index begin, Index end, Index* cols, Real* vals,
                                 F f)
{
   const Index row = begin + (Index)(blockIdx.x * blockDim.x + threadIdx.x);
   if (row >= end) return;
   const Index b = offsets[row], e = offsets[row + 1];
   for (Index k = b; k < e; k++) f(row, k - b, cols[k], vals[k]);
}
}  // namespace detail
#endif

template <typename Real = double, typename Device = Devices::Cuda, typename Index = int,
          typename MatrixType = GeneralMatrix,
          template <typename, typename, typename> class Segments = Algorithms::Segments::CSR,
          Algorithms::Segments::ElementsOrganization Organization = Algorithms::Segments::ColumnMajorOrder>
class SparseMatrix {
   static_assert(std::is_same<Index, int>::value, "int32 indices");

public:
   using RealType = Real;
   using IndexType = Index;

   SparseMatrix() = default;
   SparseMatrix(Index rows, Index columns) { setDimensions(rows, columns); }
   SparseMatrix(const SparseMatrix&) = delete;
   SparseMatrix& operator=(const SparseMatrix&) = delete;
   ~SparseMatrix() { tnlb_segments_destroy(seg_); }

   void setDimensions(Index rows, Index columns)
   {
      if (rows < 0 || columns < 0) throw std::invalid_argument("negative matrix dimensions");
      rows_ = rows;
      columns_ = columns;
   }
   // SparseMatrix::setRowCapacities (SparseMatrix.hpp:303-325): values 0,
   // column indexes the padding index -1.
   void setRowCapacities(const std::vector<Index>& caps)
   {
      if ((Index)caps.size() != rows_)
         throw std::invalid_argument("setRowCapacities: the number of capacities does not match the number of rows");
      Containers::Vector<Index> d((Index)caps.size());
      d.copyFromHost(caps.data());
      tnlb_segments_destroy(seg_);
      seg_ = nullptr;
      tnlb::check(tnlb_segments_create(Segments<Device, Index, void>::format, (tnlb_organization)Organization,
                                       d.getData(), rows_, nullptr, &seg_));
      tnlb_segments_info info;
      tnlb::check(tnlb_segments_get_info(seg_, &info));
      values_.setSize((Index)info.storage);
      columns_idx_.setSize((Index)info.storage);
      values_.setValue(Real(0));
      columns_idx_.setValue(-1);
   }
   // The cross-format operator= (SparseOperations.hpp:106-186) from a host
   // CSR matrix: capacities = row lengths, zeros and padding dropped.
   void setFromCSR(Index rows, Index columns, const std::vector<Index>& rowptr, const std::vector<Index>& cols,
                   const std::vector<Real>& vals)
   {
      setDimensions(rows, columns);
      std::vector<Index> caps(rows);
      for (Index i = 0; i < rows; i++) caps[i] = rowptr[i + 1] - rowptr[i];
      setRowCapacities(caps);
      Containers::Vector<Index> drp(rows + 1), dc((Index)cols.size());
      Containers::Vector<Real> dv((Index)vals.size());
      drp.copyFromHost(rowptr.data());
      dc.copyFromHost(cols.data());
      dv.copyFromHost(vals.data());
      tnlb::check(tnlb_matrix_fill_from_csr(seg_, tnlb::real_code<Real>(), drp.getData(), dc.getData(), dv.getData(),
                                            columns_idx_.getData(), values_.getData(), nullptr));
   }
   // y = matrixMultiplicator * A x + outVectorMultiplicator * y on rows [begin, end)
   // (SparseMatrixBase.h:1020-1035); end == 0 means all rows.  Synchronous.
   template <typename InVector, typename OutVector>
   void vectorProduct(const InVector& in, OutVector& out, Real matrixMultiplicator = 1, Real outVectorMultiplicator = 0,
                      Index begin = 0, Index end = 0,
                      const Algorithms::Segments::LaunchConfiguration& lc = {}) const
   {
      if (in.getSize() != columns_)
         throw std::invalid_argument("vectorProduct: size of the input vector does not match the number of matrix columns");
      if (out.getSize() != rows_)
         throw std::invalid_argument("vectorProduct: size of the output vector does not match the number of matrix rows");
      if (std::is_same<MatrixType, SymmetricMatrix>::value)
         tnlb::check(tnlb_spmv_symmetric(seg_, tnlb::real_code<Real>(), columns_idx_.getData(), values_.getData(),
                                         in.getData(), out.getData(), matrixMultiplicator, outVectorMultiplicator,
                                         begin, end, nullptr));
      else
         tnlb::check(tnlb_spmv(seg_, tnlb::real_code<Real>(), columns_idx_.getData(), values_.getData(), columns_,
                               in.getData(), out.getData(), matrixMultiplicator, outVectorMultiplicator, begin, end,
                               lc.kernel(), lc.tps(), nullptr));
      tnlb::cuda_check(cudaStreamSynchronize(nullptr));
   }
   // y = matrixMultiplicator * A^T x + outVectorMultiplicator * y on columns
   // [begin, end) (SparseMatrixBase.hpp:542-588); symmetric matrices use
   // vectorProduct.  Synchronous.
   template <typename InVector, typename OutVector>
   void transposedVectorProduct(const InVector& in, OutVector& out, Real matrixMultiplicator = 1,
                                Real outVectorMultiplicator = 0, Index begin = 0, Index end = 0) const
   {
      if (in.getSize() != rows_)
         throw std::invalid_argument(
            "transposedVectorProduct: size of the input vector does not match the number of matrix rows");
      if (out.getSize() != columns_)
         throw std::invalid_argument(
            "transposedVectorProduct: size of the output vector does not match the number of matrix columns");
      if (std::is_same<MatrixType, SymmetricMatrix>::value) {
         vectorProduct(in, out, matrixMultiplicator, outVectorMultiplicator, begin, end);
         return;
      }
      tnlb::check(tnlb_spmv_transposed(seg_, tnlb::real_code<Real>(), columns_idx_.getData(), values_.getData(),
                                       columns_, in.getData(), out.getData(), matrixMultiplicator,
                                       outVectorMultiplicator, begin, end, nullptr));
      tnlb::cuda_check(cudaStreamSynchronize(nullptr));
   }
   // SparseMatrix::getTransposition (SparseMatrix.hpp:495-551): this matrix
   // becomes matrixMultiplicator * matrix^T (any format of `matrix`, same
   // real type), the rows in ascending column order.  Filled through the
   // cross-format assignment: an explicitly stored zero leaves a padding slot.
   template <typename Matrix2>
   void getTransposition(const Matrix2& matrix, Real matrixMultiplicator = 1)
   {
      static_assert(std::is_same<typename Matrix2::RealType, Real>::value, "getTransposition: same real type");
      const Index nt = matrix.getColumns();
      Containers::Vector<Index> trp(nt + 1);
      int64_t nnz = 0;
      tnlb::check(tnlb_matrix_transpose_rowptr(matrix.segments(), matrix.getColumnIndexes().getData(), nt,
                                               trp.getData(), &nnz, nullptr));
      Containers::Vector<Index> tc((Index)(nnz > 0 ? nnz : 1));
      Containers::Vector<Real> tv((Index)(nnz > 0 ? nnz : 1));
      tnlb::check(tnlb_matrix_transpose_fill(matrix.segments(), tnlb::real_code<Real>(),
                                             matrix.getColumnIndexes().getData(), matrix.getValues().getData(), nt,
                                             (double)matrixMultiplicator, tc.getData(), tv.getData(), nullptr));
      std::vector<Index> hrp(nt + 1), caps(nt);
      trp.copyToHost(hrp.data());
      for (Index i = 0; i < nt; i++) caps[i] = hrp[i + 1] - hrp[i];
      setDimensions(nt, matrix.getRows());
      setRowCapacities(caps);
      tnlb::check(tnlb_matrix_fill_from_csr(seg_, tnlb::real_code<Real>(), trp.getData(), tc.getData(), tv.getData(),
                                            columns_idx_.getData(), values_.getData(), nullptr));
      tnlb::cuda_check(cudaStreamSynchronize(nullptr));
   }
   // The matrix type string of TNL's binary file (SparseMatrixBase.hpp:46-53).
   static std::string getSerializationType()
   {
      const tnlb_format f = Segments<Device, Index, void>::format;
      const std::string org = Organization == Algorithms::Segments::RowMajorOrder ? "RowMajorOrder" : "ColumnMajorOrder";
      std::string seg;
      switch (f) {
         case TNLB_CSR: seg = "CSR< int >"; break;
         case TNLB_ADAPTIVE_CSR: seg = "AdaptiveCSR< int >"; break;
         case TNLB_ELLPACK: seg = "Ellpack< int, " + org + ", 32 >"; break;
         case TNLB_SLICED_ELLPACK: seg = "SlicedEllpack< int, " + org + ", 32 >"; break;
         case TNLB_CHUNKED_ELLPACK: seg = "ChunkedEllpack< int, " + org + " >"; break;
         case TNLB_BIELLPACK: seg = "BiEllpack< int, " + org + ", 32 >"; break;
      }
      return std::string("Matrices::SparseMatrix< ") + (std::is_same<Real, double>::value ? "double" : "float") + ", " +
             seg + ", [any_device], int, " + (isSymmetric() ? "Symmetric" : "General") +
             ", [any_allocator], [any_allocator] >";
   }
   // SparseMatrix::save (SparseMatrix.hpp:632-643): the reference's bytes.
   void save(const std::string& fileName) const
   {
      tnlb::check(tnlb_matrix_save(fileName.c_str(), seg_, tnlb::real_code<Real>(), columns_idx_.getData(),
                                   values_.getData(), rows_, columns_, isSymmetric() ? 1 : 0));
   }
   // SparseMatrix::load (SparseMatrix.hpp:646-694): the file's type must be
   // this matrix's type (else std::runtime_error with the reference's
   // FileDeserializationError message); segments from the stored metadata.
   void load(const std::string& fileName)
   {
      tnlb_matrix_file_info info;
      tnlb::check(tnlb_matrix_file_info_read(fileName.c_str(), &info));
      const std::string expected = getSerializationType();
      if (expected != info.type)
         throw std::runtime_error(fileName + ": object type does not match (expected " + expected + ", found " +
                                  info.type + ").");
      const Index slots = (Index)(info.storage > 0 ? info.storage : 1);
      values_.setSize(slots);
      columns_idx_.setSize(slots);
      tnlb_segments* s = nullptr;
      tnlb::check(tnlb_matrix_load(fileName.c_str(), &s, columns_idx_.getData(), values_.getData(), slots));
      tnlb_segments_destroy(seg_);
      seg_ = s;
      rows_ = (Index)info.rows;
      columns_ = (Index)info.columns;
      values_.setSize((Index)info.storage);
      columns_idx_.setSize((Index)info.storage);
   }
#ifdef __CUDACC__
   // SparseMatrixBase::forElements (Matrices/SparseMatrixBase.h:858):
   // f(rowIdx, localIdx, columnIdx&, value&) on every slot of rows [begin,
   // end), run on the GPU by one thread per row; f is a __device__ callable
   // (an extended __host__ __device__ lambda).  The matrix must use CSR or
   // AdaptiveCSR segments, whose rows are contiguous in storage (other
   // formats: assemble a CSR matrix and assign it).  Synchronous.
   template <typename F>
   void forElements(Index begin, Index end, F f)
   {
      if (begin < 0 || end > rows_ || begin > end) throw std::invalid_argument("forElements: bad row range");
      const int32_t* offsets = nullptr;
      tnlb::check(tnlb_segments_offsets_view(seg_, &offsets));
      if (end == begin) return;
      const unsigned blocks = (unsigned)((end - begin + 255) / 256);
      detail::for_elements_csr<Index, Real, F><<<blocks, 256>>>(offsets, begin, end, columns_idx_.getData(),
                                                                  values_.getData(), f);
      tnlb::cuda_check(cudaGetLastError());
      tnlb::cuda_check(cudaStreamSynchronize(nullptr));
   }
   // SparseMatrixBase::forAllElements (SparseMatrixBase.h:904).
   template <typename F>
   void forAllElements(F f)
   {
      forElements(0, rows_, f);
   }
#endif
   Index getRows() const { return rows_; }
   Index getColumns() const { return columns_; }
   static constexpr bool isSymmetric() { return std::is_same<MatrixType, SymmetricMatrix>::value; }
   // The stored elements as host CSR (segment order, padding dropped) in FP64.
   void toHostCSR(std::vector<Index>& rp, std::vector<Index>& cols, std::vector<double>& vals) const
   {
      tnlb_host_csr h{};
      tnlb::check(tnlb_matrix_to_host_csr(seg_, tnlb::real_code<Real>(), columns_idx_.getData(), values_.getData(),
                                          columns_, &h));
      rp.assign(h.rowptr, h.rowptr + h.rows + 1);
      cols.assign(h.cols, h.cols + h.nnz);
      vals.assign(h.values, h.values + h.nnz);
      tnlb_host_csr_free(&h);
   }
   const tnlb_segments* segments() const { return seg_; }
   const Containers::Vector<Real>& getValues() const { return values_; }
   const Containers::Vector<Index>& getColumnIndexes() const { return columns_idx_; }
   // SparseMatrixBase::getValues / getColumnIndexes (SparseMatrixBase.h):
   // writable views of the storage, e.g. for a device-side assembler.
   Containers::Vector<Real>& getValues() { return values_; }
   Containers::Vector<Index>& getColumnIndexes() { return columns_idx_; }

private:
   Index rows_ = 0, columns_ = 0;
   tnlb_segments* seg_ = nullptr;
   Containers::Vector<Real> values_;
   Containers::Vector<Index> columns_idx_;
};

// MatrixReader::readMtx / MatrixWriter::writeMtx (Matrices/MatrixReader.h,
// MatrixWriter.h) over tnlb_mtx_read / tnlb_mtx_write.
template <typename Matrix>
struct MatrixReader {
   static void readMtx(const std::string& fileName, Matrix& matrix, bool verbose = false)
   {
      (void)verbose;
      tnlb_host_csr h{};
      tnlb::check(tnlb_mtx_read(fileName.c_str(), Matrix::isSymmetric() ? 1 : 0, &h));
      std::vector<int> rp(h.rowptr, h.rowptr + h.rows + 1), cols(h.cols, h.cols + h.nnz);
      std::vector<typename Matrix::RealType> vals(h.values, h.values + h.nnz);
      const int rows = h.rows, columns = h.columns;
      tnlb_host_csr_free(&h);
      matrix.setFromCSR(rows, columns, rp, cols, vals);
   }
};

template <typename Matrix>
struct MatrixWriter {
   static void writeMtx(const std::string& fileName, const Matrix& matrix, bool verbose = false)
   {
      (void)verbose;
      std::vector<int> rp, cols;
      std::vector<double> vals;
      matrix.toHostCSR(rp, cols, vals);
      tnlb::check(tnlb_mtx_write(fileName.c_str(), matrix.getRows(), matrix.getColumns(), rp.data(), cols.data(),
                                 vals.data()));
   }
};

}  // namespace Matrices

namespace Solvers {
namespace Linear {
namespace Preconditioners {

template <typename Matrix, tnlb_precond_kind Kind>
class PreconditionerBase {
public:
   using MatrixPointer = std::shared_ptr<const Matrix>;
   ~PreconditionerBase() { tnlb_precond_destroy(p_); }
   // Preconditioner::update (Preconditioner.h:96-104)
   void update(const MatrixPointer& m)
   {
      if (m->getRows() == 0) throw std::invalid_argument("Preconditioner::update: the matrix is empty");
      if (m->getRows() != m->getColumns()) throw std::invalid_argument("Preconditioner::update: matrix must be square");
      tnlb_precond_destroy(p_);
      p_ = nullptr;
      tnlb::check(tnlb_precond_create(Kind, m->segments(), tnlb::real_code<typename Matrix::RealType>(),
                                      m->getColumnIndexes().getData(), m->getValues().getData(), nullptr, &p_));
      matrix_ = m;
   }
   template <typename V1, typename V2>
   void solve(const V1& b, V2& x) const
   {
      tnlb::check(tnlb_precond_solve(p_, b.getData(), x.getData(), nullptr));
   }
   const tnlb_precond* handle() const { return p_; }

private:
   tnlb_precond* p_ = nullptr;
   MatrixPointer matrix_;
};

template <typename Matrix>
using Diagonal = PreconditionerBase<Matrix, TNLB_PRECOND_JACOBI>;
template <typename Matrix>
using ILU0 = PreconditionerBase<Matrix, TNLB_PRECOND_ILU0>;
template <typename Matrix>
using FSAI = PreconditionerBase<Matrix, TNLB_PRECOND_FSAI>;

// Preconditioners::ILUT (ILUT.h, ILUT.hpp:27-258): factorised on the host
// with the reference's arithmetic and selection, applied on the GPU.  Setup
// keys "ilut-p" (default 0) and "ilut-threshold" (default 1e-4).
template <typename Matrix>
class ILUT {
public:
   using MatrixPointer = std::shared_ptr<const Matrix>;
   ~ILUT() { tnlb_precond_destroy(p_); }
   bool setup(const std::map<std::string, std::string>& prm, const std::string& prefix = "")
   {
      auto it = prm.find(prefix + "ilut-p");
      if (it != prm.end()) ilut_p_ = std::stoi(it->second);
      it = prm.find(prefix + "ilut-threshold");
      if (it != prm.end()) tau_ = std::stod(it->second);
      return true;
   }
   void update(const MatrixPointer& m)
   {
      if (m->getRows() == 0) throw std::invalid_argument("ILUT::update: the matrix is empty");
      if (m->getRows() != m->getColumns()) throw std::invalid_argument("ILUT::update: matrix must be square");
      tnlb_precond_destroy(p_);
      p_ = nullptr;
      tnlb::check(tnlb_precond_create_ilut(m->segments(), tnlb::real_code<typename Matrix::RealType>(),
                                           m->getColumnIndexes().getData(), m->getValues().getData(), ilut_p_, tau_,
                                           nullptr, &p_));
      matrix_ = m;
   }
   template <typename V1, typename V2>
   void solve(const V1& b, V2& x) const
   {
      tnlb::check(tnlb_precond_solve(p_, b.getData(), x.getData(), nullptr));
   }
   const tnlb_precond* handle() const { return p_; }

private:
   tnlb_precond* p_ = nullptr;
   MatrixPointer matrix_;
   int ilut_p_ = 0;
   double tau_ = 1e-4;
};

}  // namespace Preconditioners

template <typename Matrix, tnlb_solver_kind Kind>
class SolverBase {
public:
   using MatrixPointer = std::shared_ptr<const Matrix>;
   using RealType = typename Matrix::RealType;
   SolverBase() { tnlb_solver_params_default(&p_); }
   void setMatrix(const MatrixPointer& m)
   {
      if (m->getRows() != m->getColumns()) throw std::invalid_argument("LinearSolver::setMatrix: matrix must be square");
      matrix_ = m;
   }
   template <typename P>
   void setPreconditioner(const std::shared_ptr<P>& pre)
   {
      precond_ = pre ? pre->handle() : nullptr;
      keep_ = pre;
   }
   // setup(ParameterContainer) keys (IterativeSolver.hpp:14-36, GMRES.hpp:20-37, BICGStab.hpp:14-21,
   // BICGStabL.hpp:14-33, IDRs.hpp:18-34)
   bool setup(const std::map<std::string, std::string>& prm, const std::string& prefix = "")
   {
      auto get = [&](const char* k) -> const std::string* {
         auto it = prm.find(prefix + k);
         return it == prm.end() ? nullptr : &it->second;
      };
      if (auto v = get("max-iterations")) p_.max_iterations = std::stoi(*v);
      if (auto v = get("min-iterations")) p_.min_iterations = std::stoi(*v);
      if (auto v = get("convergence-residue")) p_.convergence_residue = std::stod(*v);
      if (auto v = get("divergence-residue")) p_.divergence_residue = std::stod(*v);
      if (auto v = get("gmres-variant")) {
         const std::map<std::string, int> m{{"CGS", 0}, {"CGSR", 1}, {"MGS", 2}, {"MGSR", 3}, {"CWY", 4}};
         p_.gmres_variant = m.at(*v);
      }
      if (auto v = get("gmres-restarting-min")) p_.gmres_restarting_min = std::stoi(*v);
      if (auto v = get("gmres-restarting-max")) p_.gmres_restarting_max = std::stoi(*v);
      if (auto v = get("gmres-restarting-step-min")) p_.gmres_restarting_step_min = std::stoi(*v);
      if (auto v = get("gmres-restarting-step-max")) p_.gmres_restarting_step_max = std::stoi(*v);
      if (auto v = get("bicgstab-exact-residue")) p_.bicgstab_exact_residue = (*v == "true" || *v == "1");
      if (auto v = get("bicgstab-ell")) p_.bicgstab_ell = std::stoi(*v);
      if (auto v = get("idr-s")) p_.idr_s = std::stoi(*v);
      if (auto v = get("idr-residual-smoothing")) p_.idr_residual_smoothing = (*v == "true" || *v == "1");
      return true;
   }
   void setConvergenceResidue(double r) { p_.convergence_residue = r; }
   void setDivergenceResidue(double r) { p_.divergence_residue = r; }
   void setMaxIterations(int n) { p_.max_iterations = n; }
   void setMinIterations(int n) { p_.min_iterations = n; }
   // LinearSolver::solve (LinearSolver.h:157-158): x holds the initial guess.
   template <typename V1, typename V2>
   bool solve(const V1& b, V2& x)
   {
      if (!matrix_) throw std::logic_error("No matrix was set. Call setMatrix() before solve().");
      tnlb_solve_result r;
      tnlb::check(tnlb_solve_preconditioned(Kind, precond_, &p_, matrix_->segments(), tnlb::real_code<RealType>(),
                                            matrix_->getColumnIndexes().getData(), matrix_->getValues().getData(),
                                            b.getData(), x.getData(), nullptr, &r));
      iterations_ = r.iterations;
      residue_ = r.residue;
      return r.converged != 0;
   }
   int getIterations() const { return iterations_; }
   double getResidue() const { return residue_; }

private:
   tnlb_solver_params p_;
   MatrixPointer matrix_;
   const tnlb_precond* precond_ = nullptr;
   std::shared_ptr<const void> keep_;
   int iterations_ = 0;
   double residue_ = 0;
};

template <typename Matrix>
using CG = SolverBase<Matrix, TNLB_SOLVER_CG>;
template <typename Matrix>
using BICGStab = SolverBase<Matrix, TNLB_SOLVER_BICGSTAB>;
template <typename Matrix>
using GMRES = SolverBase<Matrix, TNLB_SOLVER_GMRES>;
template <typename Matrix>
using FGMRES = SolverBase<Matrix, TNLB_SOLVER_FGMRES>;
template <typename Matrix>
using TFQMR = SolverBase<Matrix, TNLB_SOLVER_TFQMR>;
template <typename Matrix>
using BICGStabL = SolverBase<Matrix, TNLB_SOLVER_BICGSTABL>;
template <typename Matrix>
using IDRs = SolverBase<Matrix, TNLB_SOLVER_IDRS>;

}  // namespace Linear
}  // namespace Solvers

}  // namespace TNL
