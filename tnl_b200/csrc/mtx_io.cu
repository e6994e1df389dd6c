// mtx_io.cu -- MatrixMarket files (host code): the reader of
// Matrices/MatrixReader.hpp:18-330 and the writer of
// Matrices/MatrixWriter.hpp:107-129, with their rules kept so that a file
// reads and writes as it does in the reference:
//  * header "%%MatrixMarket matrix coordinate(s) real|integer|pattern
//    general|symmetric" (at least 5 space-separated words);
//  * lines starting with '%' are comments; the size line has exactly three
//    words; rows and columns must be positive;
//  * words are separated by spaces only (tabs are not separators); sizes
//    and values are read with atoi / atof; an element's row and column must
//    start with an integer in [1, rows] and [1, columns] (an error
//    otherwise, where the reference would index outside the matrix);
//  * elements go through an ordered map keyed by (row, column): a repeated
//    position keeps the last value, rows and columns come out sorted, and
//    explicit zeros are kept;
//  * a symmetric file read into general storage gets both triangles; read
//    into symmetric storage (one triangle), entries are folded onto the lower
//    one; a general file cannot be read into symmetric storage;
//  * the writer prints "row column value" with widths 9, 9, 12, default
//    stream precision, 1-based, skipping zero values.
#include <cerrno>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "internal.cuh"
#include "segview.cuh"

namespace {

std::vector<std::string> split_spaces(const std::string& line)
{
   std::vector<std::string> out;
   std::string cur;
   for (char ch : line) {
      if (ch == ' ') {
         if (!cur.empty()) out.push_back(cur);
         cur.clear();
      }
      else
         cur += ch;
   }
   if (!cur.empty()) out.push_back(cur);
   return out;
}

tnlb_status io_error(const std::string& msg)
{
   tnlb::set_error(msg);
   return TNLB_ERR_IO;
}

// An element's row or column word, read as atoi reads it (leading digits,
// anything after them ignored), but a word with no leading number is an
// error rather than 0, and so is one outside the int range.
bool parse_index(const std::string& w, int& out)
{
   errno = 0;
   const char* begin = w.c_str();
   char* end = nullptr;
   const long v = std::strtol(begin, &end, 10);
   if (end == begin || errno != 0 || v < INT32_MIN || v > INT32_MAX) return false;
   out = (int)v;
   return true;
}

}  // namespace

extern "C" tnlb_status tnlb_mtx_read(const char* path, int32_t symmetric_storage, tnlb_host_csr* out)
{
   using namespace tnlb;
   clear_error();
   TNLB_REQUIRE(path && out, TNLB_ERR_INVALID_ARGUMENT, "null argument");
   *out = tnlb_host_csr{};
   std::ifstream file(path);
   if (!file) return io_error(std::string("I am not able to open the file ") + path);
   std::string line;
   bool symmetric = false, pattern = false;
   // header (MatrixReader.hpp:146-178)
   if (!std::getline(file, line)) line.clear();
   {
      const auto w = split_spaces(line);
      if ((int)w.size() < 5 || w[0] != "%%MatrixMarket")
         return io_error(
            "Unknown format of the source file. We expect line like this: %%MatrixMarket matrix coordinate real general");
      if (w[1] != "matrix") return io_error("Keyword 'matrix' is expected in the header line: " + line);
      if (w[2] != "coordinates" && w[2] != "coordinate")
         return io_error("Error: Only 'coordinates' format is supported now, not " + w[2]);
      if (w[3] != "real" && w[3] != "integer" && w[3] != "pattern")
         return io_error("Only 'real' and 'integer' matrices are supported, not " + w[3]);
      pattern = w[3] == "pattern";
      if (w[4] != "general") {
         if (w[4] == "symmetric")
            symmetric = true;
         else
            return io_error("Only 'general' matrices are supported, not " + w[4]);
      }
   }
   if (symmetric_storage && !symmetric)
      return io_error("Matrix is not symmetric, but flag for symmetric matrix is given. Aborting.");
   // size line (:195-215)
   int rows = 0, columns = 0;
   while (true) {
      if (!std::getline(file, line)) return io_error("Wrong number of parameters in the matrix header - should be 3.");
      if (!line.empty() && line[0] == '%') continue;
      const auto w = split_spaces(line);
      if ((int)w.size() != 3) return io_error("Wrong number of parameters in the matrix header - should be 3.");
      rows = atoi(w[0].c_str());
      columns = atoi(w[1].c_str());
      if (rows <= 0 || columns <= 0) return io_error("Row or column index is negative.");
      break;
   }
   // elements (:222-290)
   std::map<std::pair<int, int>, double> map;
   while (std::getline(file, line)) {
      if (line.empty() || line[0] == '%') continue;
      const auto w = split_spaces(line);
      if ((int)w.size() != 3 - (int)pattern)
         return io_error("Wrong number of parameters in the matrix row at line:" + line);
      int row = 0, column = 0;
      if (!parse_index(w[0], row) || !parse_index(w[1], column))
         return io_error("The row or column of the element is not an integer at line:" + line);
      const double value = pattern ? 1.0 : atof(w[2].c_str());
      // 1-based positions: a row or column below 1 is outside the matrix as
      // much as one past its size (the reference would index row -1)
      if (column > columns || row > rows || column < 1 || row < 1) {
         std::stringstream s;
         s << "There is an element at position " << row << ", " << column << " out of the matrix dimensions " << rows
           << " x " << columns << ".";
         return io_error(s.str());
      }
      if (!symmetric_storage || row >= column)
         map[{row - 1, column - 1}] = value;
      else
         map[{column - 1, row - 1}] = value;
      if (symmetric && row != column && !symmetric_storage) map[{column - 1, row - 1}] = value;
   }
   const int64_t nnz = (int64_t)map.size();
   TNLB_REQUIRE(nnz <= INT32_MAX, TNLB_ERR_OVERFLOW, "MatrixMarket file with more than 2^31-1 elements");
   out->rows = rows;
   out->columns = columns;
   out->nnz = nnz;
   out->rowptr = (int32_t*)calloc((size_t)rows + 1, sizeof(int32_t));
   out->cols = (int32_t*)malloc(sizeof(int32_t) * (nnz > 0 ? nnz : 1));
   out->values = (double*)malloc(sizeof(double) * (nnz > 0 ? nnz : 1));
   if (!out->rowptr || !out->cols || !out->values) {
      tnlb_host_csr_free(out);
      set_error("host allocation failed");
      return TNLB_ERR_OUT_OF_MEMORY;
   }
   int64_t k = 0;
   for (const auto& e : map) {
      out->rowptr[e.first.first + 1]++;
      out->cols[k] = e.first.second;
      out->values[k] = e.second;
      k++;
   }
   for (int r = 0; r < rows; r++) out->rowptr[r + 1] += out->rowptr[r];
   return TNLB_OK;
}

extern "C" void tnlb_host_csr_free(tnlb_host_csr* m)
{
   if (!m) return;
   free(m->rowptr);
   free(m->cols);
   free(m->values);
   *m = tnlb_host_csr{};
}

extern "C" tnlb_status tnlb_mtx_write(const char* path, int32_t rows, int32_t columns, const int32_t* h_rowptr,
                                      const int32_t* h_cols, const double* h_values)
{
   using namespace tnlb;
   clear_error();
   TNLB_REQUIRE(path && rows >= 0 && columns >= 0 && h_rowptr && (h_rowptr[rows] == 0 || (h_cols && h_values)),
                TNLB_ERR_INVALID_ARGUMENT, "null or negative argument");
   std::ofstream str(path);
   if (!str) return io_error(std::string("I am not able to open the file ") + path);
   int64_t nonzeros = 0;
   for (int64_t k = 0; k < h_rowptr[rows]; k++)
      if (h_cols[k] != -1 && h_values[k] != 0) nonzeros++;
   str << "%%MatrixMarket matrix coordinate real general\n";
   str << "%%\n";
   str << "%% This file was generated by TNL (www.tnl-project.org)\n";
   str << "%%" << std::setw(9) << " ROWS " << std::setw(9) << " COLUMNS " << std::setw(12) << " ELEMENTS \n";
   str << std::setw(9) << rows << " " << std::setw(9) << columns << " " << std::setw(12) << nonzeros << '\n';
   for (int32_t r = 0; r < rows; r++)
      for (int32_t k = h_rowptr[r]; k < h_rowptr[r + 1]; k++) {
         if (h_cols[k] == -1) continue;
         const double value = h_values[k];
         if (value != 0) str << std::setw(9) << r + 1 << std::setw(9) << h_cols[k] + 1 << std::setw(12) << value << '\n';
      }
   if (!str) return io_error(std::string("writing the file ") + path + " failed");
   return TNLB_OK;
}

extern "C" tnlb_status tnlb_matrix_to_host_csr(const tnlb_segments* seg, tnlb_real real, const int32_t* d_cols,
                                               const void* d_values, int32_t columns, tnlb_host_csr* out)
{
   using namespace tnlb;
   clear_error();
   TNLB_REQUIRE(seg && out, TNLB_ERR_INVALID_ARGUMENT, "null argument");
   TNLB_REQUIRE(real == TNLB_F32 || real == TNLB_F64, TNLB_ERR_INVALID_ARGUMENT, "unknown real type");
   *out = tnlb_host_csr{};
   DeviceBuffer rp, oc, ov;
   TNLB_TRY_STATUS(gather_csr(view_of(seg), real, d_cols, d_values, rp, oc, ov, nullptr));
   const int32_t n = seg->n;
   out->rows = n;
   out->columns = columns;
   out->rowptr = (int32_t*)calloc((size_t)n + 1, sizeof(int32_t));
   if (!out->rowptr) {
      set_error("host allocation failed");
      return TNLB_ERR_OUT_OF_MEMORY;
   }
   TNLB_CUDA_TRY(cudaMemcpy(out->rowptr, rp.ptr, sizeof(int32_t) * ((size_t)n + 1), cudaMemcpyDeviceToHost));
   const int64_t nnz = out->rowptr[n];
   out->nnz = nnz;
   out->cols = (int32_t*)malloc(sizeof(int32_t) * (nnz > 0 ? nnz : 1));
   out->values = (double*)malloc(sizeof(double) * (nnz > 0 ? nnz : 1));
   if (!out->cols || !out->values) {
      tnlb_host_csr_free(out);
      set_error("host allocation failed");
      return TNLB_ERR_OUT_OF_MEMORY;
   }
   if (nnz > 0) {
      TNLB_CUDA_TRY(cudaMemcpy(out->cols, oc.ptr, sizeof(int32_t) * nnz, cudaMemcpyDeviceToHost));
      if (real == TNLB_F64)
         TNLB_CUDA_TRY(cudaMemcpy(out->values, ov.ptr, sizeof(double) * nnz, cudaMemcpyDeviceToHost));
      else {
         std::vector<float> f((size_t)nnz);
         TNLB_CUDA_TRY(cudaMemcpy(f.data(), ov.ptr, sizeof(float) * nnz, cudaMemcpyDeviceToHost));
         for (int64_t k = 0; k < nnz; k++) out->values[k] = f[k];
      }
   }
   return TNLB_OK;
}
