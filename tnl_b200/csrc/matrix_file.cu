// matrix_file.cu -- TNL's binary matrix file: SparseMatrix::save / load
// (Matrices/SparseMatrix.hpp:632-700, SparseMatrixBase.hpp:1148-1159).
//
// Layout, as the reference's File / Object serialization writes it
// (Object.hpp:37-88, File.hpp:200-255, Containers/Array.hpp:585-620):
//   object header   "TNLMN", int32 length, the type string
//                   "Matrices::SparseMatrix< <Real>, <Segments type>,
//                    [any_device], int, General|Symmetric, [any_allocator],
//                    [any_allocator] >"
//   size_t rows, size_t columns
//   the segments' own save():
//     CSR            Array< int > offsets (CSR.hpp:116-121)
//     AdaptiveCSR    CSR, then 6 arrays of block descriptors (AdaptiveCSR.hpp:146-153)
//     Ellpack        int segmentSize, segmentsCount, alignedSize (Ellpack.hpp:105-112)
//     SlicedEllpack  int size, storageSize, segmentsCount; Array< int > sliceOffsets,
//                    sliceSegmentSizes (SlicedEllpack.hpp:166-175)
//     ChunkedEllpack int size, storageSize, numberOfSlices, chunksInSlice, desiredChunkSize;
//                    arrays segmentToChunkMapping, segmentToSliceMapping,
//                    chunksToSegmentsMapping, segmentPointers, slices (ChunkedEllpack.hpp:241-252)
//     BiEllpack      int size, storageSize; Array< int > segmentsPermutation,
//                    groupPointers (BiEllpack.hpp:223-230)
//   Array< Real > values, Array< int > columnIndexes
// where an array is an object header with "TNL::Containers::Array< T >",
// a size_t element count and the raw elements.  All integers are
// little-endian, as the reference writes them on x86.
//
// The metadata of a segments object here is bit-identical to the
// reference's, so saving is a download and a serialisation, and loading
// uploads the arrays into a segments object directly (no rebuild).  Two
// arrays of the reference hold bytes it never initialises: the slices array
// of ChunkedEllpack has one entry per segment of which only the first
// numberOfSlices are set, and AdaptiveCSR descriptors leave fields and
// padding unset per type.  Those bytes are written as zeros here.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "internal.cuh"

namespace tnlb {

namespace {

constexpr char kMagic[] = "TNLMN";
constexpr int kAcsrDescBytes = 20;  // the reference's descriptor: 1 + 3 pad + 3 * 4 + 1 + 1 + 2 pad

const char* org_name(int org) { return org == TNLB_ROW_MAJOR ? "RowMajorOrder" : "ColumnMajorOrder"; }

std::string segments_type(int format, int org)
{
   switch (format) {
      case TNLB_CSR: return "CSR< int >";
      case TNLB_ADAPTIVE_CSR: return "AdaptiveCSR< int >";
      case TNLB_ELLPACK: return std::string("Ellpack< int, ") + org_name(org) + ", 32 >";
      case TNLB_SLICED_ELLPACK: return std::string("SlicedEllpack< int, ") + org_name(org) + ", 32 >";
      case TNLB_CHUNKED_ELLPACK: return std::string("ChunkedEllpack< int, ") + org_name(org) + " >";
      case TNLB_BIELLPACK: return std::string("BiEllpack< int, ") + org_name(org) + ", 32 >";
   }
   return "";
}

std::string matrix_type(int format, int org, tnlb_real real, bool symmetric)
{
   return std::string("Matrices::SparseMatrix< ") + (real == TNLB_F64 ? "double" : "float") + ", " +
          segments_type(format, org) + ", [any_device], int, " + (symmetric ? "Symmetric" : "General") +
          ", [any_allocator], [any_allocator] >";
}

const std::string kArrInt = "TNL::Containers::Array< int >";
const std::string kArrSlice = "TNL::Containers::Array< TNL::Algorithms::Segments::detail::ChunkedEllpackSliceInfo<int> >";
const std::string kArrDesc =
   "TNL::Containers::Array< TNL::Algorithms::Segments::detail::CSRAdaptiveKernelBlockDescriptor<int> >";

std::string arr_real(tnlb_real real)
{
   return real == TNLB_F64 ? "TNL::Containers::Array< double >" : "TNL::Containers::Array< float >";
}

// ------------------------------------------------------------- writing

struct Writer {
   std::vector<char> b;
   void raw(const void* p, size_t n)
   {
      const char* c = static_cast<const char*>(p);
      b.insert(b.end(), c, c + n);
   }
   template <typename T>
   void val(T v)
   {
      raw(&v, sizeof(T));
   }
   void header(const std::string& type)
   {
      raw(kMagic, 5);
      val<int32_t>((int32_t)type.size());
      raw(type.data(), type.size());
   }
   void array(const std::string& type, const void* data, size_t count, size_t elem)
   {
      header(type);
      val<uint64_t>(count);
      raw(data, count * elem);
   }
};

template <typename T>
tnlb_status download(const DeviceBuffer& d, size_t count, std::vector<T>& h)
{
   h.resize(count);
   if (count) TNLB_CUDA_TRY(cudaMemcpy(h.data(), d.ptr, sizeof(T) * count, cudaMemcpyDeviceToHost));
   return TNLB_OK;
}

tnlb_status write_segments(const tnlb_segments* seg, Writer& w)
{
   const int32_t n = seg->n;
   std::vector<int32_t> a, b2, c, d;
   switch (seg->format) {
      case TNLB_CSR:
      case TNLB_ADAPTIVE_CSR: {
         TNLB_TRY_STATUS(download(seg->offsets, (size_t)n + 1, a));
         w.array(kArrInt, a.data(), a.size(), 4);
         if (seg->format == TNLB_ADAPTIVE_CSR)
            for (int k = 0; k < 6; k++) {
               const size_t cnt = (size_t)seg->acsr_count[k];
               std::vector<tnlb_acsr_block> blk;
               TNLB_TRY_STATUS(download(seg->acsr_blocks[k], cnt, blk));
               std::vector<unsigned char> bytes(cnt * kAcsrDescBytes, 0);
               for (size_t q = 0; q < cnt; q++) {
                  unsigned char* o = bytes.data() + q * kAcsrDescBytes;
                  o[0] = blk[q].type;
                  std::memcpy(o + 4, &blk[q].first_segment, 4);
                  std::memcpy(o + 8, &blk[q].block_size, 4);
                  std::memcpy(o + 12, &blk[q].segments_in_block, 4);
                  o[16] = blk[q].warp_idx;
                  o[17] = blk[q].warps_count;
               }
               w.array(kArrDesc, bytes.data(), cnt, kAcsrDescBytes);
            }
         return TNLB_OK;
      }
      case TNLB_ELLPACK:
         w.val<int32_t>(seg->segment_size);
         w.val<int32_t>(n);
         w.val<int32_t>(seg->aligned_size);
         return TNLB_OK;
      case TNLB_SLICED_ELLPACK:
         w.val<int32_t>((int32_t)seg->elements);
         w.val<int32_t>((int32_t)seg->storage);
         w.val<int32_t>(n);
         TNLB_TRY_STATUS(download(seg->slice_offsets, (size_t)seg->slices + 1, a));
         TNLB_TRY_STATUS(download(seg->slice_segment_sizes, (size_t)seg->slices, b2));
         w.array(kArrInt, a.data(), a.size(), 4);
         w.array(kArrInt, b2.data(), b2.size(), 4);
         return TNLB_OK;
      case TNLB_CHUNKED_ELLPACK: {
         const int32_t s = seg->ch_slices;
         w.val<int32_t>((int32_t)seg->elements);
         w.val<int32_t>((int32_t)seg->storage);
         w.val<int32_t>(s);
         w.val<int32_t>(kChunksInSlice);
         w.val<int32_t>(kDesiredChunkSize);
         TNLB_TRY_STATUS(download(seg->ch_segment_to_chunk, (size_t)n, a));
         w.array(kArrInt, a.data(), a.size(), 4);
         TNLB_TRY_STATUS(download(seg->ch_segment_to_slice, (size_t)n, a));
         w.array(kArrInt, a.data(), a.size(), 4);
         TNLB_TRY_STATUS(download(seg->ch_chunks_to_segments, (size_t)s * kChunksInSlice, a));
         w.array(kArrInt, a.data(), a.size(), 4);
         TNLB_TRY_STATUS(download(seg->ch_segment_pointers, (size_t)n + 1, a));
         w.array(kArrInt, a.data(), a.size(), 4);
         // slices: one entry per segment, the first numberOfSlices defined
         TNLB_TRY_STATUS(download(seg->ch_slice_size, (size_t)s, a));
         TNLB_TRY_STATUS(download(seg->ch_slice_chunk_size, (size_t)s, b2));
         TNLB_TRY_STATUS(download(seg->ch_slice_first, (size_t)s, c));
         TNLB_TRY_STATUS(download(seg->ch_slice_pointer, (size_t)s, d));
         std::vector<int32_t> info((size_t)n * 4, 0);
         for (int32_t q = 0; q < s && q < n; q++) {
            info[4 * q] = a[q];
            info[4 * q + 1] = b2[q];
            info[4 * q + 2] = c[q];
            info[4 * q + 3] = d[q];
         }
         w.array(kArrSlice, info.data(), (size_t)n, 16);
         return TNLB_OK;
      }
      case TNLB_BIELLPACK:
         w.val<int32_t>((int32_t)seg->elements);
         w.val<int32_t>((int32_t)seg->storage);
         TNLB_TRY_STATUS(download(seg->bi_perm, (size_t)n, a));
         w.array(kArrInt, a.data(), a.size(), 4);
         TNLB_TRY_STATUS(download(seg->bi_group_pointers, (size_t)seg->strips * kBiGroups + 1, a));
         w.array(kArrInt, a.data(), a.size(), 4);
         return TNLB_OK;
   }
   set_error("save: unknown segments format");
   return TNLB_ERR_INVALID_ARGUMENT;
}

// ------------------------------------------------------------- reading

struct Reader {
   std::vector<char> b;
   size_t pos = 0;
   bool fail = false;
   bool take(void* out, size_t n)
   {
      if (fail || pos + n > b.size()) {
         fail = true;
         return false;
      }
      std::memcpy(out, b.data() + pos, n);
      pos += n;
      return true;
   }
   template <typename T>
   T val()
   {
      T v{};
      take(&v, sizeof(T));
      return v;
   }
   std::string header()
   {
      char mn[5];
      if (!take(mn, 5) || std::memcmp(mn, kMagic, 5) != 0) {
         fail = true;
         return "";
      }
      const int32_t len = val<int32_t>();
      if (fail || len < 0 || pos + (size_t)len > b.size()) {
         fail = true;
         return "";
      }
      std::string t(b.data() + pos, (size_t)len);
      pos += (size_t)len;
      return t;
   }
   // an array of the given type string; elem bytes per element
   bool array(const std::string& type, size_t elem, std::vector<char>& out, uint64_t* count)
   {
      if (header() != type) {
         fail = true;
         return false;
      }
      const uint64_t n = val<uint64_t>();
      if (fail || n > (b.size() - pos) / (elem ? elem : 1)) {
         fail = true;
         return false;
      }
      out.assign(b.data() + pos, b.data() + pos + n * elem);
      pos += n * elem;
      *count = n;
      return true;
   }
   bool ints(std::vector<int32_t>& out, uint64_t expect)
   {
      std::vector<char> raw;
      uint64_t n = 0;
      if (!array(kArrInt, 4, raw, &n) || n != expect) {
         fail = true;
         return false;
      }
      out.resize(n);
      if (n) std::memcpy(out.data(), raw.data(), n * 4);
      return true;
   }
};

tnlb_status read_file(const char* path, std::vector<char>& out)
{
   FILE* f = std::fopen(path, "rb");
   if (!f) {
      set_error(std::string("unable to open the file ") + path);
      return TNLB_ERR_IO;
   }
   std::fseek(f, 0, SEEK_END);
   const long size = std::ftell(f);
   std::fseek(f, 0, SEEK_SET);
   out.resize(size > 0 ? (size_t)size : 0);
   const size_t got = out.empty() ? 0 : std::fread(out.data(), 1, out.size(), f);
   std::fclose(f);
   if (got != out.size()) {
      set_error(std::string("unable to read the file ") + path);
      return TNLB_ERR_IO;
   }
   return TNLB_OK;
}

// Matches a type string against the ones this library writes.
bool parse_type(const std::string& t, tnlb_matrix_file_info* info)
{
   const int formats[] = {TNLB_CSR, TNLB_ADAPTIVE_CSR, TNLB_ELLPACK, TNLB_SLICED_ELLPACK, TNLB_CHUNKED_ELLPACK,
                          TNLB_BIELLPACK};
   for (int f : formats)
      for (int org : {TNLB_COLUMN_MAJOR, TNLB_ROW_MAJOR})
         for (tnlb_real real : {TNLB_F64, TNLB_F32})
            for (int sym = 0; sym < 2; sym++)
               if (t == matrix_type(f, org, real, sym != 0)) {
                  info->format = f;
                  // CSR-based formats have no organization; report the default
                  info->organization = (f == TNLB_CSR || f == TNLB_ADAPTIVE_CSR) ? TNLB_COLUMN_MAJOR : org;
                  info->real = real;
                  info->symmetric = sym;
                  return true;
               }
   return false;
}

tnlb_status corrupt(const char* path)
{
   set_error(std::string("the file ") + path + " is not a valid TNL sparse matrix file (truncated or inconsistent)");
   return TNLB_ERR_IO;
}

template <typename T>
tnlb_status upload(DeviceBuffer& d, const std::vector<T>& h)
{
   TNLB_TRY_STATUS(d.alloc(sizeof(T) * (h.empty() ? 1 : h.size())));
   if (!h.empty()) TNLB_CUDA_TRY(cudaMemcpy(d.ptr, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice));
   return TNLB_OK;
}

// Parses the header and the segments; fills `info` and, when `seg` is
// given, the segments object.  Leaves the reader at the values array.
tnlb_status parse(const char* path, Reader& r, tnlb_matrix_file_info* info, tnlb_segments* seg)
{
   const std::string type = r.header();
   if (r.fail) {
      set_error(std::string("the file ") + path + " is not in a TNL-compatible format (wrong magic number)");
      return TNLB_ERR_IO;
   }
   std::memset(info, 0, sizeof(*info));
   std::snprintf(info->type, sizeof(info->type), "%s", type.c_str());
   if (!parse_type(type, info)) {
      set_error("unsupported object type in " + std::string(path) + ": " + type);
      return TNLB_ERR_IO;
   }
   const uint64_t rows = r.val<uint64_t>(), columns = r.val<uint64_t>();
   if (r.fail || rows > (uint64_t)INT32_MAX || columns > (uint64_t)INT32_MAX) return corrupt(path);
   info->rows = (int64_t)rows;
   info->columns = (int64_t)columns;
   const int32_t n = (int32_t)rows;
   std::vector<int32_t> a, b2, c, d;
   int64_t storage = 0, elements = 0;
   switch (info->format) {
      case TNLB_CSR:
      case TNLB_ADAPTIVE_CSR: {
         if (!r.ints(a, (uint64_t)n + 1)) return corrupt(path);
         if (a[0] != 0) return corrupt(path);
         for (int32_t i = 0; i < n; i++)
            if (a[i + 1] < a[i]) return corrupt(path);
         storage = elements = a[n];
         std::vector<std::vector<char>> desc(6);
         uint64_t cnt[6] = {0, 0, 0, 0, 0, 0};
         if (info->format == TNLB_ADAPTIVE_CSR)
            for (int k = 0; k < 6; k++)
               if (!r.array(kArrDesc, kAcsrDescBytes, desc[k], &cnt[k])) return corrupt(path);
         if (seg) {
            // the CSR formats are rebuilt from the row lengths: the offsets
            // come out equal, the AdaptiveCSR descriptors equal the file's
            // where the reference defines them (its builder is the same)
            seg->format = info->format;
            seg->organization = TNLB_COLUMN_MAJOR;
            seg->n = n;
            TNLB_CUDA_TRY(cudaGetDevice(&seg->device));
            std::vector<int32_t> sizes((size_t)n);
            for (int32_t i = 0; i < n; i++) sizes[i] = a[i + 1] - a[i];
            DeviceBuffer ds;
            TNLB_TRY_STATUS(upload(ds, sizes));
            TNLB_TRY_STATUS(build_segments(seg, ds.as<int32_t>(), nullptr));
            for (int k = 0; k < 6 && info->format == TNLB_ADAPTIVE_CSR; k++)
               if ((uint64_t)seg->acsr_count[k] != cnt[k]) return corrupt(path);
         }
         break;
      }
      case TNLB_ELLPACK: {
         const int32_t size = r.val<int32_t>(), count = r.val<int32_t>(), aligned = r.val<int32_t>();
         if (r.fail || count != n || (n > 0 && (size < 0 || aligned < n))) return corrupt(path);
         storage = n > 0 ? (int64_t)aligned * size : 0;
         elements = n > 0 ? (int64_t)n * size : 0;
         if (seg) {
            seg->segment_size = size;
            seg->aligned_size = aligned;
            seg->max_size = n > 0 ? size : 0;
         }
         break;
      }
      case TNLB_SLICED_ELLPACK: {
         const int32_t size = r.val<int32_t>(), st = r.val<int32_t>(), count = r.val<int32_t>();
         const int32_t slices = (n + kSellSlice - 1) / kSellSlice;
         if (r.fail || count != n || !r.ints(a, (uint64_t)slices + 1) || !r.ints(b2, (uint64_t)slices))
            return corrupt(path);
         if (a[0] != 0 || a[slices] != st) return corrupt(path);
         for (int32_t q = 0; q < slices; q++)
            if (b2[q] < 0 || (int64_t)a[q + 1] - a[q] != (int64_t)kSellSlice * b2[q]) return corrupt(path);
         storage = st;
         elements = size;
         if (seg) {
            seg->slices = slices;
            TNLB_TRY_STATUS(upload(seg->slice_offsets, a));
            TNLB_TRY_STATUS(upload(seg->slice_segment_sizes, b2));
            int32_t mx = 0;
            for (int32_t v : b2) mx = std::max(mx, v);
            seg->max_size = mx;
         }
         break;
      }
      case TNLB_CHUNKED_ELLPACK: {
         const int32_t size = r.val<int32_t>(), st = r.val<int32_t>(), slices = r.val<int32_t>();
         const int32_t cis = r.val<int32_t>(), dcs = r.val<int32_t>();
         if (r.fail || cis != kChunksInSlice || dcs != kDesiredChunkSize || slices < 0 || slices > n + 1)
            return corrupt(path);
         std::vector<int32_t> s2c, s2s, c2s, sp;
         if (!r.ints(s2c, (uint64_t)n) || !r.ints(s2s, (uint64_t)n) ||
             !r.ints(c2s, (uint64_t)slices * kChunksInSlice) || !r.ints(sp, (uint64_t)n + 1))
            return corrupt(path);
         std::vector<char> raw;
         uint64_t cnt = 0;
         if (!r.array(kArrSlice, 16, raw, &cnt) || cnt != (uint64_t)n || (uint64_t)slices > cnt) return corrupt(path);
         // what the product's kernel indexes with: every slice inside the
         // storage and the segments, chunk indexes inside a slice
         if (st < 0 || sp[0] != 0 || sp[n] != st) return corrupt(path);
         for (int32_t q = 0; q < slices; q++) {
            int32_t v[4];
            std::memcpy(v, raw.data() + 16 * (size_t)q, 16);
            if (v[0] < 0 || v[0] > kChunksInSlice || v[1] < 0 || v[2] < 0 || (int64_t)v[2] + v[0] > n || v[3] < 0 ||
                (int64_t)v[3] + (int64_t)v[1] * kChunksInSlice > st)
               return corrupt(path);
         }
         for (int32_t i = 0; i < n; i++)
            if (s2c[i] < 0 || s2c[i] > kChunksInSlice || s2s[i] < 0 || s2s[i] >= std::max(slices, 1))
               return corrupt(path);
         storage = st;
         elements = size;
         if (seg) {
            seg->ch_slices = slices;
            std::vector<int32_t> ssz(slices), scs(slices), sfi(slices), spt((size_t)slices + 1);
            for (int32_t q = 0; q < slices; q++) {
               int32_t v[4];
               std::memcpy(v, raw.data() + 16 * (size_t)q, 16);
               ssz[q] = v[0];
               scs[q] = v[1];
               sfi[q] = v[2];
               spt[q] = v[3];
            }
            spt[slices] = st;
            TNLB_TRY_STATUS(upload(seg->ch_slice_size, ssz));
            TNLB_TRY_STATUS(upload(seg->ch_slice_chunk_size, scs));
            TNLB_TRY_STATUS(upload(seg->ch_slice_first, sfi));
            TNLB_TRY_STATUS(upload(seg->ch_slice_pointer, spt));
            TNLB_TRY_STATUS(upload(seg->ch_segment_to_chunk, s2c));
            TNLB_TRY_STATUS(upload(seg->ch_segment_to_slice, s2s));
            TNLB_TRY_STATUS(upload(seg->ch_segment_pointers, sp));
            TNLB_TRY_STATUS(upload(seg->ch_chunks_to_segments, c2s));
            int32_t mx = 0;
            for (int32_t i = 0; i < n; i++) mx = std::max(mx, sp[i + 1] - sp[i]);
            seg->max_size = mx;
         }
         break;
      }
      case TNLB_BIELLPACK: {
         const int32_t size = r.val<int32_t>(), st = r.val<int32_t>();
         const int32_t strips = (n + kBiStrip - 1) / kBiStrip;
         if (r.fail || !r.ints(a, (uint64_t)n) || !r.ints(b2, (uint64_t)strips * kBiGroups + 1)) return corrupt(path);
         if (b2[0] != 0 || b2[(size_t)strips * kBiGroups] != st) return corrupt(path);
         for (size_t q = 0; q + 1 < b2.size(); q++)
            if (b2[q + 1] < b2[q]) return corrupt(path);
         storage = st;
         elements = size;
         if (seg) {
            seg->strips = strips;
            TNLB_TRY_STATUS(upload(seg->bi_perm, a));
            TNLB_TRY_STATUS(upload(seg->bi_group_pointers, b2));
         }
         break;
      }
   }
   info->storage = storage;
   if (seg && info->format != TNLB_CSR && info->format != TNLB_ADAPTIVE_CSR) {
      seg->format = info->format;
      seg->organization = info->organization;
      seg->n = n;
      seg->elements = elements;
      seg->storage = storage;
      TNLB_CUDA_TRY(cudaGetDevice(&seg->device));
   }
   return TNLB_OK;
}

}  // namespace

}  // namespace tnlb

extern "C" tnlb_status tnlb_matrix_save(const char* path, const tnlb_segments* seg, tnlb_real real,
                                        const int32_t* d_cols, const void* d_values, int32_t rows, int32_t columns,
                                        int32_t symmetric)
{
   using namespace tnlb;
   clear_error();
   TNLB_REQUIRE(path && seg, TNLB_ERR_INVALID_ARGUMENT, "null argument");
   TNLB_REQUIRE(real == TNLB_F32 || real == TNLB_F64, TNLB_ERR_INVALID_ARGUMENT, "unknown real type");
   TNLB_REQUIRE(rows == seg->n && columns >= 0, TNLB_ERR_INVALID_ARGUMENT, "save: rows differ from the segments");
   Writer w;
   w.header(matrix_type(seg->format, seg->organization, real, symmetric != 0));
   w.val<uint64_t>((uint64_t)rows);
   w.val<uint64_t>((uint64_t)columns);
   TNLB_TRY_STATUS(write_segments(seg, w));
   const size_t rs = real == TNLB_F64 ? 8 : 4;
   const size_t slots = (size_t)seg->storage;
   std::vector<char> vals(slots * rs);
   std::vector<int32_t> cols(slots);
   if (slots) {
      TNLB_CUDA_TRY(cudaMemcpy(vals.data(), d_values, slots * rs, cudaMemcpyDeviceToHost));
      TNLB_CUDA_TRY(cudaMemcpy(cols.data(), d_cols, slots * 4, cudaMemcpyDeviceToHost));
   }
   w.array(arr_real(real), vals.data(), slots, rs);
   w.array(kArrInt, cols.data(), slots, 4);
   FILE* f = std::fopen(path, "wb");
   if (!f) {
      set_error(std::string("unable to open the file ") + path + " for writing");
      return TNLB_ERR_IO;
   }
   const size_t put = w.b.empty() ? 0 : std::fwrite(w.b.data(), 1, w.b.size(), f);
   const int closed = std::fclose(f);
   if (put != w.b.size() || closed != 0) {
      set_error(std::string("unable to write the file ") + path);
      return TNLB_ERR_IO;
   }
   return TNLB_OK;
}

extern "C" tnlb_status tnlb_matrix_file_info_read(const char* path, tnlb_matrix_file_info* info)
{
   using namespace tnlb;
   clear_error();
   TNLB_REQUIRE(path && info, TNLB_ERR_INVALID_ARGUMENT, "null argument");
   Reader r;
   TNLB_TRY_STATUS(read_file(path, r.b));
   return parse(path, r, info, nullptr);
}

extern "C" tnlb_status tnlb_matrix_load(const char* path, tnlb_segments** out, int32_t* d_cols, void* d_values,
                                        int64_t capacity)
{
   using namespace tnlb;
   clear_error();
   TNLB_REQUIRE(path && out, TNLB_ERR_INVALID_ARGUMENT, "null argument");
   *out = nullptr;
   Reader r;
   TNLB_TRY_STATUS(read_file(path, r.b));
   tnlb_matrix_file_info info;
   auto* seg = new tnlb_segments();
   tnlb_status s = parse(path, r, &info, seg);
   if (s == TNLB_OK && capacity < info.storage) {
      set_error("load: the value and column arrays hold fewer slots than the file's storage");
      s = TNLB_ERR_INVALID_ARGUMENT;
   }
   if (s == TNLB_OK) {
      std::vector<char> vraw, craw;
      uint64_t nv = 0, nc = 0;
      const size_t rs = info.real == TNLB_F64 ? 8 : 4;
      if (!r.array(arr_real((tnlb_real)info.real), rs, vraw, &nv) || !r.array(kArrInt, 4, craw, &nc) ||
          nv != (uint64_t)info.storage || nc != (uint64_t)info.storage)
         s = corrupt(path);
      else {
         // every stored column is padding (-1) or a column of the matrix:
         // the products gather x[column] without a bounds check
         const int32_t* c = reinterpret_cast<const int32_t*>(craw.data());
         for (uint64_t k = 0; k < nc; k++)
            if (c[k] < -1 || c[k] >= info.columns) {
               s = corrupt(path);
               break;
            }
      }
      if (s == TNLB_OK && info.storage > 0) {
         if (cudaMemcpy(d_values, vraw.data(), vraw.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
             cudaMemcpy(d_cols, craw.data(), craw.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
            set_error("load: copy to the device failed");
            s = TNLB_ERR_CUDA;
         }
      }
   }
   if (s != TNLB_OK) {
      delete seg;
      return s;
   }
   *out = seg;
   return TNLB_OK;
}
