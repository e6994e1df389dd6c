/*
 * tnlb200.h -- C ABI of libtnlb200.so: TNL's sparse segments formats, the
 * sparse matrix-vector product on them and the Krylov solvers built on it,
 * implemented for NVIDIA B200 (sm_100a).
 *
 * Conventions
 *  - Every entry point returns tnlb_status (0 = success) and never throws.
 *    tnlb_last_error() gives a message for the calling host thread.
 *  - Arrays named d_* are DEVICE pointers owned by the caller (values,
 *    column indexes, vectors); the library never frees them.  Arrays named
 *    h_* are host pointers.  Segment metadata (row pointers, slice offsets,
 *    chunk maps, permutations, block descriptors) lives in an opaque
 *    tnlb_segments handle created and destroyed here.
 *  - Index type is int32 (TNL's `int` Index), sizes of storage int64.
 *  - Work is enqueued on the given stream (0 = the calling thread's default
 *    stream) and is asynchronous unless the entry point says otherwise.  The
 *    reference's vectorProduct is synchronous on return
 *    (Algorithms/Segments/detail/ReducingOperations_CSR.h:327); the C++
 *    drop-in headers (include/tnlb/) add that synchronisation.
 *  - Every citation below is a path inside the reference project TNL 0.4.0.
 */
#ifndef TNLB200_H
#define TNLB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* tnlb_stream; /* == cudaStream_t */

/* Status codes.  The C++ layer maps them onto the reference's exceptions:
 * INVALID_ARGUMENT -> std::invalid_argument (Matrices/SparseMatrixBase.hpp:279-282),
 * OVERFLOW -> std::overflow_error (Algorithms/Segments/Ellpack.hpp:92-95),
 * CUDA -> Exceptions::BackendRuntimeError (Backend/Macros.h:14-24),
 * NOT_IMPLEMENTED -> Exceptions::NotImplementedError,
 * BREAKDOWN -> the `throw 1` of GMRES::update (Solvers/Linear/GMRES.hpp:657-667),
 * TIMEOUT -> a bounded device-side wait gave up (no reference counterpart),
 * IO -> std::runtime_error of the MatrixMarket reader and writer. */
typedef enum {
   TNLB_OK = 0,
   TNLB_ERR_INVALID_ARGUMENT = 1,
   TNLB_ERR_OVERFLOW = 2,
   TNLB_ERR_CUDA = 3,
   TNLB_ERR_NOT_IMPLEMENTED = 4,
   TNLB_ERR_BREAKDOWN = 5,
   TNLB_ERR_TIMEOUT = 6,
   TNLB_ERR_OUT_OF_MEMORY = 7,
   TNLB_ERR_IO = 8
} tnlb_status;

/* Real types of values and vectors. */
typedef enum { TNLB_F32 = 0, TNLB_F64 = 1 } tnlb_real;

/* Segment formats: Algorithms/Segments/{CSR,Ellpack,SlicedEllpack,
 * ChunkedEllpack,BiEllpack,AdaptiveCSR}.h. */
typedef enum {
   TNLB_CSR = 0,
   TNLB_ELLPACK = 1,
   TNLB_SLICED_ELLPACK = 2,
   TNLB_CHUNKED_ELLPACK = 3,
   TNLB_BIELLPACK = 4,
   TNLB_ADAPTIVE_CSR = 5
} tnlb_format;

/* ElementsOrganization (Algorithms/Segments/ElementsOrganization.h:15-32);
 * the GPU default of the reference is column-major. */
typedef enum { TNLB_COLUMN_MAJOR = 0, TNLB_ROW_MAJOR = 1 } tnlb_organization;

/* SpMV kernel selection, mirroring Segments::LaunchConfiguration
 * (Algorithms/Segments/LaunchConfiguration.h:18-86) and the legacy kernel
 * classes of Algorithms/SegmentsReductionKernels (CSRScalarKernel,
 * CSRVectorKernel, CSRLightKernel, CSRAdaptiveKernel, ...).
 *  TNLB_KERNEL_DEFAULT   -- the tuned kernel of the format (for CSR: one
 *                           thread per row when no row holds more than 16
 *                           entries, else the nnz-balanced tile kernel);
 *  TNLB_KERNEL_SCALAR    -- one thread per segment (Fixed, TPS 1);
 *  TNLB_KERNEL_VECTOR    -- `threads_per_segment` lanes per segment
 *                           (Fixed TPS 2..32, Warp = 32, 64/128 multi-warp);
 *  TNLB_KERNEL_LIGHT     -- TPS picked from the mean segment length as in
 *                           LaunchConfigurationSetter_LightCSR.h:30-58;
 *  TNLB_KERNEL_ADAPTIVE  -- the AdaptiveCSR block-descriptor kernel (CSR and
 *                           AdaptiveCSR only);
 *  TNLB_KERNEL_TILE      -- CSR: the nnz-balanced merge-path tile kernel
 *                           whatever the row lengths (no reference
 *                           counterpart; DynamicGrouping is the nearest).
 * Formats other than CSR accept DEFAULT and, where the reference offers a
 * TPS choice (Ellpack, SlicedEllpack), VECTOR. */
typedef enum {
   TNLB_KERNEL_DEFAULT = 0,
   TNLB_KERNEL_SCALAR = 1,
   TNLB_KERNEL_VECTOR = 2,
   TNLB_KERNEL_LIGHT = 3,
   TNLB_KERNEL_ADAPTIVE = 4,
   TNLB_KERNEL_TILE = 5
} tnlb_kernel;

typedef struct tnlb_segments tnlb_segments;

/* Sizes of a built segments object (mirrors getSegmentCount, getElementCount,
 * getStorageSize and the per-format metadata sizes). */
typedef struct {
   int32_t format;           /* tnlb_format */
   int32_t organization;     /* tnlb_organization */
   int32_t segments;         /* getSegmentCount() */
   int32_t reserved0;
   int64_t elements;         /* getElementCount(): sum of segment sizes */
   int64_t storage;          /* getStorageSize(): slots incl. padding */
   int32_t segment_size;     /* Ellpack: getSegmentSize() */
   int32_t aligned_size;     /* Ellpack: getAlignedSize() */
   int32_t slices;           /* SlicedEllpack slices / ChunkedEllpack numberOfSlices / BiEllpack strips */
   int32_t chunks_in_slice;  /* ChunkedEllpack: 256 */
   int64_t acsr_blocks[6];   /* AdaptiveCSR: descriptor count per value-size log 0..5 */
} tnlb_segments_info;

/* Metadata arrays that can be read back (tnlb_segments_read_metadata). */
typedef enum {
   TNLB_META_OFFSETS = 0,              /* CSR / AdaptiveCSR: int32[n+1] */
   TNLB_META_SLICE_OFFSETS = 1,        /* SlicedEllpack: int32[slices+1] */
   TNLB_META_SLICE_SEGMENT_SIZES = 2,  /* SlicedEllpack: int32[slices] */
   TNLB_META_CH_SLICE_SIZE = 3,        /* ChunkedEllpack slices[].size: int32[slices] */
   TNLB_META_CH_SLICE_CHUNK_SIZE = 4,  /* slices[].chunkSize */
   TNLB_META_CH_SLICE_FIRST = 5,       /* slices[].firstSegment */
   TNLB_META_CH_SLICE_POINTER = 6,     /* slices[].pointer */
   TNLB_META_CH_SEGMENT_TO_CHUNK = 7,  /* int32[n] */
   TNLB_META_CH_SEGMENT_TO_SLICE = 8,  /* int32[n] */
   TNLB_META_CH_SEGMENT_POINTERS = 9,  /* int32[n+1] */
   TNLB_META_CH_CHUNKS_TO_SEGMENTS = 10, /* int32[slices*chunks_in_slice] */
   TNLB_META_BI_PERMUTATION = 11,      /* BiEllpack: int32[n] */
   TNLB_META_BI_GROUP_POINTERS = 12    /* BiEllpack: int32[strips*6+1] */
} tnlb_metadata;

/* AdaptiveCSR block descriptor (non-union layout of
 * Algorithms/Segments/detail/CSRAdaptiveKernelBlockDescriptor.h:134-199). */
typedef struct {
   uint8_t type; /* LONG = 0, STREAM = 1, VECTOR = 2 */
   uint8_t warp_idx;
   uint8_t warps_count;
   uint8_t reserved;
   int32_t first_segment;
   int32_t block_size;        /* elements covered (STREAM/VECTOR) */
   int32_t segments_in_block; /* STREAM/VECTOR */
} tnlb_acsr_block;

/* ------------------------------------------------------------ library */

/* Message of the last failed call on this host thread ("" if none). */
const char* tnlb_last_error(void);
/* Library version string. */
const char* tnlb_version(void);

/* ------------------------------------------------------------ segments */

/* Build a segments object from DEVICE segment sizes (row capacities) on the
 * GPU.  Replaces Segments::setSegmentsSizes of every format:
 * CSR.hpp:87-103, Ellpack.hpp:74-96, SlicedEllpack.hpp:116-150 (slice 32),
 * ChunkedEllpack.hpp:158-380 (256 chunks per slice, desired chunk size 16),
 * BiEllpack.hpp:106-342 (strips of 32), AdaptiveCSR.hpp:104-230.  Metadata
 * is bit-identical to the reference's Host builders.  Blocks until built.
 * Ellpack storage beyond int32 -> TNLB_ERR_OVERFLOW (Ellpack.hpp:92-95). */
tnlb_status tnlb_segments_create(tnlb_format format, tnlb_organization organization, const int32_t* d_sizes,
                                 int32_t segments, tnlb_stream stream, tnlb_segments** out);

/* Release a segments object (Segments::reset). Accepts NULL. */
tnlb_status tnlb_segments_destroy(tnlb_segments* seg);

/* Sizes of a segments object. */
tnlb_status tnlb_segments_get_info(const tnlb_segments* seg, tnlb_segments_info* info);

/* Copy one metadata array to host memory (for inspection and the bit-exact
 * checks against the reference's builders); `count` is the capacity of h_out
 * in int32 elements.  Blocks until copied. */
tnlb_status tnlb_segments_read_metadata(const tnlb_segments* seg, tnlb_metadata which, int32_t* h_out, int64_t count);

/* Copy the AdaptiveCSR descriptors of one value-size log (0..5: 1..32 B) to
 * host memory.  Blocks until copied. */
tnlb_status tnlb_segments_read_acsr_blocks(const tnlb_segments* seg, int32_t size_log, tnlb_acsr_block* h_out,
                                           int64_t count);

/* Global index of (segment, local) -- Segments::getGlobalIndex
 * (EllpackBase.hpp:110-117, SlicedEllpackBase.hpp:121-145,
 * detail/ChunkedEllpack.h:86-113, detail/BiEllpack.h:134-163).  Computes a
 * DEVICE array d_global[i] for the pairs (d_segment[i], d_local[i]). */
tnlb_status tnlb_segments_global_index(const tnlb_segments* seg, const int32_t* d_segment, const int32_t* d_local,
                                       int64_t count, int64_t* d_global, tnlb_stream stream);

/* ------------------------------------------------------------ matrices */

/* Fill a matrix stored in `seg` from a CSR matrix on the device: the
 * cross-format SparseMatrix::operator= (SparseMatrix.hpp:626-629 ->
 * copySparseToSparseMatrix, Matrices/SparseOperations.hpp:106-186).
 * Target columns start as the padding index -1 and values as 0; source
 * elements with value 0 or column -1 are skipped, the rest are packed into
 * local slots 0,1,2,... of their row.  d_cols/d_values have
 * info.storage slots.  The segment sizes of `seg` must be >= the source
 * row lengths. */
tnlb_status tnlb_matrix_fill_from_csr(const tnlb_segments* seg, tnlb_real real, const int32_t* d_rowptr,
                                      const int32_t* d_src_cols, const void* d_src_values, int32_t* d_cols,
                                      void* d_values, tnlb_stream stream);

/* y[begin:end] = alpha * (A x)[begin:end] + beta * y[begin:end]
 * -- SparseMatrixBase::vectorProduct (Matrices/SparseMatrixBase.h:1020-1035,
 * SparseMatrixBase.hpp:270-393) for a general (non-symmetric) matrix.
 * Padding slots (column -1) contribute 0; beta == 0 does not read y; end == 0
 * means all rows.  `kernel` and `threads_per_segment` select the kernel as in
 * LaunchConfiguration (threads_per_segment: power of two, 0 = automatic).
 * x has `columns` entries, y has info.segments entries. */
tnlb_status tnlb_spmv(const tnlb_segments* seg, tnlb_real real, const int32_t* d_cols, const void* d_values,
                      int32_t columns, const void* d_x, void* d_y, double alpha, double beta, int32_t begin,
                      int32_t end, tnlb_kernel kernel, int32_t threads_per_segment, tnlb_stream stream);

/* Number of CUDA kernels the most recent tnlb_spmv on this host thread
 * enqueued (for launch accounting). */
int32_t tnlb_spmv_last_launch_count(void);

/* y = alpha * A x + beta * y for a SYMMETRIC matrix of which one triangle is
 * stored (vectorProduct of SparseMatrix<..., SymmetricMatrix, ...>,
 * Matrices/SparseMatrixBase.hpp:296-330): a stored a_rc with c < r also adds
 * alpha a_rc x[r] to y[c].  As in the reference, y is first multiplied by
 * beta unless beta == 1 (y is read even when beta == 0) and the scattered
 * additions are atomic, so the last bits of y vary from call to call.
 * Rows [begin, end) (end == 0: all); any segment format.  Asynchronous. */
tnlb_status tnlb_spmv_symmetric(const tnlb_segments* seg, tnlb_real real, const int32_t* d_cols, const void* d_values,
                                const void* d_x, void* d_y, double alpha, double beta, int32_t begin, int32_t end,
                                tnlb_stream stream);

/* y = alpha * A^T x + beta * y (SparseMatrixBase::transposedVectorProduct,
 * Matrices/SparseMatrixBase.hpp:542-588): x has info.segments entries, y has
 * `columns`; only output entries with index in [begin, end) receive products
 * (end == 0: all columns), y is multiplied by beta unless beta == 1, and the
 * additions are atomic as in the reference.  Any segment format.
 * Asynchronous. */
tnlb_status tnlb_spmv_transposed(const tnlb_segments* seg, tnlb_real real, const int32_t* d_cols,
                                 const void* d_values, int32_t columns, const void* d_x, void* d_y, double alpha,
                                 double beta, int32_t begin, int32_t end, tnlb_stream stream);

/* y = alpha * A x + beta * y for a CSR matrix given as plain device arrays
 * (row offsets d_rowptr[rows + 1], d_cols / d_values[nnz], nnz == d_rowptr[rows]),
 * computed by the same tile kernels as tnlb_spmv with TNLB_KERNEL_TILE on
 * CSR segments and giving the same bits, but allocating no device memory: the tile plan and the
 * carries of rows split between tiles go to a statically sized scratch
 * array compiled into the library (5.2 MB per device).  No counterpart in
 * the reference, whose SpMV takes the segments' own arrays.
 *
 * For callers that must not allocate: code running while a caching
 * allocator or memory pool owns the device's free memory, code on a path
 * where cudaMalloc / cudaFree would synchronise the device and stall other
 * streams, and host code that holds CSR arrays from another library and no
 * segments handle.
 *
 * Limit: rows + nnz <= 67,108,864 (262,144 tiles of 256 rows + nonzeros);
 * larger matrices are rejected with TNLB_ERR_INVALID_ARGUMENT before any
 * launch.  nnz must equal d_rowptr[rows]: the value is not read back from
 * the device, and a mismatch is undefined behaviour (the tiles are cut from
 * nnz).  Nothing in the scratch has to start at zero: every call rewrites
 * what it reads.  Every call looks up the scratch address in the current
 * device's context (cudaGetSymbolAddress; nothing is cached, so a device
 * reset leaves no stale address); the first call on a device may load the
 * library's device code there, so make one call per device before capturing
 * a stream.  Calls that overlap on one device -- on two streams, or from two
 * host threads -- share the scratch and race: order them on one stream.
 * Enqueues three kernels on `stream`; returns before they finish. */
tnlb_status tnlb_spmv_csr_noalloc(tnlb_real real, int32_t rows, int32_t columns, int64_t nnz,
                                  const int32_t* d_rowptr, const int32_t* d_cols, const void* d_values,
                                  const void* d_x, void* d_y, double alpha, double beta, tnlb_stream stream);

/* ------------------------------------------------- device assembly */

/* The 2D Laplace operator of an N x N grid (identity rows on the boundary,
 * 1, 1, -4, 1, 1 inside) assembled on the GPU straight into the storage of
 * a matrix of any format -- SparseMatrixBase::forAllRows / forElements
 * (Matrices/SparseMatrixBase.h:589, 858) with the lambda of the reference's
 * sparse set-up benchmark (Documentation/UsersGuide/Matrices/
 * SparseMatrixSetup_Benchmark.cpp:157-198).  `seg` has N^2 segments whose
 * capacities hold the stencil (5 per row suffices); unused slots keep the
 * padding column -1.  Blocks until assembled. */
tnlb_status tnlb_matrix_assemble_laplace_2d(const tnlb_segments* seg, tnlb_real real, int32_t grid_size,
                                            int32_t* d_cols, void* d_values, tnlb_stream stream);

/* The device row offsets of CSR or AdaptiveCSR segments (n+1 entries, valid
 * while the segments live): row i owns storage slots [offsets[i],
 * offsets[i+1]).  The forElements template of include/tnlb/tnlb.hpp runs a
 * caller's device lambda on them (CSR::getGlobalIndex, CSRBase.hpp).  Other
 * formats give TNLB_ERR_INVALID_ARGUMENT. */
tnlb_status tnlb_segments_offsets_view(const tnlb_segments* seg, const int32_t** d_offsets);

/* ------------------------------------------------------ measurement */

/* The attainable rate of a CSR product's memory traffic (no counterpart in
 * the reference; a measurement kernel): moves exactly the bytes of
 * y = A x -- every column index and value streamed once, the row pointer
 * read once, y written once -- and, with mode 1, gathers x at every column
 * as the product does, but sums nothing by rows (y receives garbage).
 * Mode 0 streams without the gathers.  The time of this kernel bounds the
 * product on the same matrix from below.  Asynchronous. */
tnlb_status tnlb_bench_stream_gather(tnlb_real real, int32_t mode, int32_t rows, int64_t nnz, const int32_t* d_rowptr,
                                     const int32_t* d_cols, const void* d_values, const void* d_x, void* d_y,
                                     tnlb_stream stream);

/* ------------------------------------------------------------ files */

/* A CSR matrix in HOST memory, as read from a file. */
typedef struct {
   int32_t rows;
   int32_t columns;
   int64_t nnz;
   int32_t* rowptr; /* rows + 1 */
   int32_t* cols;   /* nnz, ascending in each row */
   double* values;  /* nnz */
} tnlb_host_csr;

/* Read a MatrixMarket file as MatrixReader::readMtx does
 * (Matrices/MatrixReader.hpp:18-330): coordinate real / integer / pattern,
 * general or symmetric; a repeated position keeps its last value; with
 * symmetric_storage != 0 (a SymmetricMatrix) the lower triangle is kept,
 * else a symmetric file is expanded to both triangles.  The arrays are
 * allocated here; release them with tnlb_host_csr_free.  Errors (with the
 * reader's messages) return TNLB_ERR_IO.  Host only: needs no GPU. */
tnlb_status tnlb_mtx_read(const char* path, int32_t symmetric_storage, tnlb_host_csr* out);
void tnlb_host_csr_free(tnlb_host_csr* m);

/* The stored elements of a matrix (any format) as host CSR in segment order,
 * padding dropped, values in FP64 -- what getRow() walks row by row.  The
 * arrays are allocated here; release them with tnlb_host_csr_free.
 * Synchronous. */
tnlb_status tnlb_matrix_to_host_csr(const tnlb_segments* seg, tnlb_real real, const int32_t* d_cols,
                                    const void* d_values, int32_t columns, tnlb_host_csr* out);

/* Transposition -- SparseMatrix::getTransposition (Matrices/SparseMatrix.hpp:
 * 495-551): B = multiplicator * A^T (A of any format, `columns` columns)
 * as device CSR arrays, B having `columns` rows.  Step 1 writes B's row
 * pointer (columns + 1 entries) into d_trowptr and its number of entries
 * (the stored, non-padding entries of A, zeros included) into *h_nnz; step
 * 2 writes B's columns and values (h_nnz entries each).  The entries of a
 * row of B come in ascending column order -- what the reference's
 * single-threaded build gives (its multi-threaded build leaves each row in
 * the order its atomic cursor was claimed).  A column index outside
 * [0, columns) is an invalid argument.  Synchronous. */
tnlb_status tnlb_matrix_transpose_rowptr(const tnlb_segments* seg, const int32_t* d_cols, int32_t columns,
                                         int32_t* d_trowptr, int64_t* h_nnz, tnlb_stream stream);
tnlb_status tnlb_matrix_transpose_fill(const tnlb_segments* seg, tnlb_real real, const int32_t* d_cols,
                                       const void* d_values, int32_t columns, double multiplicator,
                                       int32_t* d_tcols, void* d_tvalues, tnlb_stream stream);

/* TNL's binary matrix file (SparseMatrix::save / load,
 * Matrices/SparseMatrix.hpp:632-700, SparseMatrixBase.hpp:1148-1159): the
 * object header "TNLMN" + the matrix type string, size_t rows and columns,
 * the segments' own save() and the value and column arrays -- the bytes the
 * reference writes for the same matrix.  Two arrays of the reference hold
 * bytes it never initialises (ChunkedEllpack's slice records beyond
 * numberOfSlices, unset fields and padding of AdaptiveCSR descriptors);
 * those are written as zeros. */
typedef struct {
   int32_t format;       /* tnlb_format */
   int32_t organization; /* tnlb_organization (column-major for the CSR formats) */
   int32_t real;         /* tnlb_real */
   int32_t symmetric;    /* 1 for a SymmetricMatrix */
   int64_t rows;
   int64_t columns;
   int64_t storage;      /* slots of the value and column arrays */
   char type[512];       /* the object type string */
} tnlb_matrix_file_info;

/* Save a matrix (segments + device columns/values of `real` type) to `path`.
 * Synchronous.  I/O failure: TNLB_ERR_IO. */
tnlb_status tnlb_matrix_save(const char* path, const tnlb_segments* seg, tnlb_real real, const int32_t* d_cols,
                             const void* d_values, int32_t rows, int32_t columns, int32_t symmetric);
/* The header of a matrix file: format, organization, real type, symmetry,
 * dimensions, storage and the type string.  Host only.  A file that is not
 * a TNL object (wrong magic number), has an unsupported type or is
 * truncated: TNLB_ERR_IO with the reason. */
tnlb_status tnlb_matrix_file_info_read(const char* path, tnlb_matrix_file_info* info);
/* Load a matrix file: a new segments object built from the stored metadata
 * (no rebuild) into *out, and the values and columns copied into device
 * arrays of `capacity` >= info.storage slots (of the file's real type).
 * Synchronous. */
tnlb_status tnlb_matrix_load(const char* path, tnlb_segments** out, int32_t* d_cols, void* d_values,
                             int64_t capacity);

/* Write host CSR arrays as MatrixWriter::writeMtx does
 * (Matrices/MatrixWriter.hpp:107-129): "coordinate real general", 1-based
 * "row column value" lines of widths 9, 9, 12 at default stream precision,
 * zero values and padding (column -1) skipped.  Host only. */
tnlb_status tnlb_mtx_write(const char* path, int32_t rows, int32_t columns, const int32_t* h_rowptr,
                           const int32_t* h_cols, const double* h_values);

/* ------------------------------------------------------------ vectors */

/* Dot product (a, b) into a DEVICE scalar -- Containers/Expressions/
 * ExpressionTemplates.h:372-387 (the reference copies it to the host). */
tnlb_status tnlb_dot(tnlb_real real, int64_t n, const void* d_a, const void* d_b, double* d_result, tnlb_stream stream);

/* y = alpha * x + beta * y over n entries (device) -- the vector
 * assignment y = alpha * x + beta * y of Containers/detail/
 * VectorAssignment.h:35-203 through the expression templates; beta == 0
 * does not read y.  Asynchronous. */
tnlb_status tnlb_axpby(tnlb_real real, int64_t n, double alpha, const void* d_x, double beta, void* d_y,
                       tnlb_stream stream);

/* ------------------------------------------------------------ solvers */

/* FGMRES: restarted GMRES with right, flexible preconditioning (the
 * preconditioned basis is kept; residues are unpreconditioned).  No
 * counterpart in the reference; its orthogonalisation and Givens steps follow
 * GMRES.hpp:280-347, 731-770. */
/* TFQMR (Solvers/Linear/TFQMR.hpp:12-113), BiCGStab(ell)
 * (Solvers/Linear/BICGStabL.hpp:36-242) and IDR(s)
 * (Solvers/Linear/IDRs.hpp:50-250): the other solvers of the reference's
 * linear-solver benchmark. */
typedef enum {
   TNLB_SOLVER_CG = 0,
   TNLB_SOLVER_BICGSTAB = 1,
   TNLB_SOLVER_GMRES = 2,
   TNLB_SOLVER_FGMRES = 3,
   TNLB_SOLVER_TFQMR = 4,
   TNLB_SOLVER_BICGSTABL = 5,
   TNLB_SOLVER_IDRS = 6
} tnlb_solver_kind;
/* Preconditioners: none, Diagonal (Jacobi), ILU0, and factorised sparse
 * approximate inverses (no counterpart in the reference; Kolotilina-Yeremin
 * values on the lower triangle of A's pattern): FSAI M^-1 = G^T G for SPD
 * matrices, FSAI2 M^-1 = G_U G_L (two factors) for nonsymmetric ones. */
typedef enum {
   TNLB_PRECOND_NONE = 0,
   TNLB_PRECOND_JACOBI = 1,
   TNLB_PRECOND_ILU0 = 2,
   TNLB_PRECOND_FSAI = 3,
   TNLB_PRECOND_FSAI2 = 4,
   TNLB_PRECOND_ILUT = 5
} tnlb_precond_kind;

typedef struct tnlb_precond tnlb_precond;
/* GMRES::Variant (Solvers/Linear/GMRES.h:122-129). */
typedef enum { TNLB_GMRES_CGS = 0, TNLB_GMRES_CGSR = 1, TNLB_GMRES_MGS = 2, TNLB_GMRES_MGSR = 3, TNLB_GMRES_CWY = 4 } tnlb_gmres_variant;

/* Solver parameters: the setup() keys of IterativeSolver.hpp:14-36,
 * GMRES.hpp:20-37, BICGStab.hpp:14-21, BICGStabL.hpp:14-33 and
 * IDRs.hpp:18-34, with the reference's defaults filled in by
 * tnlb_solver_params_default. */
typedef struct {
   int32_t max_iterations;       /* max-iterations, default 1e9 */
   int32_t min_iterations;       /* min-iterations, default 0 */
   double convergence_residue;   /* convergence-residue, default 1e-6 */
   double divergence_residue;    /* divergence-residue, default DBL_MAX */
   int32_t gmres_variant;        /* gmres-variant (tnlb_gmres_variant), default MGSR */
   int32_t gmres_restarting_min; /* default 10 */
   int32_t gmres_restarting_max; /* default 10 */
   int32_t gmres_restarting_step_min; /* default 3 */
   int32_t gmres_restarting_step_max; /* default 3 */
   int32_t bicgstab_exact_residue;    /* default 0 */
   int32_t spmv_kernel;          /* tnlb_kernel used by the solver's products */
   int32_t bicgstab_ell;         /* bicgstab-ell (BiCGStab(ell)), default 1 */
   int32_t idr_s;                /* idr-s (IDR(s) shadow space), default 4 */
   int32_t idr_residual_smoothing; /* idr-residual-smoothing, default 0 */
   int32_t reliable_layout;      /* tnlb_solve_mixed_reliable's internal FP32 copies: 0 (default) the
                                    diagonal layout where the matrix fits it (the products of FSAI
                                    factors of more than 5 diagonals staged in shared memory by bulk
                                    copies), else CSR with 16-bit column offsets; 1 the 16-bit offsets
                                    only; 2 the diagonal layout read by ordinary loads throughout.
                                    All give the same row sums bit for bit */
   int32_t reliable_operator;    /* its FP32 copy of A: 0 (default) the row-excess form (each diagonal
                                    entry holds the row's FP64 sum; rows summed as
                                    s_i x_i + sum a_ij (x_j - x_i)) when every row has its diagonal
                                    entry; 1 the values as they are */
} tnlb_solver_params;

/* Result of a solve: getIterations(), getResidue() and the bool of solve(). */
typedef struct {
   int32_t converged;     /* solve() return value */
   int32_t iterations;    /* getIterations() */
   double residue;        /* getResidue(): the solver's stopping residue */
   int32_t status_detail; /* 0, or a tnlb_status for breakdowns/timeouts */
   int32_t fallback_iterations; /* tnlb_solve_mixed_reliable: FP64 iterations after a stall */
} tnlb_solve_result;

void tnlb_solver_params_default(tnlb_solver_params* p);

/* Solve A x = b on the GPU -- LinearSolver::solve (Solvers/Linear/
 * LinearSolver.h:157-158) of CG (CG.hpp:12-109), BICGStab (BICGStab.hpp:
 * 34-122) or GMRES (GMRES.hpp:73-180) with the Diagonal (Jacobi,
 * Preconditioners/Diagonal.hpp:15-43) or ILU0 (Preconditioners/ILU0.hpp:
 * 15-140; the reference has no GPU ILU(0), ILU0.h:121-143) preconditioner.
 * A is given by `seg` + d_cols/d_values (FP64 or FP32); b and x are device
 * vectors of the same real type; x holds the initial guess.  Synchronous.
 * Stopping rules follow IterativeSolver.hpp:98-143 exactly. */
tnlb_status tnlb_solve(tnlb_solver_kind solver, tnlb_precond_kind precond, const tnlb_solver_params* params,
                       const tnlb_segments* seg, tnlb_real real, const int32_t* d_cols, const void* d_values,
                       const void* d_b, void* d_x, tnlb_stream stream, tnlb_solve_result* result);

/* True residual ||b - A x|| / ||b|| in FP64 (Solvers/Linear/Utils/
 * LinearResidueGetter.hpp:11-23), computed on the GPU.  Synchronous. */
tnlb_status tnlb_true_residual(const tnlb_segments* seg, tnlb_real real, const int32_t* d_cols, const void* d_values,
                               const void* d_b, const void* d_x, tnlb_stream stream, double* h_result);

/* FP32-inner / FP64-outer iterative refinement (no counterpart in the
 * reference): the FP64 residual r = b - A x is formed with the FP64 values,
 * normalised, rounded to FP32 and solved with `inner_solver` (CG for SPD
 * matrices, FGMRES/GMRES/BiCGStab otherwise) on an FP32 copy of the values
 * to the inner solver's residue `inner_tolerance`; x += |r| d in FP64.  The
 * outer residual is computed exactly as tnlb_true_residual computes it.
 * The inner preconditioner is `inner` (an FP32 preconditioner of this
 * matrix, e.g. a learned FSAI) or, when NULL, one of kind `inner_precond`
 * built from the FP32 values.  Stops
 * when ||b - A x|| / ||b|| < params->convergence_residue (the TRUE FP64
 * residual) or after `max_outer` corrections.  result->iterations is the
 * total number of inner CG iterations; *outer_iterations the corrections.
 * Synchronous. */
tnlb_status tnlb_solve_mixed(const tnlb_solver_params* params, const tnlb_segments* seg, const int32_t* d_cols,
                             const double* d_values, const double* d_b, double* d_x, double inner_tolerance,
                             int32_t max_outer, tnlb_solver_kind inner_solver, tnlb_precond_kind inner_precond,
                             const tnlb_precond* inner, tnlb_stream stream, tnlb_solve_result* result,
                             int32_t* outer_iterations);

/* Mixed-precision PCG with reliable updates (no counterpart in the
 * reference).  CG iterates on an FP32 copy of the values, with vectors of
 * type `vectors` (TNLB_F32: FP32 vectors; TNLB_F64: FP64 vectors, only the
 * matrix and preconditioner stored in FP32) and dot products accumulated in
 * FP64.  Its correction is folded into the FP64 x, and the residual is
 * replaced by the FP64 b - A x, whenever the recursive residual norm has
 * fallen below max(delta * |r| at the last update,
 * convergence_residue * |b|).  The search direction is kept across an
 * update, so unlike tnlb_solve_mixed the Krylov space is not restarted.
 *
 * The preconditioner is `inner` (an FP32 Jacobi or symmetric FSAI
 * preconditioner of this matrix, e.g. a learned FSAI) or, when NULL, one of
 * kind `inner_precond` (NONE, JACOBI or FSAI) built from the FP32 values.
 * Stops when ||b - A x|| / ||b|| < params->convergence_residue (the TRUE
 * FP64 residual, computed as tnlb_true_residual computes it) or after
 * params->max_iterations iterations.
 *
 * The FP32 iteration has stalled when the true residual at the updates has
 * not halved within the last max(16384, iterations to the best residual so
 * far) iterations, or on a breakdown ((p, A p) zero or not finite) or a
 * non-finite residual (x then goes back to its last finite value); an
 * update is forced after 4096 iterations without one, so that a recursion
 * which stops falling is checked too.  After a stall the solve finishes
 * with FP64 Jacobi PCG from x, for the iterations left.
 * result->iterations counts all iterations (FP32 and FP64),
 * result->fallback_iterations the FP64 ones, result->residue is the true
 * residual, result->status_detail is 0, 2 when the FP64 fallback ran, or 1
 * on a stall with no iterations left, and *reliable_updates counts the
 * updates.  Synchronous. */
tnlb_status tnlb_solve_mixed_reliable(const tnlb_solver_params* params, const tnlb_segments* seg,
                                      const int32_t* d_cols, const double* d_values, const double* d_b, double* d_x,
                                      double delta, tnlb_real vectors, tnlb_precond_kind inner_precond,
                                      const tnlb_precond* inner, tnlb_stream stream, tnlb_solve_result* result,
                                      int32_t* reliable_updates);

/* Build a preconditioner for a matrix -- Preconditioner::update
 * (Preconditioners/Preconditioner.h:96-110; Diagonal.hpp:15-36,
 * ILU0.hpp:15-118).  The values must stay valid while it is used.
 * Blocks until built. */
tnlb_status tnlb_precond_create(tnlb_precond_kind kind, const tnlb_segments* seg, tnlb_real real,
                                const int32_t* d_cols, const void* d_values, tnlb_stream stream,
                                tnlb_precond** out);

/* Build an ILUT preconditioner (Preconditioners/ILUT.h, ILUT.hpp:27-258; the
 * reference has it on the host only): dual threshold -- entries below
 * tau * ||A_i|| dropped, at most (stored entries of A_i left of / from the
 * diagonal) + p kept per row in L / U -- factorised on the host with the
 * reference's arithmetic and selection, applied on the GPU by the
 * level-scheduled triangular solves of ILU0.  Setup keys "ilut-p"
 * (default 0) and "ilut-threshold" (default 1e-4).  Blocks until built. */
tnlb_status tnlb_precond_create_ilut(const tnlb_segments* seg, tnlb_real real, const int32_t* d_cols,
                                     const void* d_values, int32_t p, double threshold, tnlb_stream stream,
                                     tnlb_precond** out);

/* x = M^{-1} b -- Preconditioner::solve (Diagonal.hpp:40-43,
 * ILU0.hpp:121-140).  Synchronous. */
tnlb_status tnlb_precond_solve(const tnlb_precond* precond, const void* d_b, void* d_x, tnlb_stream stream);

/* The factors of an FSAI / FSAI2 / learned FSAI preconditioner, copied to
 * host memory as CSR: which = 0 gives G (G_L), which = 1 gives the second
 * factor as stored for the product (G^T, or G_U).  `capacity` bounds h_cols
 * and h_values; h_rowptr has n+1 entries.  Synchronous. */
tnlb_status tnlb_precond_read_factor(const tnlb_precond* precond, int32_t which, int32_t* h_rowptr, int32_t* h_cols,
                                     void* h_values, int64_t capacity);

/* Release a preconditioner.  Accepts NULL. */
tnlb_status tnlb_precond_destroy(tnlb_precond* precond);

/* tnlb_solve with a preconditioner built beforehand (NULL = none):
 * LinearSolver::setPreconditioner (LinearSolver.h:133-137) then solve. */
tnlb_status tnlb_solve_preconditioned(tnlb_solver_kind solver, const tnlb_precond* precond,
                                      const tnlb_solver_params* params, const tnlb_segments* seg, tnlb_real real,
                                      const int32_t* d_cols, const void* d_values, const void* d_b, void* d_x,
                                      tnlb_stream stream, tnlb_solve_result* result);

/* The ILU(0) factors computed on the GPU, copied to host memory: CSR pattern
 * of A (h_rowptr n+1, h_cols nnz) with L strictly below the diagonal (unit
 * diagonal implied) and U from the diagonal on in h_values (ILU0.hpp:15-118;
 * the reference stores U's rows in reverse order, the values are the same).
 * `capacity` bounds h_cols/h_values.  Synchronous. */
tnlb_status tnlb_ilu0_factors(const tnlb_segments* seg, tnlb_real real, const int32_t* d_cols, const void* d_values,
                              int32_t* h_rowptr, int32_t* h_cols, void* h_values, int64_t capacity,
                              tnlb_stream stream);

/* ------------------------------------------------- learned FSAI (new) */
/* A per-row network (32 -> 64 -> 64 -> 64 -> 8, ReLU, BF16 weights, FP32
 * accumulation) maps scale-free local coefficients of an SPD matrix A to the
 * values of G on a lower-triangular pattern of at most 8 entries per row:
 * the lower triangle of A (level 0) or of the pattern of A^2 (level 1, the
 * default: one level of fill); M^-1 = G^T G.  No counterpart in the
 * reference.  The features, network, output map, losses and parameter
 * layout are defined in oracle/lfsai_ref.py (FP64 restatement used by the
 * tests).  The dense layers run on tcgen05 tensor cores by default, forward
 * and backward. */
typedef struct tnlb_lfsai tnlb_lfsai;

/* Number of network parameters (10952). */
int64_t tnlb_lfsai_num_params(void);
/* New network with deterministic initial parameters from `seed`. */
tnlb_status tnlb_lfsai_create(uint64_t seed, tnlb_stream stream, tnlb_lfsai** out);
tnlb_status tnlb_lfsai_destroy(tnlb_lfsai* net);
/* Parameters (FP32, tnlb_lfsai_num_params entries) to / from host memory;
 * setting them resets the optimiser state. */
tnlb_status tnlb_lfsai_get_params(const tnlb_lfsai* net, float* h_out, int64_t count);
tnlb_status tnlb_lfsai_set_params(tnlb_lfsai* net, const float* h_in, int64_t count);
/* Gradient of the last tnlb_lfsai_gradient call, FP32, to host memory. */
tnlb_status tnlb_lfsai_get_grad(const tnlb_lfsai* net, float* h_out, int64_t count);
/* Run the dense layers on tcgen05 tensor cores (1, the default) or on CUDA
 * cores (0). */
tnlb_status tnlb_lfsai_set_tensor_cores(tnlb_lfsai* net, int32_t enable);
/* The pattern of G the network fills: 0 (lower triangle of A) or 1 (lower
 * triangle of the pattern of A^2, the default). */
tnlb_status tnlb_lfsai_set_level(tnlb_lfsai* net, int32_t level);
/* The two-factor form for nonsymmetric A (enable = 1): the network fills
 * G_L and H = G_U^T on the lower triangle of A (at most 4 entries a row),
 * M^-1 = G_U G_L as tnlb_precond_create with TNLB_PRECOND_FSAI2 builds it
 * classically; features and outputs as defined for it in
 * oracle/lfsai_ref.py; the probe loss (1/(n P)) sum_p ||z_p - G_L A G_U
 * z_p||^2 and the warm start (mode 1, towards the classical two-factor
 * values) train it. */
tnlb_status tnlb_lfsai_set_two_factor(tnlb_lfsai* net, int32_t enable);
/* Loss and gradient on one matrix, kept in the handle.  mode 0: probe loss
 * (1/(n P)) sum_p ||z_p - G A G^T z_p||^2 with P probe vectors stored one
 * after another in d_probes (device, n*P values of `real`); mode 1: warm
 * start, mean squared distance of the scaled outputs to the classical FSAI
 * values of the level-0 pattern (zero on fill entries); mode 2: Kaporin
 * loss log(trace(G A G^T)/n) - (2/n) sum_i log G'_ii, exact (no probes).
 * Synchronous. */
tnlb_status tnlb_lfsai_gradient(tnlb_lfsai* net, int32_t mode, const tnlb_segments* seg, tnlb_real real,
                                const int32_t* d_cols, const void* d_values, const void* d_probes, int32_t nprobes,
                                tnlb_stream stream, double* h_loss);
/* One Adam step (beta1 0.9, beta2 0.999, eps 1e-8) with learning rate lr. */
tnlb_status tnlb_lfsai_adam_step(tnlb_lfsai* net, double lr, tnlb_stream stream);
/* The preconditioner M^-1 = G^T G of a matrix, G from the network. */
tnlb_status tnlb_lfsai_precond_create(const tnlb_lfsai* net, const tnlb_segments* seg, tnlb_real real,
                                      const int32_t* d_cols, const void* d_values, tnlb_stream stream,
                                      tnlb_precond** out);
/* Features (n*32) and raw network outputs (n*8) of a matrix, to host memory
 * (either may be NULL).  Synchronous. */
tnlb_status tnlb_lfsai_eval(const tnlb_lfsai* net, const tnlb_segments* seg, tnlb_real real, const int32_t* d_cols,
                            const void* d_values, tnlb_stream stream, float* h_features, float* h_outputs);

/* Classical FSAI (Kolotilina-Yeremin, M^-1 = G^T G, SPD A) on the level-0
 * pattern (as tnlb_precond_create with TNLB_PRECOND_FSAI) or the level-1
 * pattern (lower triangle of the pattern of A^2, at most 32 entries per
 * row).  No counterpart in the reference.  Blocks until built. */
tnlb_status tnlb_precond_create_fsai(const tnlb_segments* seg, tnlb_real real, const int32_t* d_cols,
                                     const void* d_values, int32_t level, tnlb_stream stream, tnlb_precond** out);

#ifdef __cplusplus
}
#endif

#endif /* TNLB200_H */
