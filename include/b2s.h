/*
 * b2s.h — C ABI of libb2sparse.so, a B200-native (sm_100a) implementation of
 * TNL's sparse hot path: SparseMatrix<Real, Devices::Cuda, int>::vectorProduct
 * over the CSR, Ellpack, SlicedEllpack, ChunkedEllpack and BiEllpack segment
 * layouts, the Algorithms reduce/scan primitives beneath it, and the
 * Solvers::Linear CG / BICGStab / GMRES loops.
 *
 * Plain pointers, sizes and enums only: no C++ or torch types cross this
 * boundary. Every entry point returns a b2s_status; the text of the last
 * error of the calling thread is available from b2s_last_error().
 *
 * Citations name the TNL interface each entry point replaces (paths relative
 * to TNL's src/ tree).
 */
#ifndef B2S_H
#define B2S_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define B2S_ABI_VERSION 2

/* Status codes. TNL reports the same conditions as C++ exceptions
 * (Exceptions::CudaBadAlloc, CudaRuntimeError, std::logic_error) or as
 * `false` from solve() (TNL/Solvers/IterativeSolver.hpp:121-146). */
typedef enum
{
   B2S_OK = 0,
   B2S_NOT_CONVERGED = 1,  /* iteration limit reached (solve() == false)          */
   B2S_NAN = 2,            /* residue became NaN                                  */
   B2S_DIVERGED = 3,       /* residue above the divergence residue                */
   B2S_OOM = 4,            /* device allocation failed (CudaBadAlloc)             */
   B2S_CUDA_ERROR = 5,     /* CUDA runtime error (CudaRuntimeError)               */
   B2S_TIMEOUT = 6,        /* a bounded device wait gave up                       */
   B2S_INVALID_ARG = 7,    /* bad pointer / size / enum                           */
   B2S_INDEX_OVERFLOW = 8, /* layout needs more slots than a 32-bit index holds   */
   B2S_UNSUPPORTED = 9,    /* option not implemented                              */
   B2S_BREAKDOWN = 10,     /* Krylov breakdown (zero pivot in the GMRES update)   */
   B2S_BUDGET = 11,        /* request exceeds the memory budget of a server       */
   B2S_CANCELLED = 12,     /* request dropped by b2s_server_destroy before admission */
   B2S_IO_ERROR = 13       /* file could not be opened / read / written           */
} b2s_status;

typedef enum
{
   B2S_F64 = 0,
   B2S_F32 = 1,
   /* Binary matrix, TNL's SparseMatrix< bool, ... > (Matrices/SparseMatrix.h:23-26):
    * only the column indexes are stored; every stored element is 1. Its product
    * runs in TNL's ComputeReal = Index (SparseMatrixView.h:22-30): each stored
    * column adds (int) x[column] (truncation toward zero) to an int32 row sum,
    * and alpha / beta act as ints (truncated), in TNL's keepers. Vectors are
    * FP64 or FP32 (b2s_spmv_ex). Creation (b2s_matrix_create, and
    * b2s_matrix_from_coo, where every triplet stores its column whatever its
    * value) and the product are provided; the solvers, conversion, permutation
    * and file I/O of binary matrices return B2S_UNSUPPORTED. */
   B2S_BOOL = 2
} b2s_dtype;

/* Segment layouts: TNL/Algorithms/Segments/{CSR,Ellpack,SlicedEllpack,
 * ChunkedEllpack,BiEllpack}.h. The padded layouts use TNL's Devices::Cuda
 * element organization (ColumnMajorOrder, Segments/ElementsOrganization.h:21-29),
 * Ellpack alignment 32, SlicedEllpack slice 32, BiEllpack warp 32,
 * ChunkedEllpack 256 chunks per slice with desired chunk size 16. */
typedef enum
{
   B2S_CSR = 0,
   B2S_ELLPACK = 1,
   B2S_SLICED_ELLPACK = 2,
   B2S_CHUNKED_ELLPACK = 3,
   B2S_BIELLPACK = 4,
   B2S_MULTIDIAGONAL = 5  /* Matrices::MultidiagonalMatrix (MultidiagonalMatrix.h:27-60,
                             MultidiagonalMatrixView.hpp:488-528): no column indices; the
                             diagonals are the distinct (column - row) offsets of the input
                             pattern, ascending, at most 128; values ColumnMajor as on
                             Devices::Cuda (details/MultidiagonalMatrixIndexer.h): element d
                             of row r at d * nonemptyRows + r, absent entries 0; columns
                             outside [0, cols) are skipped */
} b2s_format;

typedef enum
{
   B2S_HOST = 0,  /* pointers refer to host memory (pinned or pageable) */
   B2S_DEVICE = 1 /* pointers refer to memory of the current device     */
} b2s_memory;

typedef struct b2s_matrix_t* b2s_matrix;
typedef struct b2s_solver_t* b2s_solver;

/* CUDA stream as an opaque pointer (cudaStream_t); NULL = legacy default stream. */
typedef void* b2s_stream;

const char* b2s_status_string( b2s_status s );
/* Message of the last failing call on this host thread ("" if none). */
const char* b2s_last_error( void );
int b2s_abi_version( void );

/* ------------------------------------------------------------------------
 * Matrices
 * ------------------------------------------------------------------------ */

/* Kernel choice for the CSR layout (TNL names its CSR kernels by segment type,
 * Segments/CSR.h:577-605). B2S_CSR_AUTO lets the library pick by row-length
 * statistics; the others force one path. */
typedef enum
{
   B2S_CSR_AUTO = 0,
   B2S_CSR_SCALAR = 1,   /* one thread per row                        */
   B2S_CSR_VECTOR = 2,   /* 2..32 threads per row (threads_per_row)   */
   B2S_CSR_ADAPTIVE = 3  /* nnz-balanced row blocks                   */
} b2s_csr_kernel;

typedef struct
{
   int32_t csr_kernel;      /* b2s_csr_kernel                                    */
   int32_t threads_per_row; /* CSR vector kernel: 0 = choose from mean row length */
   int32_t keep_fp32_copy;  /* also keep an FP32 copy of the values (mixed precision) */
   int32_t slice_size;      /* SlicedEllpack< ..., SliceSize >: 0 = 32 (TNL's default), or 8, 16, 64 */
   int32_t csr_row_groups;  /* adaptive CSR: 0 = 32-row groups staged in shared memory when every
                               group holds <= 256 nonzeros, -1 = nnz windows only            */
   int32_t symmetric;       /* 1: SparseMatrix< ..., SymmetricMatrix, Segments >: only the
                               lower triangle (column <= row) is stored and A = L + L^T -
                               diag(L); every layout (Matrices/SparseMatrixView.hpp:413-476) */
   int32_t reserved[ 2 ];
} b2s_matrix_opts;

void b2s_matrix_opts_default( b2s_matrix_opts* o );

/* Build a matrix of layout `format` and value type `dtype` from a CSR
 * description (offsets[rows+1], columns[nnz], values[nnz] of type
 * `values_dtype`), in host or device memory. For dtype B2S_BOOL, values may be
 * NULL (every entry is stored); otherwise entries with value 0 are not stored,
 * as in TNL's assignment of a real matrix to a binary one (operator=), and the
 * CSR rows are compacted (no -1 slots, see the CSR note below).
 *
 * Replaces TNL's assembly + conversion sequence
 *   SparseMatrix::setDimensions / setRowCapacities (Matrices/SparseMatrix.hpp:284-304)
 *   SparseMatrix::operator=( const RHSMatrix& )      (Matrices/SparseMatrix.hpp:1069-1193)
 * with the same semantics: for format B2S_CSR the arrays are taken as given;
 * for the padded layouts the row capacities are the CSR row lengths, explicit
 * zero values are dropped, unused slots hold column -1 and value 0, and the
 * segment metadata are bit-identical to TNL's Devices::Cuda segments. */
b2s_status b2s_matrix_create( b2s_format format, b2s_dtype dtype, int32_t rows, int32_t cols, int64_t nnz,
                              const int32_t* offsets, const int32_t* columns, const void* values,
                              b2s_dtype values_dtype, b2s_memory where, const b2s_matrix_opts* opts,
                              b2s_stream stream, b2s_matrix* out );

/* Convert into another layout / value type: SparseMatrix::operator=
 * (Matrices/SparseMatrix.hpp:1069-1193), device to device, from any layout
 * (padding and zero values of the source are not copied). */
b2s_status b2s_matrix_convert( b2s_matrix src, b2s_format format, b2s_dtype dtype, const b2s_matrix_opts* opts,
                               b2s_stream stream, b2s_matrix* out );

b2s_status b2s_matrix_destroy( b2s_matrix m );

/* ------------------------------------------------------------------------
 * Assembly and MatrixMarket files
 * ------------------------------------------------------------------------ */

/* How b2s_matrix_from_coo merges repeated (row, column) pairs, in input order. */
typedef enum
{
   B2S_DUP_SET = 0, /* SparseMatrix::setElement: value = 0 * old + new (the last one wins) */
   B2S_DUP_ADD = 1  /* SparseMatrix::addElement: value = old + new                       */
} b2s_duplicates;

/* Assemble a matrix on the device from `count` triplets (0-based row and
 * column indexes, values of type values_dtype), in host or device memory.
 * Replaces setDimensions + setRowCapacities( row_capacities ) + setElement /
 * addElement for every triplet in order (Matrices/SparseMatrix.hpp:284-304,
 * SparseMatrixView.hpp:256-340): rows sorted by column, repeated pairs merged
 * by `duplicates`, explicit zeros stored. row_capacities (rows entries, same
 * memory as the triplets) may be NULL: the per-row triplet counts, as
 * MatrixReader sets them. A row with more distinct columns than its capacity
 * is B2S_INVALID_ARG (TNL: "The capacity of the sparse matrix row ... was
 * exceeded"). The padded layouts keep the capacities (unused slots are
 * padding); CSR rows hold exactly the merged elements. */
b2s_status b2s_matrix_from_coo( b2s_format format, b2s_dtype dtype, int32_t rows, int32_t cols, int64_t count,
                                const int32_t* row_indexes, const int32_t* column_indexes, const void* values,
                                b2s_dtype values_dtype, b2s_memory where, int32_t duplicates,
                                const int32_t* row_capacities, const b2s_matrix_opts* opts, b2s_stream stream,
                                b2s_matrix* out );

/* A MatrixMarket coordinate file as host triplets (owned by the library). */
typedef struct
{
   int32_t rows, cols;
   int64_t count;            /* triplets; a symmetric file contributes both triangles  */
   int32_t symmetric;        /* the header said "symmetric"                             */
   int32_t reserved;
   int32_t* row_indexes;     /* 0-based, in the order TNL's reader calls setElement     */
   int32_t* column_indexes;
   double* values;
} b2s_mtx;

/* MatrixReader::readMtx's parsing and checks (Matrices/MatrixReader.hpp:51-359):
 * header "%%MatrixMarket matrix coordinate(s) real general|symmetric", '%'
 * comment lines, a dimensions line, element lines of exactly three
 * space-separated tokens (atoi, atoi, atof). Errors give B2S_INVALID_ARG /
 * B2S_IO_ERROR with TNL's message in b2s_last_error(). */
b2s_status b2s_mtx_read( const char* path, b2s_mtx** out );
void b2s_mtx_free( b2s_mtx* m );

/* MatrixReader< Matrix, Devices::Cuda >::readMtx( fileName, matrix ): read,
 * then b2s_matrix_from_coo with B2S_DUP_SET. */
b2s_status b2s_matrix_read_mtx( const char* path, b2s_format format, b2s_dtype dtype, const b2s_matrix_opts* opts,
                                b2s_stream stream, b2s_matrix* out );

/* MatrixWriter::writeMtx( fileName, matrix ) (Matrices/MatrixWriter.hpp:103-128),
 * byte for byte: TNL's header, one line per nonzero value in storage order,
 * values with six significant digits. Any layout. */
b2s_status b2s_matrix_write_mtx( b2s_matrix m, const char* path );

/* SparseMatrix::save( fileName ) (Matrices/SparseMatrix.hpp:1233-1290, Object.hpp,
 * File.hpp): TNL's binary file of the matrix — object header ("TNLMN" and the
 * serialization type), rows, columns, the values and columnIndexes arrays, the
 * segments' own fields — as TNL writes it for Devices::Host CSR and for the
 * ColumnMajor padded layouts, so SparseMatrix::load reads it back. */
b2s_status b2s_matrix_save( b2s_matrix m, const char* path );

/* SparseMatrix::load( fileName ): the layout and value type named in the file
 * (CSR, Ellpack, SlicedEllpack, ChunkedEllpack, BiEllpack; double or float;
 * int indexes), the arrays as stored, after checks that every index derived
 * from them stays inside the storage. The file does not record SlicedEllpack's
 * slice size: opts->slice_size (0: 32). CSR slots left unused (column -1)
 * are dropped. B2S_IO_ERROR / B2S_INVALID_ARG with the reason. */
b2s_status b2s_matrix_load( const char* path, const b2s_matrix_opts* opts, b2s_stream stream, b2s_matrix* out );

typedef struct
{
   int32_t format, dtype, rows, cols;
   int64_t nnz;             /* stored nonzeros (zeros dropped for padded layouts) */
   int64_t storage_size;    /* TNL getStorageSize() of the segments              */
   int64_t device_bytes;    /* bytes this handle holds on the device             */
   int32_t csr_kernel;      /* effective CSR kernel                               */
   int32_t threads_per_row; /* effective threads per row (CSR vector)             */
   int32_t csr_path;        /* adaptive CSR kernel: 1 = 32-row groups, 2 = nnz windows, 0 = n/a */
   int32_t symmetric;       /* SymmetricMatrix: the lower triangle is stored       */
} b2s_matrix_info;

b2s_status b2s_matrix_get_info( b2s_matrix m, b2s_matrix_info* info );

/* Copy one storage array to host memory, in TNL's layout, so it can be
 * compared element by element with TNL's own arrays. Names:
 *   "values" (matrix dtype), "columnIndexes" (int32), and per layout
 *   CSR: "offsets"; Ellpack: "segmentSize","size","alignedSize";
 *   SlicedEllpack: "sliceOffsets","sliceSegmentSizes","size","alignedSize";
 *   ChunkedEllpack: "rowToChunkMapping","rowToSliceMapping","chunksToSegmentsMapping",
 *     "rowPointers","slices" (size,chunkSize,firstSegment,pointer per slice),
 *     "numberOfSlices","storageSize";
 *   BiEllpack: "rowPermArray","groupPointers","virtualRows","storageSize".
 * Index arrays and scalars are written as int64. With host_out == NULL only
 * *count is set. */
b2s_status b2s_matrix_export( b2s_matrix m, const char* name, void* host_out, int64_t capacity, int64_t* count );

/* Elements [first, first + count) of "values" (matrix dtype) or
 * "columnIndexes" (int32), in TNL's layout, so that storage arrays too large
 * to hold twice on the host can be compared or written piece by piece. Slots
 * past the allocated part (BiEllpack's unaddressed tail) read as padding.
 * Same arrays as b2s_matrix_export (SparseMatrix::getValues /
 * getColumnIndexes, Matrices/SparseMatrix.h:1249, Matrices/Matrix.h:247). */
b2s_status b2s_matrix_export_range( b2s_matrix m, const char* name, int64_t first, int64_t count, void* host_out );

/* y = alpha * A x + beta * y over rows [row_begin, row_end) (row_end == 0: all
 * rows). x and y have the matrix value type.
 * Replaces SparseMatrix::vectorProduct( in, out, matrixMultiplicator,
 * outVectorMultiplicator, begin, end ) (Matrices/SparseMatrix.h:1078-1085,
 * SparseMatrixView.hpp:390-490). With where == B2S_HOST, x is copied in and y
 * copied in (when beta != 0) and out on `stream`, and the call returns after
 * the result is on the host. */
b2s_status b2s_spmv( b2s_matrix A, const void* x, void* y, double alpha, double beta, int32_t row_begin,
                     int32_t row_end, b2s_memory where, b2s_stream stream );

/* b2s_spmv with the vector value type given: `vectors` is B2S_F64 or B2S_F32.
 * For an FP64 or FP32 matrix it must be the matrix's own value type; a binary
 * (B2S_BOOL) matrix takes either (x and y of the same type). Replaces
 * vectorProduct with any InVector / OutVector type of TNL's binary matrices
 * (Matrices/SparseMatrixView.hpp:390-490). */
b2s_status b2s_spmv_ex( b2s_matrix A, const void* x, void* y, b2s_dtype vectors, double alpha, double beta,
                        int32_t row_begin, int32_t row_end, b2s_memory where, b2s_stream stream );

/* Permutations (Matrices/MatrixPermutationApplier.h, Matrices/SparseOperations.h).
 * perm / iperm are int32 arrays in `where` memory; every index is range-checked.
 *
 * b2s_matrix_permute_rows: permuteMatrixRows( A, perm ) (MatrixPermutationApplier.h:17-62):
 *   row i of A becomes the old row perm[i]. CSR matrices (B2S_UNSUPPORTED for the
 *   padded layouts: permute the CSR matrix, then convert). The handle keeps its identity.
 * b2s_matrix_permute_columns: permuteMatrixColumns( A, iperm ) (:64-90): every stored
 *   column c becomes iperm[c]; slots keep their order (rows are not re-sorted); any layout.
 * b2s_matrix_reorder: reorderSparseMatrix( A, B, perm, iperm ) (SparseOperations_impl.h:253-312):
 *   a new CSR matrix B, row i = row perm[i] of A with columns iperm[c], sorted.
 * b2s_reorder_array: reorderArray( src, dest, perm ) (SparseOperations_impl.h:314-338):
 *   dest[i] = src[perm[i]] for 4- or 8-byte elements; device arrays.
 * A solver keeps the Jacobi diagonal it was created with: create solvers after permuting. */
b2s_status b2s_matrix_permute_rows( b2s_matrix A, const int32_t* perm, b2s_memory where, b2s_stream stream );
b2s_status b2s_matrix_permute_columns( b2s_matrix A, const int32_t* iperm, b2s_memory where, b2s_stream stream );
b2s_status b2s_matrix_reorder( b2s_matrix A, const int32_t* perm, const int32_t* iperm, b2s_memory where,
                               b2s_stream stream, b2s_matrix* out );
b2s_status b2s_reorder_array( int32_t element_size, int64_t n, const void* src, void* dest, const int32_t* perm,
                              b2s_stream stream );

/* Synchronize `stream` and report B2S_TIMEOUT if a bounded wait inside a kernel
 * working on A gave up since the last check (the flag is then cleared). TNL
 * checks the device after every launch (TNL_CHECK_CUDA_DEVICE,
 * Cuda/CheckDevice.h:36); device-vector calls here do not synchronize, so the
 * check is explicit. Host-vector b2s_spmv calls perform it themselves. */
b2s_status b2s_matrix_device_status( b2s_matrix A, b2s_stream stream );

/* ------------------------------------------------------------------------
 * Autotuner of the SpMV layout. TNL fixes the layout at compile time (the
 * Segments argument of SparseMatrix, Matrices/SparseMatrix.h:40-49); this
 * builds `src` (a CSR matrix) in every candidate layout — CSR adaptive (32-row
 * groups when they fit, and nnz windows), CSR vector with 1..32 threads per row, Ellpack, SlicedEllpack with slice 8, 16,
 * 32, 64, ChunkedEllpack, BiEllpack — times b2s_spmv on the device and
 * returns the fastest. Layouts whose padded storage (the slots allocated on the
 * device; BiEllpack allocates only the slots it addresses) exceeds
 * max_storage_ratio x nnz (or 32-bit indexing) are skipped. By default every
 * timed product starts with L2 evicted (a 256 MiB write and a 256 MiB read
 * between products, outside the timing), as a Krylov iteration over a matrix
 * larger than L2 meets it; warm_l2 = 1 times back-to-back products instead.
 * ------------------------------------------------------------------------ */
typedef struct
{
   int32_t reps;              /* timed products per candidate, default 10      */
   int32_t warm_l2;           /* 1: back-to-back products (L2 kept warm)        */
   double max_storage_ratio;  /* default 3.0                                    */
   int32_t reserved[ 4 ];
} b2s_tune_opts;

typedef struct
{
   int32_t format, csr_kernel, threads_per_row, slice_size; /* pass these to b2s_matrix_create */
   double spmv_us;            /* device time of one product in this layout      */
   int32_t candidates;        /* layouts timed                                  */
   int32_t csr_row_groups;    /* pass as b2s_matrix_opts::csr_row_groups        */
   int32_t reserved[ 4 ];
} b2s_tune_result;

typedef struct
{
   int32_t format, csr_kernel, threads_per_row, slice_size;
   int32_t skipped;           /* storage limit, 32-bit indexing, or (Multidiagonal) more than 128 diagonals */
   int32_t csr_row_groups;    /* CSR adaptive: the kernel that ran, 0 = 32-row groups,
                                 -1 = nnz windows (groups need every 32 rows <= 256 nonzeros) */
   int64_t storage_size;
   double spmv_us;            /* -1 when skipped                                */
} b2s_tune_entry;

void b2s_tune_opts_default( b2s_tune_opts* o );
/* `table` (optional, `capacity` entries) receives every candidate; *count
 * the number of candidates considered. */
b2s_status b2s_autotune_spmv( b2s_matrix src, b2s_dtype dtype, const b2s_tune_opts* opts, b2s_stream stream,
                              b2s_tune_result* best, b2s_tune_entry* table, int32_t capacity, int32_t* count );

/* ------------------------------------------------------------------------
 * Algorithms primitives on device vectors (Algorithms/reduce.h:71,
 * Containers/Expressions/ExpressionTemplates.h:391-476, Algorithms/scan.h).
 * Results land in device memory; deterministic (fixed reduction order).
 * ------------------------------------------------------------------------ */

/* *result = sum_i a[i]*b[i] (device double). a, b of type dtype. */
b2s_status b2s_dot( b2s_dtype dtype, int64_t n, const void* a, const void* b, double* result, b2s_stream stream );
/* *result = sqrt( sum_i a[i]^2 ) — lpNorm( a, 2.0 ). */
b2s_status b2s_norm2( b2s_dtype dtype, int64_t n, const void* a, double* result, b2s_stream stream );
/* y = alpha * x + beta * y (vector expression assignment, detail/VectorAssignment.h). */
b2s_status b2s_axpby( b2s_dtype dtype, int64_t n, double alpha, const void* x, double beta, void* y,
                      b2s_stream stream );
/* dest[i] = src[idx[i]] for i < n, 4- or 8-byte elements, device arrays; an index
 * outside [0, src_size) gives 0. The pack step of a halo exchange (the send side
 * of TNL's distributed-array synchronizers, Containers/ByteArraySynchronizer.h). */
b2s_status b2s_gather( int32_t element_size, int64_t n, const void* src, int64_t src_size, const int32_t* idx,
                       void* dest, b2s_stream stream );
/* In-place exclusive / inclusive prefix sum of int32 values
 * (Algorithms::inplaceExclusiveScan / inplaceInclusiveScan). */
b2s_status b2s_scan_i32( int64_t n, int32_t* data, int32_t inclusive, b2s_stream stream );

/* Same result as b2s_scan_i32, but allocates no device memory. It is meant for
 * callers that cannot call cudaMalloc: an application that hands out every
 * byte of device memory through its own pool allocator or runs under a fixed
 * memory budget (a cudaMalloc beside the pool can fail or fragment it), and
 * latency-critical code that cannot afford the device-wide synchronization a
 * cudaFree implies. No counterpart in the reference (TNL's scan allocates its
 * buffers). Its working memory is a fixed array inside the library, one per
 * device, held until the process exits: n is limited to 67,108,864 elements
 * (larger n returns B2S_INVALID_ARG). All calls on a device share that array
 * and it keeps the previous call's contents, so calls that overlap on the GPU
 * race. The first call on a device looks the array up (cudaGetSymbolAddress)
 * and remembers the address for that device's current context; the first call
 * after a cudaDeviceReset looks it up again. Make those calls before any stream
 * capture starts. Unlike b2s_scan_i32, which waits for its result, this call
 * is asynchronous on `stream`: synchronize with the stream before reading
 * `data` on the host or starting a call on another stream. */
b2s_status b2s_scan_i32_noalloc( int64_t n, int32_t* data, int32_t inclusive, b2s_stream stream );

/* ------------------------------------------------------------------------
 * Krylov solvers
 * ------------------------------------------------------------------------ */

typedef enum
{
   B2S_CG = 0,
   B2S_BICGSTAB = 1,
   B2S_GMRES = 2,
   B2S_TFQMR = 3,     /* Solvers::Linear::TFQMR */
   B2S_BICGSTABL = 4, /* Solvers::Linear::BICGStabL (BiCGStab(ell)) */
   B2S_JACOBI = 5,    /* Solvers::Linear::Jacobi (Jacobi.hpp:67-128): weighted Jacobi sweeps,
                         two per loop pass, the residue every `residue_period` iterations */
   B2S_SOR = 6        /* Solvers::Linear::SOR (SOR.hpp:66-118): the sequential forward sweep
                         (x_i += omega / a_ii (b_i - row_i . x) with the rows before i already
                         updated), as TNL's Devices::Host solver computes it; TNL's Devices::Cuda
                         sweep updates x in place from all threads at once and is not
                         reproducible. The sweep runs as a dependency kernel over the levels
                         of the strict lower triangle (bounded waits, B2S_TIMEOUT) */
} b2s_solver_kind;

typedef enum
{
   B2S_PRECOND_NONE = 0,
   B2S_PRECOND_JACOBI = 1, /* Preconditioners::Diagonal */
   B2S_PRECOND_ILU0 = 2,   /* Preconditioners::ILU0 (TNL: Devices::Host, or cuSPARSE on Cuda) */
   B2S_PRECOND_ILUT = 3    /* Preconditioners::ILUT (ILUT.hpp:33-289; TNL: Devices::Host only, its
                              Cuda specialization throws): TNL's host factorization with
                              "ilut-p" extra entries per factor row and "ilut-threshold"
                              dropping, applied on the device like ILU(0) */
} b2s_precond_kind;

/* A preconditioner on its own: Preconditioner::update( matrix ) at creation,
 * Preconditioner::solve( b, x ) per application
 * (Solvers/Linear/Preconditioners/Preconditioner.h, Diagonal.hpp:13-47,
 * ILU0.hpp:23-144). ILU(0) needs a square matrix with the columns of each row
 * sorted and every diagonal entry stored ("A(i, i) is missing" otherwise); it
 * factorizes on the device and applies L^-1 then U^-1 with bounded-wait
 * dependency kernels (B2S_TIMEOUT if a wait gives up). x may be b. */
typedef struct b2s_precond_t* b2s_precond;
b2s_status b2s_precond_create( b2s_matrix A, int32_t kind, b2s_stream stream, b2s_precond* out );
/* ILUT with its parameters ("ilut-p" >= 0, default 0; "ilut-threshold", default
 * 1e-4; ILUT.h:79-82); b2s_precond_create( A, B2S_PRECOND_ILUT, ... ) uses the
 * defaults. The factorization runs on the host (it is TNL's sequential
 * algorithm), the application on the device. */
b2s_status b2s_precond_create_ilut( b2s_matrix A, int32_t p, double threshold, b2s_stream stream, b2s_precond* out );
b2s_status b2s_precond_solve( b2s_precond M, const void* b, void* x, b2s_memory where, b2s_stream stream );
b2s_status b2s_precond_destroy( b2s_precond M );

typedef enum
{
   B2S_GMRES_CGS = 0,
   B2S_GMRES_CGSR = 1,
   B2S_GMRES_MGS = 2,
   B2S_GMRES_MGSR = 3,
   B2S_GMRES_CWY = 4 /* Householder reflections in compact WY form (GMRES.hpp:348-640) */
} b2s_gmres_variant;

typedef enum
{
   B2S_PRECISION_PLAIN = 0, /* everything in the matrix value type                       */
   B2S_PRECISION_MIXED = 1  /* FP32 matrix + vectors inside FP64 iterative refinement    */
} b2s_precision;

/* Solver options. Field names follow TNL's configuration keys
 * (Solvers/IterativeSolver.hpp:16-56, Linear/GMRES.hpp:19-67,
 * Linear/BICGStab.hpp:13-29, Linear/BICGStabL.hpp:19-40); defaults are TNL's. */
typedef struct
{
   int32_t solver;                /* b2s_solver_kind                                         */
   int32_t preconditioner;        /* b2s_precond_kind                                        */
   double convergence_residue;    /* "convergence-residue", default 1e-6                     */
   double divergence_residue;     /* "divergence-residue", default DBL_MAX                    */
   int64_t max_iterations;        /* "max-iterations", default 1e9                           */
   int64_t min_iterations;        /* "min-iterations", default 0                             */
   int32_t gmres_variant;         /* "gmres-variant", default MGSR                           */
   int32_t gmres_restarting_min;  /* "gmres-restarting-min", default 10                      */
   int32_t gmres_restarting_max;  /* "gmres-restarting-max", default 10                      */
   int32_t gmres_restarting_step_min; /* default 3 */
   int32_t gmres_restarting_step_max; /* default 3 */
   int32_t bicgstab_exact_residue; /* "bicgstab-exact-residue", default 0                    */
   int32_t precision;             /* b2s_precision                                            */
   double inner_tolerance;        /* mixed: relative reduction asked of each FP32 inner solve
                                     (GMRES, TFQMR, BiCGStab(ell): not below 1e-6)             */
   int32_t max_refinements;       /* mixed: outer refinement steps, default 20                */
   int32_t check_interval;        /* iterations per device-side graph chunk (0 = auto)        */
   int32_t graphs;                /* 0: capture iteration chunks into CUDA graphs (default);
                                     1: launch directly (cheaper for a solver used once on a
                                     small system: no graph capture and instantiation)       */
   int32_t bicgstab_ell;          /* "bicgstab-ell" (BICGStabL), default 1; at most 16        */
   double omega;                  /* "jacobi-omega" / "sor-omega", default 1                   */
   int32_t residue_period;        /* "residue-period" (Jacobi, SOR), default 4                 */
   int32_t ilut_p;                /* "ilut-p" (preconditioner ILUT), default 0                 */
   double ilut_threshold;         /* "ilut-threshold", default 1e-4                            */
   int32_t reserved[ 2 ];
} b2s_solve_opts;

void b2s_solve_opts_default( b2s_solve_opts* o );

typedef struct
{
   int32_t status;          /* b2s_status of the solve                                  */
   int32_t converged;       /* TNL's solve() return value                               */
   int64_t iterations;      /* IterativeSolver::getIterations() (inner iterations total) */
   double residue;          /* IterativeSolver::getResidue() of the last (inner) solve   */
   double true_residual;    /* ||b - A x|| / ||b|| in FP64 after the solve               */
   int64_t refinements;     /* mixed precision: outer steps taken                        */
   double device_ms;        /* device time of the solve (CUDA events)                    */
} b2s_solve_report;

/* setMatrix + setup: LinearSolver::setMatrix (Solvers/Linear/LinearSolver.h:121),
 * setPreconditioner (:132), setup( ParameterContainer ) (:109-113). The
 * solver keeps its work vectors on the device between solves. */
b2s_status b2s_solver_create( b2s_matrix A, const b2s_solve_opts* opts, b2s_solver* out );
b2s_status b2s_solver_destroy( b2s_solver s );

/* bool solve( ConstVectorViewType b, VectorViewType x ) (Solvers/Linear/LinearSolver.h:155-156):
 * x is the initial guess on entry and the solution on exit. Returns B2S_OK when
 * converged, B2S_NOT_CONVERGED / B2S_NAN / B2S_DIVERGED as TNL's solve()
 * returns false, other codes on errors. b and x have the matrix value type
 * (FP64 for mixed precision). */
b2s_status b2s_solve( b2s_solver s, const void* b, void* x, b2s_memory where, b2s_stream stream,
                      b2s_solve_report* report );

/* ------------------------------------------------------------------------
 * Batched solves in one persistent launch: many independent SPD systems
 * (uneven sizes, 1..8 right-hand sides each) solved by CG with the Jacobi
 * preconditioner, the recurrence of Solvers/Linear/CG.hpp:17-104 run per
 * right-hand side. No counterpart in TNL, which solves one system per call.
 *
 * The systems are the diagonal blocks of one CSR matrix: system s owns rows
 * [row_ptr[s], row_ptr[s+1]) and its columns lie in the same range.
 * Right-hand sides and solutions are interleaved per system: element (i, j)
 * of system s is at vec(s) + i*nrhs[s] + j, vec(s) = sum over t < s of
 * rows(t)*nrhs(t). Report slots (iterations, residues) are numbered the same
 * way, one per right-hand side.
 * ------------------------------------------------------------------------ */
typedef struct b2s_batch_t* b2s_batch;

typedef struct
{
   int32_t preconditioner;      /* b2s_precond_kind, default JACOBI                   */
   int32_t cluster_size;        /* CTAs (SMs) per system: 0 = autotune, 1, 2, 4, 8    */
   double convergence_residue;  /* per right-hand side, TNL's CG residue, default 1e-8 */
   double divergence_residue;
   int64_t max_iterations;
   int64_t min_iterations;
   int32_t reserved[ 8 ];
} b2s_batch_opts;

typedef struct
{
   int64_t solves;              /* right-hand sides solved                            */
   int64_t converged;
   int64_t total_iterations;    /* summed over right-hand sides                       */
   int64_t max_iterations;
   double max_residue;
   double device_ms;            /* the persistent launch (CUDA events)                */
   int32_t cluster_size;        /* cluster size used (autotuned on the first solve)   */
   int32_t reserved0;
} b2s_batch_report;

void b2s_batch_opts_default( b2s_batch_opts* o );
/* row_ptr[nsys+1] and nrhs[nsys] are host arrays; the CSR arrays are in
 * `where` memory (FP64 values, int32 indices). */
b2s_status b2s_batch_create( int32_t nsys, const int64_t* row_ptr, const int32_t* nrhs, const int32_t* offsets,
                             const int32_t* columns, const double* values, b2s_memory where,
                             const b2s_batch_opts* opts, b2s_stream stream, b2s_batch* out );
/* Solve every system: B and X are device arrays in the interleaved layout,
 * X holds the initial guesses and receives the solutions. Returns B2S_OK
 * when every right-hand side converged, B2S_NOT_CONVERGED otherwise. */
b2s_status b2s_batch_solve( b2s_batch b, const double* B, double* X, b2s_stream stream, b2s_batch_report* report );
/* Per right-hand side results of the last solve (host arrays, any may be NULL). */
b2s_status b2s_batch_results( b2s_batch b, int64_t* iterations, double* residues, int32_t* statuses );
b2s_status b2s_batch_destroy( b2s_batch b );

/* ------------------------------------------------------------------------
 * Serving: a request server that keeps matrices and Krylov vectors in HBM,
 * admits solve requests by a device-memory budget and runs several of them
 * at once, each on its own streams (continuous batching). No counterpart in
 * TNL, which solves one system per call; each request runs the solvers above.
 * ------------------------------------------------------------------------ */
typedef struct b2s_server_t* b2s_server;

typedef struct
{
   int64_t memory_budget; /* bytes of device memory admitted requests may hold (default 150e9;
                             clamped to the device's free memory less 2 GiB)                */
   int32_t max_inflight;  /* requests on the device at once (worker slots), default 8       */
   int32_t mixed_min_rows;/* a request asking for mixed precision with fewer rows runs the plain
                             FP64 solver to the same tolerance: its vectors live in L2 and its
                             kernels are latency-bound, so FP32 would only add iterations.
                             0 = the default (2^19 rows), < 0 = always honour the request */
   int32_t reserved[ 6 ];
} b2s_server_opts;

void b2s_server_opts_default( b2s_server_opts* o );

/* One solve request. All pointers are host memory owned by the caller and
 * must stay valid until b2s_server_wait has returned the request's result;
 * x holds the initial guess on entry and receives the solution. */
typedef struct
{
   int32_t format;          /* b2s_format the matrix is stored in on the device      */
   int32_t rows;            /* square matrix: rows == cols                           */
   int64_t nnz;
   const int32_t* offsets;  /* CSR, FP64 values                                      */
   const int32_t* columns;
   const double* values;
   const double* b;
   double* x;
   b2s_solve_opts opts;     /* solver, tolerance, precision (mixed = FP32 + FP64 refinement) */
   int32_t reserved[ 8 ];
} b2s_request;

typedef struct
{
   int32_t status;          /* b2s_status of the solve (B2S_BUDGET: larger than the whole budget) */
   int32_t precision;       /* b2s_precision the solve ran in (see mixed_min_rows)  */
   b2s_solve_report report;
   int64_t t_submit_ns;     /* b2s_server_clock_ns() at submit, admission and completion */
   int64_t t_admit_ns;
   int64_t t_done_ns;
   int64_t device_bytes;    /* budget the request reserved                          */
   int64_t t_built_ns;      /* matrix and solver built on the device                 */
   int64_t t_solved_ns;     /* solve returned (solution on the host)                 */
} b2s_request_result;

typedef struct
{
   int64_t memory_budget, reserved_bytes, peak_reserved_bytes;
   int64_t pending, inflight, peak_inflight, completed;
} b2s_server_stats;

/* Monotonic clock of the server's timestamps, in nanoseconds. */
int64_t b2s_server_clock_ns( void );
b2s_status b2s_server_create( const b2s_server_opts* opts, b2s_server* out );
/* Queue a request; returns at once with a ticket. */
b2s_status b2s_server_submit( b2s_server s, const b2s_request* req, int64_t* ticket );
/* Wait up to timeout_seconds (< 0: no limit) for a request; on B2S_OK `out`
 * holds its result and the ticket is released. B2S_TIMEOUT: not done yet. */
b2s_status b2s_server_wait( b2s_server s, int64_t ticket, double timeout_seconds, b2s_request_result* out );
b2s_status b2s_server_get_stats( b2s_server s, b2s_server_stats* out );
/* Finish the requests on the device, cancel the queued ones (B2S_CANCELLED)
 * and release everything. Call it after every b2s_server_wait has returned. */
b2s_status b2s_server_destroy( b2s_server s );

#ifdef __cplusplus
}
#endif
#endif
