// Internal declarations of libb2sparse: error plumbing, the matrix handle,
// device helpers and the deterministic "partials + last block" reduction
// used by every kernel that produces a scalar.
#pragma once

#include "../../include/b2s.h"

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>
#include <memory>
#include <vector>

namespace b2s {

// ---------------------------------------------------------------------------
// Errors: every public entry point returns a status and records a message.
void set_error( const char* fmt, ... );
void clear_error();

#define B2S_TRY_CUDA( expr )                                                                        \
   do {                                                                                             \
      cudaError_t _e = ( expr );                                                                    \
      if( _e != cudaSuccess ) {                                                                     \
         ::b2s::set_error( "%s:%d %s: %s", __FILE__, __LINE__, #expr, cudaGetErrorString( _e ) );  \
         return _e == cudaErrorMemoryAllocation ? B2S_OOM : B2S_CUDA_ERROR;                         \
      }                                                                                             \
   } while( 0 )

#define B2S_TRY( expr )                    \
   do {                                    \
      b2s_status _s = ( expr );            \
      if( _s != B2S_OK )                   \
         return _s;                        \
   } while( 0 )

#define B2S_CHECK_ARG( cond, msg )                      \
   do {                                                 \
      if( ! ( cond ) ) {                                \
         ::b2s::set_error( "invalid argument: %s", msg ); \
         return B2S_INVALID_ARG;                        \
      }                                                 \
   } while( 0 )

inline cudaStream_t
as_stream( b2s_stream s )
{
   return reinterpret_cast< cudaStream_t >( s );
}

// Number of SMs of the current device (cached per device).
int num_sms();
int current_device();

// ---------------------------------------------------------------------------
// Stream-ordered allocation for the calling host thread. Server workers set
// it so that creating and destroying the handles of one request never waits
// for the other requests' kernels (cudaFree synchronizes the whole device;
// a pool allocation and free on the worker's own stream do not).
struct AllocCtx
{
   cudaMemPool_t pool;
   cudaStream_t stream;
   // a solver created on this thread runs on `solver_stream` with these two
   // timing events instead of creating (and later destroying) its own
   cudaStream_t solver_stream;
   cudaEvent_t ev0, ev1;
};
void set_thread_alloc_ctx( const AllocCtx* ctx );  // nullptr: cudaMalloc / cudaFree
const AllocCtx* thread_alloc_ctx();

// ---------------------------------------------------------------------------
// Device memory owned by a handle.
struct DevBuf
{
   void* p = nullptr;
   size_t bytes = 0;
   cudaStream_t pool_stream = nullptr;  // set when the memory came from a pool
   bool pooled = false;
   DevBuf() = default;
   DevBuf( const DevBuf& ) = delete;
   DevBuf& operator=( const DevBuf& ) = delete;
   DevBuf( DevBuf&& o ) noexcept : p( o.p ), bytes( o.bytes ), pool_stream( o.pool_stream ), pooled( o.pooled )
   {
      o.p = nullptr;
      o.bytes = 0;
      o.pooled = false;
   }
   DevBuf& operator=( DevBuf&& o ) noexcept
   {
      release();
      p = o.p;
      bytes = o.bytes;
      pool_stream = o.pool_stream;
      pooled = o.pooled;
      o.p = nullptr;
      o.bytes = 0;
      o.pooled = false;
      return *this;
   }
   ~DevBuf() { release(); }
   b2s_status alloc( size_t n );
   void release();
   template< typename T >
   T* as() const
   {
      return static_cast< T* >( p );
   }
};

// ---------------------------------------------------------------------------
// Layout constants (TNL defaults on Devices::Cuda).
constexpr int kEllAlign = 32;          // Ellpack< ..., Alignment = 32 >
constexpr int kSliceSize = 32;         // SlicedEllpack< ..., SliceSize = 32 >
constexpr int kBiWarp = 32;            // BiEllpack< ..., WarpSize = 32 >
constexpr int kBiLogWarp = 5;
constexpr int kBiGroups = kBiLogWarp + 1;
constexpr int kChunksInSlice = 256;    // ChunkedEllpack::chunksInSlice
constexpr int kDesiredChunkSize = 16;  // ChunkedEllpack::desiredChunkSize
constexpr int kMaxDiagonals = 128;     // Multidiagonal: diagonals one matrix may hold here
// Nonzeros per warp window of the adaptive CSR kernel: 8 per lane for FP64
// values, 12 per lane for FP32 (so one window moves ~3 KB of columns + values).
constexpr int kWinElemsF64 = 8;
constexpr int kWinElemsF32 = 12;
constexpr int kWinNnzF64 = 32 * kWinElemsF64;
constexpr int kWinNnzF32 = 32 * kWinElemsF32;
// Rows longer than this are summed by a whole warp in the adaptive kernel.
#ifndef B2S_CSR_LONG_ROW
#define B2S_CSR_LONG_ROW 48
#endif
constexpr int kCsrLongRow = B2S_CSR_LONG_ROW;
// Matrices whose every group of 32 consecutive rows holds at most this many
// nonzeros run the row-group CSR kernel.
constexpr int kCsrGroupCap = 256;

struct ChunkSlice
{
   int32_t size, chunkSize, firstSegment, pointer;
};

// Row block of the adaptive CSR kernel: rows [row_begin, row_end) whose
// nonzeros start at nnz_begin; kind 0 = stream block (many short rows),
// kind 1 = one long row split over `parts` CTAs.
struct CsrBlock
{
   int32_t row_begin, row_end;
};

}  // namespace b2s

// The matrix handle.
namespace b2s {
// Streams, events and row chunks of the pipelined host-vector SpMV: x goes up
// and y comes down in chunks, overlapped with the products of earlier chunks.
struct HostPipe
{
   int device = -1;
   cudaStream_t up = nullptr, down = nullptr, work = nullptr;
   cudaEvent_t start = nullptr, done = nullptr;
   // the whole pipeline as one graph for pinned x / y (rebuilt when they change)
   cudaGraphExec_t exec = nullptr;
   const void* gx = nullptr;
   void* gy = nullptr;
   double galpha = 0;
   std::vector< cudaEvent_t > x_ready, y_ready;  // per x chunk / per row chunk
   std::vector< int32_t > row_cut;               // row chunk c = [row_cut[c], row_cut[c+1])
   std::vector< int32_t > x_cut;                 // x chunk k = [x_cut[k], x_cut[k+1])
   std::vector< int32_t > need;                  // row chunk c reads x chunks [0, need[c]]
   ~HostPipe();
};
}  // namespace b2s

struct b2s_matrix_t
{
   int32_t format = B2S_CSR;
   int32_t dtype = B2S_F64;
   int32_t rows = 0, cols = 0;
   int64_t nnz = 0;           // stored nonzeros
   int64_t storage = 0;       // TNL getStorageSize()
   int64_t alloc_elems = 0;   // slots allocated on the device (BiEllpack: only the addressed part)
   int device = 0;

   b2s::DevBuf values, columns;
   b2s::DevBuf values32;      // optional FP32 copy (mixed precision inner solves)

   // CSR
   b2s::DevBuf offsets;
   int32_t csr_kernel = B2S_CSR_AUTO;
   int32_t tpr = 1;
   int32_t max_row = 0;
   double mean_row = 0;
   // adaptive kernel: first row of every nonzero window, one table per value
   // size ([0]: FP64 windows of kWinNnzF64, [1]: FP32 windows of kWinNnzF32)
   b2s::DevBuf csr_win[ 2 ];
   int64_t n_win[ 2 ] = { 0, 0 };
   int32_t csr_pipe = 0;      // rows short enough for the pipelined variant
   int32_t csr_group = 0;     // every 32-row group within kCsrGroupCap nonzeros
   int32_t csr_group_opt = 0; // b2s_matrix_opts::csr_row_groups as given
   int32_t symmetric = 0;     // SymmetricMatrix: the lower triangle is stored (any layout)
   int64_t cap_total = 0;     // sum of the row capacities (segments' size)

   // Ellpack
   int32_t segmentSize = 0, alignedSize = 0;
   // SlicedEllpack
   int32_t nslices = 0;
   int32_t slice_size = b2s::kSliceSize;
   b2s::DevBuf sliceOffsets, sliceSegmentSizes;
   // ChunkedEllpack
   int32_t numberOfSlices = 0;
   int32_t chunk_single = 0;  // ChunkedEllpack: every row has exactly one chunk
   b2s::DevBuf rowToChunk, rowToSlice, chunksToSeg, rowPointers, cslices;
   // BiEllpack
   int32_t virtualRows = 0;
   b2s::DevBuf rowPerm, groupPointers;
   b2s::DevBuf rankRow;       // BiEllpack: the row at each strip rank (inverse of rowPerm, -1 past the rows)
   // Multidiagonal: the diagonals' offsets (column - row), ascending; segmentSize
   // holds their count and alignedSize TNL's nonemptyRows
   b2s::DevBuf diagOffsets;

   // Jacobi diagonal (matrix dtype)
   b2s::DevBuf diagonal;
   // staging buffers of the host-vector SpMV path (grown on demand; calls on
   // the same handle from several host threads must not overlap)
   b2s::DevBuf stage_x, stage_y;
   // device-side status word: set when a bounded wait inside a kernel gave up
   b2s::DevBuf status;
   // pipelined host-vector SpMV (built on first use)
   std::unique_ptr< b2s::HostPipe > pipe;

   int64_t device_bytes() const;
};

namespace b2s {

// ---------------------------------------------------------------------------
// Device helpers
template< typename T >
__device__ __forceinline__ T
warp_sum( T v )
{
#pragma unroll
   for( int o = 16; o > 0; o >>= 1 )
      v += __shfl_xor_sync( 0xffffffffu, v, o );
   return v;
}

// Fixed-order block reduction of NR doubles; result valid in thread 0.
template< int NR, int BLOCK >
__device__ __forceinline__ void
block_sum( double ( &v )[ NR ] )
{
   static_assert( BLOCK % 32 == 0 && BLOCK <= 1024, "block size" );
   __shared__ double sh[ NR ][ BLOCK / 32 ];
   const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
   for( int k = 0; k < NR; k++ ) {
      double s = warp_sum( v[ k ] );
      if( lane == 0 )
         sh[ k ][ warp ] = s;
   }
   __syncthreads();
   if( warp == 0 ) {
#pragma unroll
      for( int k = 0; k < NR; k++ ) {
         double s = lane < BLOCK / 32 ? sh[ k ][ lane ] : 0.0;
         v[ k ] = warp_sum( s );
      }
   }
   __syncthreads();
}

// Scratch of a grid-wide reduction: per-block partials (NR * grid doubles)
// and a ticket counter that the last block resets to zero.
struct RedScratch
{
   double* partials;
   unsigned int* counter;
};

// Block-reduce `acc`, publish the block's partial sums, and let the last
// block to arrive sum all partials in block order (deterministic for a fixed
// grid). Returns true in every thread of the last block, with `total` valid
// in thread 0 of that block.
template< int NR, int BLOCK >
__device__ __forceinline__ bool
grid_reduce( double ( &acc )[ NR ], RedScratch rs, double ( &total )[ NR ] )
{
   __shared__ bool is_last;
   block_sum< NR, BLOCK >( acc );
   if( threadIdx.x == 0 ) {
#pragma unroll
      for( int k = 0; k < NR; k++ )
         rs.partials[ k * gridDim.x + blockIdx.x ] = acc[ k ];
      __threadfence();
      const unsigned int t = atomicAdd( rs.counter, 1u );
      is_last = ( t == gridDim.x - 1 );
   }
   __syncthreads();
   if( ! is_last )
      return false;
   __threadfence();
   // warp w sums the partials of values w, w + BLOCK/32, ...: each lane loads
   // its share eight at a time (independent loads), then a fixed butterfly
   __shared__ double fin[ NR ];
   const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
   const int G = (int) gridDim.x;
   for( int k = warp; k < NR; k += BLOCK / 32 ) {
      const double* pk = rs.partials + (size_t) k * G;
      double s = 0.0;
      for( int b0 = lane; b0 < G; b0 += 32 * 8 ) {
         double v[ 8 ];
#pragma unroll
         for( int u = 0; u < 8; u++ )
            v[ u ] = b0 + 32 * u < G ? __ldcg( pk + b0 + 32 * u ) : 0.0;
#pragma unroll
         for( int u = 0; u < 8; u++ )
            s += v[ u ];
      }
      s = warp_sum( s );
      if( lane == 0 )
         fin[ k ] = s;
   }
   __syncthreads();
   if( threadIdx.x == 0 ) {
#pragma unroll
      for( int k = 0; k < NR; k++ )
         total[ k ] = fin[ k ];
      *rs.counter = 0u;
   }
   return true;
}

// Largest grid used by reduction kernels (partials buffers are sized for it).
constexpr int kReduceBlock = 256;
int reduce_grid( int64_t n, int per_thread = 1 );
constexpr int kMaxReduceGrid = 148 * 16;
// Resident blocks per SM of `kernel` launched with `block` threads and no
// dynamic shared memory (occupancy calculator, cached per kernel and device).
int resident_blocks( const void* kernel, int block );

// Scratch owned by a handle: NR*kMaxReduceGrid doubles + counters.
struct Scratch
{
   DevBuf buf;
   double* partials = nullptr;
   unsigned int* counters = nullptr;
   int slots = 0;
   b2s_status init( int nslots, cudaStream_t s );
   RedScratch slot( int i ) const
   {
      return RedScratch{ partials + (size_t) i * 4 * kMaxReduceGrid, counters + i };
   }
};

// ---------------------------------------------------------------------------
// SpMV launchers (spmv.cu). `Sink` decides what happens to each row sum.
template< typename Real >
struct SpmvArgs
{
   const b2s_matrix_t* A;
   const Real* values;  // A's values in Real (may be the FP32 copy)
   const Real* x;
   int32_t row_begin, row_end;
};

// y = alpha*A*x + beta*y
template< typename Real >
b2s_status spmv_plain( const SpmvArgs< Real >& a, Real* y, Real alpha, Real beta, cudaStream_t s );

// B2S_TIMEOUT (and reset) when a bounded device wait on this matrix gave up
b2s_status device_status( b2s_matrix_t* A, cudaStream_t s );

// ---------------------------------------------------------------------------
// Matrix helpers (matrix.cu)
b2s_status build_diagonal( b2s_matrix_t* A, cudaStream_t s );
// The storage arrays of a padded layout as TNL keeps them (host side), e.g.
// read from a file. Values are in `dtype`, `alloc` of them.
// SymmetricMatrix (matrix.cu): check that a CSR matrix holds its lower
// triangle only and mark it; expand one into the general CSR matrix L + L^T - D.
b2s_status mark_symmetric( b2s_matrix_t* m, cudaStream_t s );
// BiEllpack: rankRow from rowPerm (matrix.cu)
b2s_status build_rank_row( b2s_matrix_t* m, cudaStream_t s );
b2s_status expand_symmetric( const b2s_matrix_t* m, cudaStream_t s, b2s_matrix_t** out );

struct LayoutArrays
{
   int32_t format = 0, dtype = 0, rows = 0, cols = 0;
   std::vector< unsigned char > values;  // alloc * sizeof( value )
   std::vector< int32_t > columns;
   int64_t storage = 0;  // TNL's getStorageSize()
   // Ellpack
   int32_t segmentSize = 0, alignedSize = 0;
   // SlicedEllpack
   int32_t slice_size = 32;
   int64_t size = 0;  // sum of the row capacities
   std::vector< int32_t > sliceOffsets, sliceSegmentSizes;
   // ChunkedEllpack
   int32_t numberOfSlices = 0;
   std::vector< int32_t > rowToChunk, rowToSlice, rowPointers, chunksToSeg;
   std::vector< ChunkSlice > slices;
   // BiEllpack
   int32_t virtualRows = 0;
   std::vector< int32_t > rowPerm, groupPointers;
};
// A matrix holding exactly these arrays (after checks that every index the
// kernels derive from them stays inside the storage).
b2s_status matrix_from_layout( const LayoutArrays& L, const b2s_matrix_opts& o, cudaStream_t s, b2s_matrix* out );

// A device copy of every array of `a` (TNL's copy assignment).
b2s_status clone_matrix( const b2s_matrix_t* a, b2s_matrix_t* m, cudaStream_t s );
// Rows of any layout as CSR arrays (local order; padding and, with
// drop_zeros, zero values skipped).
// Entry points that need stored values refuse binary matrices.
#define B2S_NO_BINARY( A, what )                                                                  \
   do {                                                                                           \
      if( ( A ) && ( A )->dtype == B2S_BOOL ) {                                                   \
         b2s::set_error( "%s is not provided for binary (B2S_BOOL) matrices", what );            \
         return B2S_UNSUPPORTED;                                                                  \
      }                                                                                           \
   } while( 0 )
// y += alpha A x of a SymmetricMatrix stored in a padded layout (y already scaled by beta)
b2s_status spmv_symmetric_layout( const b2s_matrix_t* A, const void* vals, const void* x, void* y, double alpha,
                                  int32_t rb, int32_t re, cudaStream_t s );
// y = alpha A x + beta y of a binary (B2S_BOOL) matrix on device vectors of type vdt
b2s_status spmv_binary( const b2s_matrix_t* A, const void* x, void* y, int vdt, double alpha, double beta, int32_t rb,
                        int32_t re, cudaStream_t s );
b2s_status layout_to_csr( const b2s_matrix_t* A, bool drop_zeros, DevBuf& off, DevBuf& col, DevBuf& val, int64_t& nnz,
                          cudaStream_t s );
// A matrix from assembled device CSR arrays (values in `dtype`), explicit row
// capacities `caps` (device, may be NULL) for the padded layouts, zeros kept.
b2s_status matrix_from_assembled( b2s_format format, b2s_dtype dtype, int32_t rows, int32_t cols, int64_t nnz,
                                  const int32_t* off, const int32_t* col, const void* val, const int32_t* caps,
                                  int64_t caps_total, const b2s_matrix_opts& o, cudaStream_t s, b2s_matrix* out );
b2s_status ensure_fp32_copy( b2s_matrix_t* A, cudaStream_t s );

// Host <-> device copies that always synchronize the stream before returning.
b2s_status copy_h2d( void* dst, const void* src, size_t bytes, cudaStream_t s );
b2s_status copy_d2h( void* dst, const void* src, size_t bytes, cudaStream_t s );

// Device-wide exclusive scan of int64 values in place (n may be large).
b2s_status scan_exclusive_i64( int64_t* data, int64_t n, cudaStream_t s );

}  // namespace b2s
