// Matrix construction, conversion and export.
//
// The padded layouts reproduce TNL's Devices::Cuda segments bit for bit:
//   Ellpack         Segments/Ellpack.hpp:69-80, EllpackView.hpp:246-253
//   SlicedEllpack   Segments/SlicedEllpack.hpp:64-101, SlicedEllpackView.hpp:108-132
//   ChunkedEllpack  Segments/ChunkedEllpack.hpp:80-241, detail/ChunkedEllpack.h:110-135
//   BiEllpack       Segments/BiEllpack.hpp:74-278, detail/BiEllpack.h:150-180
// and the element placement of SparseMatrix::operator= (Matrices/SparseMatrix.hpp:
// 1069-1110): row capacities = CSR row lengths, zero values dropped, remaining
// elements packed into consecutive local slots, padding = (column -1, value 0).
//
// Metadata are built on the device except for ChunkedEllpack, whose greedy slice
// partition is sequential and runs on the host (as TNL does for Devices::Cuda).
// BiEllpack's per-strip ordering (TNL: a host cocktail sort, stable, by
// non-increasing capacity) is a per-warp rank computation here.
#include "b2s_internal.cuh"

#include <algorithm>
#include <climits>
#include <cstring>
#include <memory>

namespace b2s {

int64_t
matrix_device_bytes( const b2s_matrix_t* m );

}  // namespace b2s

int64_t
b2s_matrix_t::device_bytes() const
{
   const b2s::DevBuf* bufs[] = { &values,      &columns,           &values32,     &offsets,    &csr_win[ 0 ],
                                 &csr_win[ 1 ], &sliceOffsets, &sliceSegmentSizes, &rowToChunk,   &rowToSlice, &chunksToSeg,
                                 &rowPointers,  &cslices,           &rowPerm,      &groupPointers, &diagonal,
                                 &rankRow,      &diagOffsets };
   int64_t t = 0;
   for( auto* b : bufs )
      t += (int64_t) b->bytes;
   return t;
}

namespace b2s {

// ---------------------------------------------------------------------------
// Element position of (row, local) in the ColumnMajor layouts.
struct LayoutView
{
   int format;
   const int32_t* offsets;
   int32_t alignedSize;
   const int32_t* sliceOffsets;
   int32_t sliceSize;
   const int32_t* rowToChunk;
   const int32_t* rowToSlice;
   const ChunkSlice* cslices;
   const int32_t* rowPerm;
   const int32_t* groupPointers;
   const int32_t* diagOffsets;  // Multidiagonal (alignedSize: nonemptyRows)
   int32_t ndiag, cols;

   // Multidiagonal: the diagonals whose column lies in [0, cols) for `row`
   // form the range [lo, hi) of the ascending offsets
   __device__ __forceinline__ void
   mdiag_range( int row, int& lo, int& hi ) const
   {
      lo = 0;
      hi = 0;
      for( int d = 0; d < ndiag; d++ ) {
         const int o = diagOffsets[ d ];
         lo += o < -row;
         hi += o < cols - row;
      }
   }

   __device__ __forceinline__ int64_t
   gidx( int row, int local ) const
   {
      switch( format ) {
         case B2S_MULTIDIAGONAL: {
            // the local-th in-range diagonal (a row's traversal skips the out-of-range ones)
            int lo, hi;
            mdiag_range( row, lo, hi );
            return row + (int64_t) alignedSize * ( lo + local );
         }
         case B2S_CSR:
            return (int64_t) offsets[ row ] + local;
         case B2S_ELLPACK:
            return row + (int64_t) alignedSize * local;
         case B2S_SLICED_ELLPACK:
            return (int64_t) sliceOffsets[ row / sliceSize ] + ( row % sliceSize ) + (int64_t) sliceSize * local;
         case B2S_CHUNKED_ELLPACK: {
            const int s = rowToSlice[ row ];
            const ChunkSlice sl = cslices[ s ];
            const int first = ( row != sl.firstSegment ) ? rowToChunk[ row - 1 ] : 0;
            return (int64_t) sl.pointer + (int64_t) ( local % sl.chunkSize ) * kChunksInSlice + first
                 + local / sl.chunkSize;
         }
         case B2S_BIELLPACK: {
            const int strip = row / kBiWarp;
            const int gb = strip * kBiGroups;
            const int p = rowPerm[ row ] - strip * kBiWarp;
            int groups = 1;
            for( int i = 0, bis = 1; i < kBiGroups; i++, bis *= 2 )
               if( p < bis ) {
                  groups = kBiGroups - i;
                  break;
               }
            int64_t g = groupPointers[ gb ];
            int h = kBiWarp;
            for( int k = 0; k < groups; k++ ) {
               const int size = groupPointers[ gb + k + 1 ] - groupPointers[ gb + k ];
               if( size ) {
                  const int w = size / h;
                  if( local >= w ) {
                     local -= w;
                     g += size;
                  }
                  else
                     return g + p + (int64_t) local * h;
               }
               h /= 2;
            }
            return -1;
         }
      }
      return -1;
   }

   // slots of `row` (its capacity in the layout; -1 for BiEllpack, which
   // ends the row through gidx() == -1)
   __device__ __forceinline__ int64_t
   capacity( int row, int32_t segmentSize ) const
   {
      switch( format ) {
         case B2S_MULTIDIAGONAL: {
            if( row >= alignedSize )
               return 0;
            int lo, hi;
            mdiag_range( row, lo, hi );
            return hi - lo;
         }
         case B2S_CSR:
            return (int64_t) offsets[ row + 1 ] - offsets[ row ];
         case B2S_ELLPACK:
            return segmentSize;
         case B2S_SLICED_ELLPACK: {
            const int s = row / sliceSize;
            return ( (int64_t) sliceOffsets[ s + 1 ] - sliceOffsets[ s ] ) / sliceSize;
         }
         case B2S_CHUNKED_ELLPACK: {
            const int s = rowToSlice[ row ];
            const ChunkSlice sl = cslices[ s ];
            const int first = ( row != sl.firstSegment ) ? rowToChunk[ row - 1 ] : 0;
            return (int64_t) ( rowToChunk[ row ] - first ) * sl.chunkSize;
         }
      }
      return INT32_MAX;
   }
};

static LayoutView
view_of( const b2s_matrix_t* m )
{
   LayoutView L{};
   L.format = m->format;
   L.offsets = m->offsets.as< int32_t >();
   L.alignedSize = m->alignedSize;
   L.sliceOffsets = m->sliceOffsets.as< int32_t >();
   L.sliceSize = m->slice_size;
   L.rowToChunk = m->rowToChunk.as< int32_t >();
   L.rowToSlice = m->rowToSlice.as< int32_t >();
   L.cslices = m->cslices.as< ChunkSlice >();
   L.rowPerm = m->rowPerm.as< int32_t >();
   L.groupPointers = m->groupPointers.as< int32_t >();
   L.diagOffsets = m->diagOffsets.as< int32_t >();
   L.ndiag = m->format == B2S_MULTIDIAGONAL ? m->segmentSize : 0;
   L.cols = m->cols;
   return L;
}

// diag[r] = A_rr found through the layout (0 when the row has none):
// Preconditioners::Diagonal::update (Diagonal.hpp:24-36)
template< typename Real >
__global__ void
layout_diag_kernel( LayoutView L, int32_t rows, int32_t segmentSize, const int32_t* __restrict__ col,
                    const Real* __restrict__ val, Real* diag )
{
   for( int64_t r = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; r < rows; r += (int64_t) gridDim.x * blockDim.x ) {
      Real d = 0;
      const int64_t cap = L.capacity( (int) r, segmentSize );
      for( int64_t k = 0; k < cap; k++ ) {
         const int64_t g = L.gidx( (int) r, (int) k );
         if( g < 0 )
            break;
         const int c = col[ g ];
         if( c == -1 )
            break;
         if( c == r ) {
            d = val[ g ];
            break;
         }
      }
      diag[ r ] = d;
   }
}

// Row r's stored elements in local order, skipping padding (column -1) and,
// with drop_zeros, zero values: counts[r] (pass 1) or the CSR arrays (pass 2).
template< typename Real, bool WRITE >
__global__ void
layout_rows_kernel( LayoutView L, int32_t rows, int32_t segmentSize, const int32_t* __restrict__ col,
                    const Real* __restrict__ val, bool drop_zeros, int64_t* __restrict__ counts,
                    int32_t* __restrict__ out_col, Real* __restrict__ out_val )
{
   for( int64_t r = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; r < rows; r += (int64_t) gridDim.x * blockDim.x ) {
      const int64_t cap = L.capacity( (int) r, segmentSize );
      int64_t o = WRITE ? counts[ r ] : 0;
      for( int64_t k = 0; k < cap; k++ ) {
         const int64_t g = L.gidx( (int) r, (int) k );
         if( g < 0 )
            break;
         const int c = col[ g ];
         const Real v = val[ g ];
         if( c == -1 || ( drop_zeros && v == Real( 0 ) ) )
            continue;
         if( WRITE ) {
            out_col[ o ] = c;
            out_val[ o ] = v;
         }
         o++;
      }
      if( ! WRITE )
         counts[ r ] = o;
   }
}

// ---------------------------------------------------------------------------
// Kernels used during construction
template< typename Tin, typename Tout >
__global__ void
cast_kernel( const Tin* __restrict__ in, Tout* __restrict__ out, int64_t n )
{
   for( int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x )
      out[ i ] = (Tout) in[ i ];
}

__global__ void
row_stats_kernel( const int32_t* __restrict__ off, int32_t rows, int32_t* caps, int* max_len, int* bad, int* max_group )
{
   int mx = 0, mg = 0;
   for( int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < rows; i += (int64_t) gridDim.x * blockDim.x ) {
      const int c = off[ i + 1 ] - off[ i ];
      if( c < 0 )
         atomicExch( bad, 1 );
      if( caps )
         caps[ i ] = c;
      mx = max( mx, c );
      if( i % 32 == 0 )  // nonzeros of the 32-row group starting here
         mg = max( mg, off[ i + 32 < rows ? i + 32 : rows ] - off[ i ] );
   }
#pragma unroll
   for( int o = 16; o > 0; o >>= 1 ) {
      mx = max( mx, __shfl_xor_sync( 0xffffffffu, mx, o ) );
      mg = max( mg, __shfl_xor_sync( 0xffffffffu, mg, o ) );
   }
   if( ( threadIdx.x & 31 ) == 0 ) {
      atomicMax( max_len, mx );
      atomicMax( max_group, mg );
   }
}

template< typename Real >
__global__ void
columns_check_kernel( const int32_t* __restrict__ col, int64_t nnz, int32_t ncols, int* bad )
{
   for( int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < nnz; i += (int64_t) gridDim.x * blockDim.x ) {
      const int c = col[ i ];
      if( c < -1 || c >= ncols )
         atomicExch( bad, 2 );
      else if( c == -1 )
         atomicCAS( bad, 0, 3 );  // padding slot: valid input for the padded layouts only
   }
}

// SlicedEllpack: slice width = max capacity in the slice (SlicedEllpack.hpp:75-97)
__global__ void
sliced_meta_kernel( const int32_t* __restrict__ caps, int32_t rows, int32_t nslices, int32_t S, int32_t* sliceSegmentSizes,
                    int64_t* slice_slots )
{
   for( int64_t s = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; s <= nslices; s += (int64_t) gridDim.x * blockDim.x ) {
      if( s == nslices ) {
         slice_slots[ s ] = 0;
         continue;
      }
      int w = 0;
      for( int k = 0; k < S; k++ ) {
         const int64_t r = s * S + k;
         if( r < rows )
            w = max( w, caps[ r ] );
      }
      sliceSegmentSizes[ s ] = w;
      slice_slots[ s ] = (int64_t) w * S;
   }
}

// BiEllpack: one warp per strip of 32 rows. The rank of a row inside its strip
// is the number of rows with a larger capacity plus the number of earlier rows
// with the same capacity — exactly the order of a stable sort by
// non-increasing capacity (BiEllpack.hpp:74-131). Group g of the strip gets
// height 32>>g and width cap(rank 2^(4-g)-1) - cap(rank 2^(5-g)-1)
// (BiEllpack.hpp:134-170); the last strip leaves the groups it cannot fill empty.
__global__ void
biell_meta_kernel( const int32_t* __restrict__ caps, int32_t rows, int32_t strips, int32_t* rowPerm,
                   int64_t* group_sizes )
{
   const int lane = threadIdx.x & 31;
   const int64_t warp_global = ( blockIdx.x * (int64_t) blockDim.x + threadIdx.x ) >> 5;
   const int64_t nwarps = ( (int64_t) gridDim.x * blockDim.x ) >> 5;
   for( int64_t st = warp_global; st <= strips; st += nwarps ) {
      if( st == strips ) {
         if( lane == 0 )
            group_sizes[ (int64_t) strips * kBiGroups ] = 0;
         continue;
      }
      const int64_t begin = st * kBiWarp;
      const int cnt = (int) min( (int64_t) kBiWarp, (int64_t) rows - begin );
      const int my = lane < cnt ? caps[ begin + lane ] : -1;
      int rank = 0;
      for( int j = 0; j < cnt; j++ ) {
         const int o = __shfl_sync( 0xffffffffu, my, j );
         if( lane < cnt && ( o > my || ( o == my && j < lane ) ) )
            rank++;
      }
      if( lane < cnt )
         rowPerm[ begin + lane ] = (int32_t) ( begin + rank );
      // capacity at each rank: lane holding rank r publishes its capacity
      __shared__ int sorted[ 8 ][ kBiWarp ];
      const int wib = threadIdx.x >> 5;
      if( lane < cnt )
         sorted[ wib ][ rank ] = my;
      __syncwarp();
      if( lane == 0 ) {
         int empty = 0;
         if( st == strips - 1 )
            while( cnt <= ( 1 << ( kBiLogWarp - 1 - empty ) ) - 1 )
               empty++;
         int64_t* gs = group_sizes + st * kBiGroups;
         for( int g = 0; g < kBiGroups; g++ )
            gs[ g ] = 0;
         int allocated = 0;
         for( int g = empty; g < kBiLogWarp; g++ ) {
            const int len = sorted[ wib ][ ( 1 << ( kBiLogWarp - 1 - g ) ) - 1 ];
            gs[ g ] = (int64_t) ( len - allocated ) * ( 1 << ( kBiLogWarp - g ) );
            allocated = len;
         }
      }
      __syncwarp();
   }
}

__global__ void
i64_to_i32_copy_kernel( const int64_t* __restrict__ in, int32_t* __restrict__ out, int64_t n )
{
   for( int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x )
      out[ i ] = (int32_t) in[ i ];
}

__global__ void
fill_padding_kernel( int32_t* cols, int64_t n )
{
   for( int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x )
      cols[ i ] = -1;
}

// One warp per row: nonzero elements are packed into consecutive local slots
// (ballot + popcount give each element its local index).
template< typename Real, typename Tin >
__global__ void
fill_kernel( LayoutView L, int32_t rows, const int32_t* __restrict__ off, const int32_t* __restrict__ col,
             const Tin* __restrict__ val, Real* __restrict__ out_val, int32_t* __restrict__ out_col, bool keep_zeros )
{
   const int lane = threadIdx.x & 31;
   const int64_t warp_global = ( blockIdx.x * (int64_t) blockDim.x + threadIdx.x ) >> 5;
   const int64_t nwarps = ( (int64_t) gridDim.x * blockDim.x ) >> 5;
   for( int64_t r = warp_global; r < rows; r += nwarps ) {
      const int b = off[ r ], e = off[ r + 1 ];
      int local = 0;
      for( int k0 = b; k0 < e; k0 += 32 ) {
         const int k = k0 + lane;
         Real v = 0;
         int c = -1;
         if( k < e ) {
            v = (Real) val[ k ];
            c = col[ k ];
         }
         const bool keep = ( k < e ) && ( keep_zeros || v != Real( 0 ) ) && c != -1;
         const unsigned m = __ballot_sync( 0xffffffffu, keep );
         if( keep ) {
            const int li = local + __popc( m & ( ( 1u << lane ) - 1u ) );
            const int64_t g = L.gidx( (int) r, li );
            out_col[ g ] = c;
            out_val[ g ] = v;
         }
         local += __popc( m );
      }
   }
}

// diagonal[i] = A(i,i) (0 when absent) — Preconditioners/Diagonal.hpp:20-40
template< typename Real, typename Tin >
__global__ void
diag_kernel( int32_t rows, const int32_t* __restrict__ off, const int32_t* __restrict__ col,
             const Tin* __restrict__ val, Real* __restrict__ diag )
{
   for( int64_t r = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; r < rows; r += (int64_t) gridDim.x * blockDim.x ) {
      Real d = 0;
      for( int k = off[ r ]; k < off[ r + 1 ]; k++ )
         if( col[ k ] == r ) {
            d = (Real) val[ k ];
            break;
         }
      diag[ r ] = d;
   }
}

// win_rows[t] = first row whose first nonzero is at or after t*win
// (the adaptive CSR kernel's nnz-balanced warp windows); win_rows[nwin] = rows
__global__ void
csr_window_table_kernel( const int32_t* __restrict__ off, int32_t rows, int64_t ntiles, int win, int32_t* tile_rows )
{
   for( int64_t t = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; t <= ntiles; t += (int64_t) gridDim.x * blockDim.x ) {
      const int64_t target = t * (int64_t) win;
      int lo = 0, hi = rows;  // lower_bound over off[0, rows)
      while( lo < hi ) {
         const int mid = lo + ( hi - lo ) / 2;
         if( (int64_t) off[ mid ] < target )
            lo = mid + 1;
         else
            hi = mid;
      }
      tile_rows[ t ] = t == ntiles ? rows : lo;
   }
}

static int
grid_for( int64_t n, int threads = 256 )
{
   const int64_t g = ( n + threads - 1 ) / threads;
   return (int) std::max< int64_t >( 1, std::min< int64_t >( g, (int64_t) num_sms() * 32 ) );
}

static size_t
dsize( int dtype )
{
   return dtype == B2S_F64 ? 8 : 4;
}

// Host-side ChunkedEllpack layout (ChunkedEllpack.hpp:80-241).
struct ChunkedHost
{
   std::vector< int32_t > rowToChunk, rowToSlice, rowPointers, chunksToSeg;
   std::vector< ChunkSlice > slices;
   int64_t storage = 0;
};

static b2s_status
build_chunked_host( const std::vector< int32_t >& caps, ChunkedHost& H )
{
   const int n = (int) caps.size();
   H.rowToChunk.assign( n, 0 );
   H.rowToSlice.assign( n, 0 );
   H.rowPointers.assign( (size_t) n + 1, 0 );
   H.slices.clear();
   const int desired = kChunksInSlice * kDesiredChunkSize;
   // greedy slices: add rows until the slice holds `desired` elements or 256 rows
   {
      int seg = 0, size = 0, alloc = 0;
      while( seg < n ) {
         alloc += caps[ seg ];
         size++;
         seg++;
         if( alloc < desired && seg < n && size < kChunksInSlice )
            continue;
         H.slices.push_back( ChunkSlice{ size, 0, seg - size, alloc } );
         size = 0;
         alloc = 0;
      }
   }
   int64_t storage = 0;
   for( size_t s = 0; s < H.slices.size(); s++ ) {
      ChunkSlice& sl = H.slices[ s ];
      const int begin = sl.firstSegment, end = begin + sl.size, inSlice = sl.pointer;
      int freeChunks = kChunksInSlice - sl.size;
      int maxLen = caps[ begin ];
      int added_total = 0;
      for( int i = begin; i < end; i++ ) {
         // a share of the free chunks proportional to the row's length, truncated
         const double share = inSlice != 0 ? (double) caps[ i ] / (double) inSlice : 0.0;
         const int add = (int) ( (double) freeChunks * share );
         H.rowToChunk[ i ] = 1 + add;
         added_total += add;
         maxLen = std::max( maxLen, caps[ i ] );
      }
      freeChunks -= added_total;
      // leftovers go round-robin to the rows of maximal length
      while( freeChunks > 0 )
         for( int i = begin; i < end && freeChunks > 0; i++ )
            if( caps[ i ] == maxLen ) {
               H.rowToChunk[ i ]++;
               freeChunks--;
            }
      int chunkSize = 0;
      for( int i = begin; i < end; i++ ) {
         const int c = caps[ i ] / H.rowToChunk[ i ] + ( caps[ i ] % H.rowToChunk[ i ] != 0 );
         chunkSize = std::max( chunkSize, c );
      }
      sl.chunkSize = chunkSize;
      if( storage > INT32_MAX ) {
         set_error( "ChunkedEllpack storage exceeds 32-bit indices" );
         return B2S_INDEX_OVERFLOW;
      }
      sl.pointer = (int32_t) storage;
      storage += (int64_t) kChunksInSlice * chunkSize;
      for( int i = begin; i < end; i++ ) {
         H.rowToSlice[ i ] = (int32_t) s;
         H.rowPointers[ i + 1 ] = chunkSize * H.rowToChunk[ i ];
      }
      for( int j = begin + 1; j < end; j++ )
         H.rowToChunk[ j ] += H.rowToChunk[ j - 1 ];
   }
   int64_t run = 0;
   for( int i = 1; i <= n; i++ ) {
      run += H.rowPointers[ i ];
      H.rowPointers[ i ] = (int32_t) run;
   }
   H.chunksToSeg.assign( H.slices.size() * kChunksInSlice, 0 );
   size_t ci = 0;
   for( int r = 0; r < n; r++ ) {
      const ChunkSlice& sl = H.slices[ H.rowToSlice[ r ] ];
      const int first = ( r != sl.firstSegment ) ? H.rowToChunk[ r - 1 ] : 0;
      for( int k = first; k < H.rowToChunk[ r ]; k++ )
         H.chunksToSeg[ ci++ ] = r;
   }
   if( storage > INT32_MAX ) {
      set_error( "ChunkedEllpack storage exceeds 32-bit indices" );
      return B2S_INDEX_OVERFLOW;
   }
   H.storage = storage;
   return B2S_OK;
}

template< typename T >
static b2s_status
upload( DevBuf& dst, const std::vector< T >& src, cudaStream_t s )
{
   B2S_TRY( dst.alloc( src.size() * sizeof( T ) ) );
   return copy_h2d( dst.p, src.data(), src.size() * sizeof( T ), s );
}

// Threads-per-row of the CSR vector kernel from the mean row length.
static int
choose_tpr( double mean )
{
   int t = 1;
   while( t < 32 && t < mean )
      t *= 2;
   return t;
}

__global__ void
max_kernel( const int32_t* __restrict__ v, int32_t n, int* out )
{
   int mx = 0;
   for( int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x )
      mx = max( mx, v[ i ] );
#pragma unroll
   for( int o = 16; o > 0; o >>= 1 )
      mx = max( mx, __shfl_xor_sync( 0xffffffffu, mx, o ) );
   if( ( threadIdx.x & 31 ) == 0 )
      atomicMax( out, mx );
}

// Build `m` (format/dtype already set) from CSR arrays in device memory.
// Padded layouts take their row capacities from the CSR row lengths and drop
// explicit zeros (SparseMatrix::operator=), unless `caps_in` (device, >= the
// row lengths) gives the capacities and `keep_zeros` keeps the zeros
// (setRowCapacities + setElement, as MatrixReader assembles a matrix).
// every row of a ChunkedEllpack layout has exactly one chunk (rowToChunk holds
// the slice-local end of each row's chunks)
static int32_t
chunked_single( const std::vector< int32_t >& rowToChunk, const std::vector< int32_t >& rowToSlice,
                const std::vector< ChunkSlice >& slices )
{
   for( size_t r = 0; r < rowToChunk.size(); r++ ) {
      const ChunkSlice& c = slices[ rowToSlice[ r ] ];
      const int32_t first = (int32_t) r != c.firstSegment ? rowToChunk[ r - 1 ] : 0;
      if( rowToChunk[ r ] - first != 1 )
         return 0;
   }
   return 1;
}

// Multidiagonal: mark[ column - row + rows - 1 ] for every element
__global__ void
mdiag_mark_kernel( const int32_t* __restrict__ off, const int32_t* __restrict__ col, int32_t rows, int32_t* mark )
{
   for( int64_t r = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; r < rows; r += (int64_t) gridDim.x * blockDim.x )
      for( int k = off[ r ]; k < off[ r + 1 ]; k++ )
         if( col[ k ] >= 0 )
            mark[ col[ k ] - r + rows - 1 ] = 1;
}

// values[ d * ne + r ] = A( r, r + offsets[ d ] ), one thread per row in
// element order (a repeated column: the last one); columns[ d * ne + r ] =
// r + offsets[ d ] inside [0, cols), else -1
template< typename Real, typename Tin >
__global__ void
mdiag_fill_kernel( const int32_t* __restrict__ off, const int32_t* __restrict__ col, const Tin* __restrict__ val,
                   int32_t rows, int32_t cols, int32_t ne, const int32_t* __restrict__ map,
                   const int32_t* __restrict__ doff, int32_t ndiag, Real* values, int32_t* columns )
{
   for( int64_t r = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; r < ne; r += (int64_t) gridDim.x * blockDim.x ) {
      for( int d = 0; d < ndiag; d++ ) {
         const int64_t c = r + doff[ d ];
         columns[ (int64_t) d * ne + r ] = ( c >= 0 && c < cols ) ? (int32_t) c : -1;
      }
      if( r < rows )
         for( int k = off[ r ]; k < off[ r + 1 ]; k++ )
            if( col[ k ] >= 0 )
               values[ (int64_t) map[ col[ k ] - r + rows - 1 ] * ne + r ] = (Real) val[ k ];
   }
}

// MultidiagonalMatrix( rows, cols, offsets ) holding the CSR pattern's
// elements: the offsets are the pattern's distinct (column - row), ascending
// (MultidiagonalMatrix.hpp:121-140 for nonemptyRows)
template< typename Tin >
static b2s_status
build_multidiagonal( b2s_matrix_t* m, const int32_t* off, const int32_t* col, const Tin* val, int64_t nnz,
                     cudaStream_t s )
{
   const int32_t rows = m->rows, cols = m->cols;
   const int64_t span = std::max< int64_t >( (int64_t) rows + cols - 1, 1 );
   DevBuf mark;
   B2S_TRY( mark.alloc( (size_t) span * sizeof( int32_t ) ) );
   B2S_TRY_CUDA( cudaMemsetAsync( mark.p, 0, (size_t) span * sizeof( int32_t ), s ) );
   if( rows > 0 && nnz > 0 ) {
      mdiag_mark_kernel<<< grid_for( rows ), 256, 0, s >>>( off, col, rows, mark.as< int32_t >() );
      B2S_TRY_CUDA( cudaGetLastError() );
   }
   std::vector< int32_t > h( (size_t) span );
   B2S_TRY( copy_d2h( h.data(), mark.p, (size_t) span * sizeof( int32_t ), s ) );
   std::vector< int32_t > offsets;
   for( int64_t i = 0; i < span; i++ )
      if( h[ i ] ) {
         h[ i ] = (int32_t) offsets.size();  // the lookup from (column - row) to the diagonal
         offsets.push_back( (int32_t) ( i - ( rows - 1 ) ) );
      }
   if( offsets.size() > (size_t) kMaxDiagonals ) {
      set_error( "the pattern has %zu diagonals; a Multidiagonal matrix holds at most %d", offsets.size(),
                 kMaxDiagonals );
      return B2S_UNSUPPORTED;
   }
   const int32_t nd = (int32_t) offsets.size();
   int64_t ne = std::min( rows, cols );
   if( nd > 0 && offsets[ 0 ] < 0 )
      ne = std::min< int64_t >( rows, ne - offsets[ 0 ] );
   const int64_t storage = ne * nd;
   if( storage > INT32_MAX ) {
      set_error( "Multidiagonal storage %lld exceeds 32-bit indices", (long long) storage );
      return B2S_INDEX_OVERFLOW;
   }
   m->segmentSize = nd;
   m->alignedSize = (int32_t) ne;
   m->max_row = nd;
   m->storage = storage;
   m->alloc_elems = storage;
   m->nnz = nnz;
   const size_t es = dsize( m->dtype );
   B2S_TRY( upload( m->diagOffsets, offsets.empty() ? std::vector< int32_t >{ 0 } : offsets, s ) );
   DevBuf map;
   B2S_TRY( map.alloc( (size_t) span * sizeof( int32_t ) ) );
   B2S_TRY( copy_h2d( map.p, h.data(), (size_t) span * sizeof( int32_t ), s ) );
   B2S_TRY( m->values.alloc( (size_t) std::max< int64_t >( storage, 1 ) * es ) );
   B2S_TRY( m->columns.alloc( (size_t) std::max< int64_t >( storage, 1 ) * sizeof( int32_t ) ) );
   if( storage > 0 ) {
      B2S_TRY_CUDA( cudaMemsetAsync( m->values.p, 0, (size_t) storage * es, s ) );
      if( m->dtype == B2S_F64 )
         mdiag_fill_kernel< double, Tin ><<< grid_for( ne ), 256, 0, s >>>(
            off, col, val, rows, cols, (int32_t) ne, map.as< int32_t >(), m->diagOffsets.as< int32_t >(), nd,
            m->values.as< double >(), m->columns.as< int32_t >() );
      else
         mdiag_fill_kernel< float, Tin ><<< grid_for( ne ), 256, 0, s >>>(
            off, col, val, rows, cols, (int32_t) ne, map.as< int32_t >(), m->diagOffsets.as< int32_t >(), nd,
            m->values.as< float >(), m->columns.as< int32_t >() );
      B2S_TRY_CUDA( cudaGetLastError() );
   }
   B2S_TRY_CUDA( cudaStreamSynchronize( s ) );
   return B2S_OK;
}

template< typename Tin >
static b2s_status
build_from_device_csr( b2s_matrix_t* m, const int32_t* off, const int32_t* col, const Tin* val, int64_t nnz,
                       const b2s_matrix_opts& opts, cudaStream_t s, const int32_t* caps_in = nullptr,
                       bool keep_zeros = false, int64_t caps_total = 0 )
{
   const int32_t rows = m->rows;
   m->cap_total = caps_in ? caps_total : nnz;
   {
      const int32_t ss = opts.slice_size == 0 ? kSliceSize : opts.slice_size;
      if( ss != 8 && ss != 16 && ss != 32 && ss != 64 ) {
         set_error( "slice_size must be 0 (32), 8, 16, 32 or 64" );
         return B2S_INVALID_ARG;
      }
      m->slice_size = ss;
   }
   DevBuf caps, flags;
   B2S_TRY( caps.alloc( (size_t) std::max( rows, 1 ) * sizeof( int32_t ) ) );
   B2S_TRY( flags.alloc( 4 * sizeof( int ) ) );
   B2S_TRY_CUDA( cudaMemsetAsync( flags.p, 0, 4 * sizeof( int ), s ) );
   int* d_max = flags.as< int >();
   int* d_bad = flags.as< int >() + 1;
   if( rows > 0 ) {
      row_stats_kernel<<< grid_for( rows ), 256, 0, s >>>( off, rows, caps.as< int32_t >(), d_max, d_bad,
                                                            flags.as< int >() + 2 );
      B2S_TRY_CUDA( cudaGetLastError() );
   }
   if( nnz > 0 ) {
      columns_check_kernel< Tin ><<< grid_for( nnz ), 256, 0, s >>>( col, nnz, m->cols, d_bad );
      B2S_TRY_CUDA( cudaGetLastError() );
   }
   if( caps_in && rows > 0 && m->format != B2S_CSR ) {
      B2S_TRY_CUDA( cudaMemcpyAsync( caps.p, caps_in, (size_t) rows * sizeof( int32_t ), cudaMemcpyDeviceToDevice, s ) );
      max_kernel<<< grid_for( rows ), 256, 0, s >>>( caps_in, rows, d_max );
      B2S_TRY_CUDA( cudaGetLastError() );
   }
   int hflags[ 3 ] = { 0, 0, 0 };
   B2S_TRY( copy_d2h( hflags, flags.p, 3 * sizeof( int ), s ) );
   int32_t off_first = 0, off_last = 0;
   if( rows > 0 ) {
      B2S_TRY( copy_d2h( &off_first, off, sizeof( int32_t ), s ) );
      B2S_TRY( copy_d2h( &off_last, off + rows, sizeof( int32_t ), s ) );
   }
   if( hflags[ 1 ] == 1 || off_first != 0 || (int64_t) off_last != nnz ) {
      set_error( "CSR offsets are not a non-decreasing sequence from 0 to nnz" );
      return B2S_INVALID_ARG;
   }
   if( hflags[ 1 ] == 2 ) {
      set_error( "CSR column index outside [-1, cols)" );
      return B2S_INVALID_ARG;
   }
   m->max_row = hflags[ 0 ];
   m->mean_row = rows > 0 ? (double) nnz / rows : 0.0;
   const size_t es = dsize( m->dtype );

   B2S_TRY( m->status.alloc( 4 * sizeof( int ) ) );
   B2S_TRY_CUDA( cudaMemsetAsync( m->status.p, 0, 4 * sizeof( int ), s ) );
   // Jacobi diagonal, from the assembled CSR
   B2S_TRY( m->diagonal.alloc( (size_t) std::max( rows, 1 ) * es ) );
   if( rows > 0 ) {
      if( m->dtype == B2S_F64 )
         diag_kernel< double, Tin ><<< grid_for( rows ), 256, 0, s >>>( rows, off, col, val, m->diagonal.as< double >() );
      else
         diag_kernel< float, Tin ><<< grid_for( rows ), 256, 0, s >>>( rows, off, col, val, m->diagonal.as< float >() );
      B2S_TRY_CUDA( cudaGetLastError() );
   }

   if( m->format == B2S_CSR ) {
      m->nnz = nnz;
      m->storage = nnz;
      m->alloc_elems = nnz;
      B2S_TRY( m->offsets.alloc( ( (size_t) rows + 1 ) * sizeof( int32_t ) ) );
      B2S_TRY_CUDA( cudaMemcpyAsync( m->offsets.p, off, ( (size_t) rows + 1 ) * sizeof( int32_t ),
                                     cudaMemcpyDeviceToDevice, s ) );
      B2S_TRY( m->columns.alloc( (size_t) std::max< int64_t >( nnz, 1 ) * sizeof( int32_t ) ) );
      B2S_TRY( m->values.alloc( (size_t) std::max< int64_t >( nnz, 1 ) * es ) );
      if( nnz > 0 ) {
         B2S_TRY_CUDA( cudaMemcpyAsync( m->columns.p, col, nnz * sizeof( int32_t ), cudaMemcpyDeviceToDevice, s ) );
         if( m->dtype == B2S_F64 )
            cast_kernel< Tin, double ><<< grid_for( nnz ), 256, 0, s >>>( val, m->values.as< double >(), nnz );
         else
            cast_kernel< Tin, float ><<< grid_for( nnz ), 256, 0, s >>>( val, m->values.as< float >(), nnz );
         B2S_TRY_CUDA( cudaGetLastError() );
      }
      if( hflags[ 1 ] == 3 ) {
         set_error( "column index -1 (padding) in a CSR matrix" );
         return B2S_INVALID_ARG;
      }
      // CSR kernel selection
      m->csr_kernel = opts.csr_kernel;
      if( m->csr_kernel == B2S_CSR_AUTO )
         m->csr_kernel = B2S_CSR_ADAPTIVE;
      m->tpr = opts.threads_per_row > 0 ? opts.threads_per_row : choose_tpr( m->mean_row );
      if( m->csr_kernel == B2S_CSR_SCALAR )
         m->tpr = 1;
      if( m->tpr != 1 && m->tpr != 2 && m->tpr != 4 && m->tpr != 8 && m->tpr != 16 && m->tpr != 32 ) {
         set_error( "threads_per_row must be a power of two <= 32" );
         return B2S_INVALID_ARG;
      }
      // nnz-balanced warp windows of the adaptive kernel, for both value sizes
      // (an FP64 matrix also runs FP32 products from its FP32 copy)
      const int wins[ 2 ] = { kWinNnzF64, kWinNnzF32 };
      for( int k = 0; k < 2; k++ ) {
         m->n_win[ k ] = nnz / wins[ k ] + 1;
         B2S_TRY( m->csr_win[ k ].alloc( ( (size_t) m->n_win[ k ] + 1 ) * sizeof( int32_t ) ) );
         csr_window_table_kernel<<< grid_for( m->n_win[ k ] + 1 ), 256, 0, s >>>(
            m->offsets.as< int32_t >(), rows, m->n_win[ k ], wins[ k ], m->csr_win[ k ].as< int32_t >() );
         B2S_TRY_CUDA( cudaGetLastError() );
      }
      // rows that all fit a lane's serial loop run the pipelined variant
      m->csr_pipe = m->max_row <= kCsrLongRow ? 1 : 0;
      // short, even rows: the row-group kernel
      m->csr_group_opt = opts.csr_row_groups;
      m->csr_group = hflags[ 2 ] <= kCsrGroupCap && opts.csr_row_groups >= 0 ? 1 : 0;
      B2S_TRY_CUDA( cudaStreamSynchronize( s ) );
      return B2S_OK;
   }

   if( m->format == B2S_MULTIDIAGONAL )
      return build_multidiagonal< Tin >( m, off, col, val, nnz, s );

   LayoutView L{};
   L.format = m->format;
   int64_t storage = 0, alloc_elems = 0;
   switch( m->format ) {
      case B2S_ELLPACK: {
         m->segmentSize = m->max_row;
         m->alignedSize = (int32_t) ( ( (int64_t) rows + kEllAlign - 1 ) / kEllAlign * kEllAlign );
         storage = (int64_t) m->alignedSize * m->segmentSize;
         if( storage > INT32_MAX ) {
            set_error( "Ellpack storage %lld exceeds 32-bit indices", (long long) storage );
            return B2S_INDEX_OVERFLOW;
         }
         alloc_elems = storage;
         L.alignedSize = m->alignedSize;
         break;
      }
      case B2S_SLICED_ELLPACK: {
         const int32_t S = m->slice_size;
         const int32_t ns = (int32_t) ( ( (int64_t) rows + S - 1 ) / S );
         m->nslices = ns;
         DevBuf slots;
         B2S_TRY( slots.alloc( ( (size_t) ns + 1 ) * sizeof( int64_t ) ) );
         B2S_TRY( m->sliceSegmentSizes.alloc( (size_t) std::max( ns, 1 ) * sizeof( int32_t ) ) );
         B2S_TRY( m->sliceOffsets.alloc( ( (size_t) ns + 1 ) * sizeof( int32_t ) ) );
         sliced_meta_kernel<<< grid_for( (int64_t) ns + 1 ), 256, 0, s >>>(
            caps.as< int32_t >(), rows, ns, S, m->sliceSegmentSizes.as< int32_t >(), slots.as< int64_t >() );
         B2S_TRY_CUDA( cudaGetLastError() );
         B2S_TRY( scan_exclusive_i64( slots.as< int64_t >(), (int64_t) ns + 1, s ) );
         B2S_TRY( copy_d2h( &storage, slots.as< int64_t >() + ns, sizeof( int64_t ), s ) );
         if( storage > INT32_MAX ) {
            set_error( "SlicedEllpack storage %lld exceeds 32-bit indices", (long long) storage );
            return B2S_INDEX_OVERFLOW;
         }
         i64_to_i32_copy_kernel<<< grid_for( (int64_t) ns + 1 ), 256, 0, s >>>( slots.as< int64_t >(),
                                                                               m->sliceOffsets.as< int32_t >(), ns + 1 );
         B2S_TRY_CUDA( cudaGetLastError() );
         B2S_TRY_CUDA( cudaStreamSynchronize( s ) );
         alloc_elems = storage;
         L.sliceOffsets = m->sliceOffsets.as< int32_t >();
         L.sliceSize = S;
         break;
      }
      case B2S_CHUNKED_ELLPACK: {
         std::vector< int32_t > hcaps( rows );
         if( rows > 0 )
            B2S_TRY( copy_d2h( hcaps.data(), caps.p, (size_t) rows * sizeof( int32_t ), s ) );
         ChunkedHost H;
         B2S_TRY( build_chunked_host( hcaps, H ) );
         m->numberOfSlices = (int32_t) H.slices.size();
         m->chunk_single = chunked_single( H.rowToChunk, H.rowToSlice, H.slices );
         B2S_TRY( upload( m->rowToChunk, H.rowToChunk, s ) );
         B2S_TRY( upload( m->rowToSlice, H.rowToSlice, s ) );
         B2S_TRY( upload( m->rowPointers, H.rowPointers, s ) );
         B2S_TRY( upload( m->chunksToSeg, H.chunksToSeg, s ) );
         B2S_TRY( upload( m->cslices, H.slices, s ) );
         storage = alloc_elems = H.storage;
         L.rowToChunk = m->rowToChunk.as< int32_t >();
         L.rowToSlice = m->rowToSlice.as< int32_t >();
         L.cslices = m->cslices.as< ChunkSlice >();
         break;
      }
      case B2S_BIELLPACK: {
         m->virtualRows = ( rows % kBiWarp ) ? rows + kBiWarp - ( rows % kBiWarp ) : rows;
         const int32_t strips = m->virtualRows / kBiWarp;
         const int64_t ng = (int64_t) strips * kBiGroups + 1;
         DevBuf gsz;
         B2S_TRY( gsz.alloc( ng * sizeof( int64_t ) ) );
         B2S_TRY( m->rowPerm.alloc( (size_t) std::max( rows, 1 ) * sizeof( int32_t ) ) );
         B2S_TRY( m->groupPointers.alloc( ng * sizeof( int32_t ) ) );
         biell_meta_kernel<<< grid_for( ( (int64_t) strips + 1 ) * 32 ), 256, 0, s >>>(
            caps.as< int32_t >(), rows, strips, m->rowPerm.as< int32_t >(), gsz.as< int64_t >() );
         B2S_TRY_CUDA( cudaGetLastError() );
         B2S_TRY( scan_exclusive_i64( gsz.as< int64_t >(), ng, s ) );
         int64_t total = 0;
         B2S_TRY( copy_d2h( &total, gsz.as< int64_t >() + ng - 1, sizeof( int64_t ), s ) );
         if( total > INT32_MAX ) {
            set_error( "BiEllpack group pointers exceed 32-bit indices" );
            return B2S_INDEX_OVERFLOW;
         }
         i64_to_i32_copy_kernel<<< grid_for( ng ), 256, 0, s >>>( gsz.as< int64_t >(), m->groupPointers.as< int32_t >(),
                                                                   ng );
         B2S_TRY_CUDA( cudaGetLastError() );
         B2S_TRY_CUDA( cudaStreamSynchronize( s ) );
         // TNL sizes the storage as WarpSize * groupPointers[last] (BiEllpack.hpp:261) but
         // addresses only [0, groupPointers[last]); only that part is allocated here.
         storage = (int64_t) kBiWarp * total;
         alloc_elems = total;
         L.rowPerm = m->rowPerm.as< int32_t >();
         L.groupPointers = m->groupPointers.as< int32_t >();
         B2S_TRY( build_rank_row( m, s ) );
         break;
      }
      default:
         set_error( "unknown format %d", m->format );
         return B2S_INVALID_ARG;
   }
   m->storage = storage;
   m->alloc_elems = alloc_elems;
   B2S_TRY( m->values.alloc( (size_t) std::max< int64_t >( alloc_elems, 1 ) * es ) );
   B2S_TRY( m->columns.alloc( (size_t) std::max< int64_t >( alloc_elems, 1 ) * sizeof( int32_t ) ) );
   if( alloc_elems > 0 ) {
      B2S_TRY_CUDA( cudaMemsetAsync( m->values.p, 0, alloc_elems * es, s ) );
      fill_padding_kernel<<< grid_for( alloc_elems ), 256, 0, s >>>( m->columns.as< int32_t >(), alloc_elems );
      B2S_TRY_CUDA( cudaGetLastError() );
   }
   if( rows > 0 && nnz > 0 ) {
      const int grid = grid_for( (int64_t) rows * 32 );
      if( m->dtype == B2S_F64 )
         fill_kernel< double, Tin ><<< grid, 256, 0, s >>>( L, rows, off, col, val, m->values.as< double >(),
                                                            m->columns.as< int32_t >(), keep_zeros );
      else
         fill_kernel< float, Tin ><<< grid, 256, 0, s >>>( L, rows, off, col, val, m->values.as< float >(),
                                                           m->columns.as< int32_t >(), keep_zeros );
      B2S_TRY_CUDA( cudaGetLastError() );
   }
   // count the nonzeros that survived (zeros dropped)
   m->nnz = nnz;
   B2S_TRY_CUDA( cudaStreamSynchronize( s ) );
   return B2S_OK;
}

template< typename Tin >
static b2s_status
build_any( b2s_matrix_t* m, const int32_t* off, const int32_t* col, const void* val, int64_t nnz, b2s_memory where,
           const b2s_matrix_opts& opts, cudaStream_t s )
{
   if( where == B2S_DEVICE )
      return build_from_device_csr< Tin >( m, off, col, static_cast< const Tin* >( val ), nnz, opts, s );
   DevBuf doff, dcol, dval;
   B2S_TRY( doff.alloc( ( (size_t) m->rows + 1 ) * sizeof( int32_t ) ) );
   B2S_TRY( dcol.alloc( (size_t) std::max< int64_t >( nnz, 1 ) * sizeof( int32_t ) ) );
   B2S_TRY( dval.alloc( (size_t) std::max< int64_t >( nnz, 1 ) * sizeof( Tin ) ) );
   B2S_TRY( copy_h2d( doff.p, off, ( (size_t) m->rows + 1 ) * sizeof( int32_t ), s ) );
   B2S_TRY( copy_h2d( dcol.p, col, (size_t) nnz * sizeof( int32_t ), s ) );
   B2S_TRY( copy_h2d( dval.p, val, (size_t) nnz * sizeof( Tin ), s ) );
   return build_from_device_csr< Tin >( m, doff.as< int32_t >(), dcol.as< int32_t >(), dval.as< Tin >(), nnz, opts, s );
}

b2s_status
layout_to_csr( const b2s_matrix_t* A, bool drop_zeros, DevBuf& off, DevBuf& col, DevBuf& val, int64_t& nnz,
               cudaStream_t s )
{
   const int32_t rows = A->rows;
   const size_t es = dsize( A->dtype );
   DevBuf cnt;
   B2S_TRY( cnt.alloc( ( (size_t) rows + 1 ) * sizeof( int64_t ) ) );
   B2S_TRY_CUDA( cudaMemsetAsync( cnt.p, 0, ( (size_t) rows + 1 ) * sizeof( int64_t ), s ) );
   const LayoutView L = view_of( A );
   if( rows > 0 ) {
      if( A->dtype == B2S_F64 )
         layout_rows_kernel< double, false ><<< grid_for( rows ), 256, 0, s >>>(
            L, rows, A->segmentSize, A->columns.as< int32_t >(), A->values.as< double >(), drop_zeros,
            cnt.as< int64_t >(), nullptr, nullptr );
      else
         layout_rows_kernel< float, false ><<< grid_for( rows ), 256, 0, s >>>(
            L, rows, A->segmentSize, A->columns.as< int32_t >(), A->values.as< float >(), drop_zeros,
            cnt.as< int64_t >(), nullptr, nullptr );
      B2S_TRY_CUDA( cudaGetLastError() );
   }
   B2S_TRY( scan_exclusive_i64( cnt.as< int64_t >(), (int64_t) rows + 1, s ) );
   B2S_TRY( copy_d2h( &nnz, cnt.as< int64_t >() + rows, sizeof( int64_t ), s ) );
   if( nnz > INT32_MAX ) {
      set_error( "more than 2^31 - 1 elements" );
      return B2S_INDEX_OVERFLOW;
   }
   B2S_TRY( off.alloc( ( (size_t) rows + 1 ) * sizeof( int32_t ) ) );
   B2S_TRY( col.alloc( (size_t) std::max< int64_t >( nnz, 1 ) * sizeof( int32_t ) ) );
   B2S_TRY( val.alloc( (size_t) std::max< int64_t >( nnz, 1 ) * es ) );
   i64_to_i32_copy_kernel<<< grid_for( (int64_t) rows + 1 ), 256, 0, s >>>( cnt.as< int64_t >(), off.as< int32_t >(),
                                                                            (int64_t) rows + 1 );
   B2S_TRY_CUDA( cudaGetLastError() );
   if( rows > 0 && nnz > 0 ) {
      if( A->dtype == B2S_F64 )
         layout_rows_kernel< double, true ><<< grid_for( rows ), 256, 0, s >>>(
            L, rows, A->segmentSize, A->columns.as< int32_t >(), A->values.as< double >(), drop_zeros,
            cnt.as< int64_t >(), col.as< int32_t >(), val.as< double >() );
      else
         layout_rows_kernel< float, true ><<< grid_for( rows ), 256, 0, s >>>(
            L, rows, A->segmentSize, A->columns.as< int32_t >(), A->values.as< float >(), drop_zeros,
            cnt.as< int64_t >(), col.as< int32_t >(), val.as< float >() );
      B2S_TRY_CUDA( cudaGetLastError() );
   }
   B2S_TRY_CUDA( cudaStreamSynchronize( s ) );
   return B2S_OK;
}

// ---------------------------------------------------------------------------
// Binary matrices (TNL's SparseMatrix< bool, ... >).

// beta * y + value as one fused multiply-add (one rounding), as TNL's keepers
// come out of its optimized host build (g++ -O3 -march=x86-64-v3 contracts them)
__device__ __forceinline__ double
keep_fma( double a, double b, double c )
{
   return fma( a, b, c );
}
__device__ __forceinline__ float
keep_fma( float a, float b, float c )
{
   return fmaf( a, b, c );
}

// y = alpha A x + beta y over rows [rb, re) in TNL's ComputeReal = int
// (SparseMatrixView.hpp:423-471): each stored column adds (int) x[column] to
// an int32 row sum (two's-complement wraparound); keepers chosen by the int
// multiplicators: 0: y = s, 1: y = alpha*s, 2: y = beta*y + s, 3: y = beta*y + alpha*s.
template< typename V >
__global__ void
binary_spmv_kernel( LayoutView L, int32_t rb, int32_t re, int32_t segmentSize, const int32_t* __restrict__ col,
                    const V* __restrict__ x, V* __restrict__ y, int alpha, int beta, int mode )
{
   for( int64_t r = rb + blockIdx.x * (int64_t) blockDim.x + threadIdx.x; r < re;
        r += (int64_t) gridDim.x * blockDim.x ) {
      unsigned s = 0;
      const int64_t cap = L.capacity( (int) r, segmentSize );
      for( int64_t k = 0; k < cap; k++ ) {
         const int64_t g = L.gidx( (int) r, (int) k );
         if( g < 0 )
            break;
         const int c = __ldg( col + g );
         if( c == -1 )
            continue;
         s += (unsigned) (int) __ldg( x + c );
      }
      const int si = (int) s;
      const int as = (int) ( (unsigned) alpha * s );
      switch( mode ) {
         case 0:
            y[ r ] = (V) si;
            break;
         case 1:
            y[ r ] = (V) as;
            break;
         case 2:
            y[ r ] = keep_fma( (V) beta, y[ r ], (V) si );
            break;
         default:
            y[ r ] = keep_fma( (V) beta, y[ r ], (V) as );
            break;
      }
   }
}

static int
to_int_multiplicator( double v )
{
   // a double passed for TNL's int ComputeReal is truncated toward zero
   if( ! ( v > (double) INT32_MIN - 1.0 && v < (double) INT32_MAX + 1.0 ) )
      return v > 0 ? INT32_MAX : ( v < 0 ? INT32_MIN : 0 );
   return (int) v;
}

b2s_status
spmv_binary( const b2s_matrix_t* A, const void* x, void* y, int vdt, double alpha, double beta, int32_t rb, int32_t re,
             cudaStream_t s )
{
   if( re <= rb )
      return B2S_OK;
   const int a = to_int_multiplicator( alpha ), b = to_int_multiplicator( beta );
   const int mode = b == 0 ? ( a == 1 ? 0 : 1 ) : ( a == 1 ? 2 : 3 );
   const LayoutView L = view_of( A );
   const int grid = grid_for( (int64_t) re - rb );
   if( vdt == B2S_F64 )
      binary_spmv_kernel< double ><<< grid, 256, 0, s >>>( L, rb, re, A->segmentSize, A->columns.as< int32_t >(),
                                                           static_cast< const double* >( x ), static_cast< double* >( y ),
                                                           a, b, mode );
   else
      binary_spmv_kernel< float ><<< grid, 256, 0, s >>>( L, rb, re, A->segmentSize, A->columns.as< int32_t >(),
                                                          static_cast< const float* >( x ), static_cast< float* >( y ),
                                                          a, b, mode );
   B2S_TRY_CUDA( cudaGetLastError() );
   return B2S_OK;
}

// SymmetricMatrix product over any layout (SparseMatrixView.hpp:413-476): each
// stored element (j <= i) adds v x[j] to row i's sum and, below the diagonal,
// alpha v x[i] to y[j] by an atomic addition; the row's sum goes in with
// alpha by an atomic addition too (y was scaled by beta before). Padding
// slots (column -1) are skipped.
template< typename Real >
__global__ void
layout_symmetric_kernel( LayoutView L, int32_t rb, int32_t re, int32_t segmentSize, const int32_t* __restrict__ col,
                         const Real* __restrict__ val, const Real* __restrict__ x, Real* y, Real alpha )
{
   for( int64_t r = rb + blockIdx.x * (int64_t) blockDim.x + threadIdx.x; r < re;
        r += (int64_t) gridDim.x * blockDim.x ) {
      const Real xr = x[ r ];
      Real sum = 0;
      const int64_t cap = L.capacity( (int) r, segmentSize );
      for( int64_t k = 0; k < cap; k++ ) {
         const int64_t g = L.gidx( (int) r, (int) k );
         if( g < 0 )
            break;
         const int j = col[ g ];
         if( j == -1 )
            continue;
         const Real v = val[ g ];
         if( j < r )
            atomicAdd( y + j, alpha * v * xr );
         sum += v * x[ j ];
      }
      atomicAdd( y + r, alpha * sum );
   }
}

b2s_status
spmv_symmetric_layout( const b2s_matrix_t* A, const void* vals, const void* x, void* y, double alpha, int32_t rb,
                       int32_t re, cudaStream_t s )
{
   if( re <= rb )
      return B2S_OK;
   const LayoutView L = view_of( A );
   const int grid = grid_for( (int64_t) re - rb );
   if( A->dtype == B2S_F64 )
      layout_symmetric_kernel< double ><<< grid, 256, 0, s >>>( L, rb, re, A->segmentSize, A->columns.as< int32_t >(),
                                                               static_cast< const double* >( vals ),
                                                               static_cast< const double* >( x ),
                                                               static_cast< double* >( y ), alpha );
   else
      layout_symmetric_kernel< float ><<< grid, 256, 0, s >>>( L, rb, re, A->segmentSize, A->columns.as< int32_t >(),
                                                              static_cast< const float* >( vals ),
                                                              static_cast< const float* >( x ), static_cast< float* >( y ),
                                                              (float) alpha );
   B2S_TRY_CUDA( cudaGetLastError() );
   return B2S_OK;
}

// Unit values for the entries of a binary matrix, on the device.
__global__ void
ones_kernel( float* v, int64_t n )
{
   for( int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x )
      v[ i ] = 1.0f;
}

// A binary matrix is built like a real one from the same CSR (padded layouts:
// TNL's operator= capacities, zero values dropped; CSR: rows compacted), with
// unit values where none are given, and then keeps its column indexes only.
static b2s_status
create_binary( b2s_format format, int32_t rows, int32_t cols, int64_t nnz, const int32_t* offsets,
               const int32_t* columns, const void* values, b2s_dtype values_dtype, b2s_memory where,
               const b2s_matrix_opts& o, cudaStream_t s, b2s_matrix* out )
{
   if( o.symmetric || o.keep_fp32_copy ) {
      set_error( "binary matrices are general matrices without an FP32 copy" );
      return B2S_UNSUPPORTED;
   }
   b2s_matrix_opts po = o;
   std::vector< float > host_ones;
   DevBuf dev_ones;
   const void* vals = values;
   b2s_dtype vdt = values_dtype;
   if( ! vals ) {
      vdt = B2S_F32;
      if( where == B2S_HOST ) {
         host_ones.assign( (size_t) std::max< int64_t >( nnz, 1 ), 1.0f );
         vals = host_ones.data();
      }
      else {
         B2S_TRY( dev_ones.alloc( (size_t) std::max< int64_t >( nnz, 1 ) * sizeof( float ) ) );
         ones_kernel<<< grid_for( std::max< int64_t >( nnz, 1 ) ), 256, 0, s >>>( dev_ones.as< float >(),
                                                                                  std::max< int64_t >( nnz, 1 ) );
         B2S_TRY_CUDA( cudaGetLastError() );
         vals = dev_ones.p;
      }
   }
   // the layout in the values' own type (a tiny FP64 value stays nonzero)
   const b2s_dtype build = vdt == B2S_F64 ? B2S_F64 : B2S_F32;
   b2s_matrix m = nullptr;
   if( format == B2S_CSR ) {
      b2s_matrix t = nullptr;
      B2S_TRY( b2s_matrix_create( B2S_CSR, build, rows, cols, nnz, offsets, columns, vals, vdt, where, &po, s, &t ) );
      std::unique_ptr< b2s_matrix_t > tmp( t );
      DevBuf off, col, val;
      int64_t kept = 0;
      B2S_TRY( layout_to_csr( tmp.get(), true, off, col, val, kept, s ) );
      tmp.reset();
      B2S_TRY( b2s_matrix_create( B2S_CSR, build, rows, cols, kept, off.as< int32_t >(), col.as< int32_t >(), val.p,
                                  build, B2S_DEVICE, &po, s, &m ) );
   }
   else
      B2S_TRY( b2s_matrix_create( format, build, rows, cols, nnz, offsets, columns, vals, vdt, where, &po, s, &m ) );
   m->values.release();
   m->values32.release();
   m->diagonal.release();
   m->dtype = B2S_BOOL;
   *out = m;
   return B2S_OK;
}

static b2s_status
dup_buf( b2s::DevBuf& dst, const b2s::DevBuf& src, cudaStream_t s )
{
   if( ! src.p )
      return B2S_OK;
   B2S_TRY( dst.alloc( src.bytes ) );
   B2S_TRY_CUDA( cudaMemcpyAsync( dst.p, src.p, src.bytes, cudaMemcpyDeviceToDevice, s ) );
   return B2S_OK;
}

b2s_status
clone_matrix( const b2s_matrix_t* a, b2s_matrix_t* m, cudaStream_t s )
{
   m->format = a->format;
   m->dtype = a->dtype;
   m->rows = a->rows;
   m->cols = a->cols;
   m->nnz = a->nnz;
   m->storage = a->storage;
   m->alloc_elems = a->alloc_elems;
   m->device = current_device();
   m->csr_kernel = a->csr_kernel;
   m->tpr = a->tpr;
   m->max_row = a->max_row;
   m->mean_row = a->mean_row;
   m->n_win[ 0 ] = a->n_win[ 0 ];
   m->n_win[ 1 ] = a->n_win[ 1 ];
   m->csr_pipe = a->csr_pipe;
   m->csr_group = a->csr_group;
   m->csr_group_opt = a->csr_group_opt;
   m->symmetric = a->symmetric;
   m->chunk_single = a->chunk_single;
   m->cap_total = a->cap_total;
   m->segmentSize = a->segmentSize;
   m->alignedSize = a->alignedSize;
   m->nslices = a->nslices;
   m->slice_size = a->slice_size;
   m->numberOfSlices = a->numberOfSlices;
   m->virtualRows = a->virtualRows;
   const b2s::DevBuf* from[] = { &a->values,        &a->columns,      &a->values32,    &a->offsets,
                                 &a->csr_win[ 0 ],  &a->csr_win[ 1 ], &a->sliceOffsets, &a->sliceSegmentSizes,
                                 &a->rowToChunk,    &a->rowToSlice,   &a->chunksToSeg, &a->rowPointers,
                                 &a->cslices,       &a->rowPerm,      &a->groupPointers, &a->diagonal,
                                 &a->rankRow };
   b2s::DevBuf* to[] = { &m->values,        &m->columns,      &m->values32,    &m->offsets,
                         &m->csr_win[ 0 ],  &m->csr_win[ 1 ], &m->sliceOffsets, &m->sliceSegmentSizes,
                         &m->rowToChunk,    &m->rowToSlice,   &m->chunksToSeg, &m->rowPointers,
                         &m->cslices,       &m->rowPerm,      &m->groupPointers, &m->diagonal,
                         &m->rankRow };
   for( size_t i = 0; i < sizeof( from ) / sizeof( from[ 0 ] ); i++ )
      B2S_TRY( dup_buf( *to[ i ], *from[ i ], s ) );
   B2S_TRY( m->status.alloc( 4 * sizeof( int ) ) );
   B2S_TRY_CUDA( cudaMemsetAsync( m->status.p, 0, 4 * sizeof( int ), s ) );
   B2S_TRY_CUDA( cudaStreamSynchronize( s ) );
   return B2S_OK;
}

static b2s_status
bad_layout( const char* what )
{
   set_error( "inconsistent layout arrays: %s", what );
   return B2S_INVALID_ARG;
}

b2s_status
matrix_from_layout( const LayoutArrays& L, const b2s_matrix_opts& o, cudaStream_t s, b2s_matrix* out )
{
   const int32_t rows = L.rows, cols = L.cols;
   if( rows < 0 || cols < 0 )
      return bad_layout( "negative dimensions" );
   const size_t es = L.dtype == B2S_F64 ? 8 : 4;
   const int64_t have = (int64_t) L.columns.size();
   if( (int64_t) L.values.size() != have * (int64_t) es )
      return bad_layout( "values and columnIndexes differ in length" );
   for( int32_t c : L.columns )
      if( c < -1 || c >= cols )
         return bad_layout( "column index outside [-1, columns)" );
   std::unique_ptr< b2s_matrix_t > m( new b2s_matrix_t() );
   m->format = L.format;
   m->dtype = L.dtype;
   m->rows = rows;
   m->cols = cols;
   m->device = current_device();
   m->storage = L.storage;
   int64_t alloc = 0;  // slots the kernels may address
   switch( L.format ) {
      case B2S_ELLPACK: {
         if( L.segmentSize < 0 || L.alignedSize < rows || (int64_t) L.alignedSize * L.segmentSize > have )
            return bad_layout( "Ellpack sizes" );
         m->segmentSize = L.segmentSize;
         m->alignedSize = L.alignedSize;
         m->max_row = L.segmentSize;
         alloc = (int64_t) L.alignedSize * L.segmentSize;
         m->cap_total = rows;
         break;
      }
      case B2S_SLICED_ELLPACK: {
         const int32_t S = L.slice_size;
         if( S != 8 && S != 16 && S != 32 && S != 64 )
            return bad_layout( "slice size" );
         const int32_t ns = (int32_t) ( ( (int64_t) rows + S - 1 ) / S );
         if( (int32_t) L.sliceOffsets.size() != ns + 1 || (int32_t) L.sliceSegmentSizes.size() != ns ||
             ( ns >= 0 && L.sliceOffsets[ 0 ] != 0 ) )
            return bad_layout( "SlicedEllpack slice arrays (is the slice size right?)" );
         int32_t mx = 0;
         for( int32_t k = 0; k < ns; k++ ) {
            if( L.sliceSegmentSizes[ k ] < 0 ||
                (int64_t) L.sliceOffsets[ k + 1 ] - L.sliceOffsets[ k ] != (int64_t) S * L.sliceSegmentSizes[ k ] )
               return bad_layout( "SlicedEllpack slice offsets" );
            mx = std::max( mx, L.sliceSegmentSizes[ k ] );
         }
         if( L.sliceOffsets[ ns ] > have )
            return bad_layout( "SlicedEllpack storage" );
         m->slice_size = S;
         m->nslices = ns;
         m->max_row = mx;
         m->cap_total = L.size;
         alloc = L.sliceOffsets[ ns ];
         B2S_TRY( upload( m->sliceOffsets, L.sliceOffsets, s ) );
         B2S_TRY( upload( m->sliceSegmentSizes, L.sliceSegmentSizes, s ) );
         break;
      }
      case B2S_CHUNKED_ELLPACK: {
         const int32_t nsl = L.numberOfSlices;
         if( nsl < 0 || (int64_t) L.slices.size() < nsl || (int32_t) L.rowToChunk.size() != rows ||
             (int32_t) L.rowToSlice.size() != rows || (int32_t) L.rowPointers.size() != rows + 1 ||
             (int64_t) L.chunksToSeg.size() != (int64_t) nsl * kChunksInSlice )
            return bad_layout( "ChunkedEllpack array sizes" );
         if( L.storage > have )
            return bad_layout( "ChunkedEllpack storage" );
         for( int32_t k = 0; k < nsl; k++ ) {
            const ChunkSlice& c = L.slices[ k ];
            if( c.size < 0 || c.chunkSize < 0 || c.firstSegment < 0 || (int64_t) c.firstSegment + c.size > rows ||
                c.pointer < 0 || (int64_t) c.pointer + (int64_t) c.chunkSize * kChunksInSlice > L.storage )
               return bad_layout( "ChunkedEllpack slice" );
         }
         int32_t mx = 0;
         for( int32_t r = 0; r < rows; r++ ) {
            const int32_t k = L.rowToSlice[ r ];
            if( k < 0 || k >= nsl )
               return bad_layout( "ChunkedEllpack row to slice" );
            const ChunkSlice& c = L.slices[ k ];
            if( r < c.firstSegment || r >= c.firstSegment + c.size )
               return bad_layout( "ChunkedEllpack row outside its slice" );
            const int32_t first = r != c.firstSegment ? L.rowToChunk[ r - 1 ] : 0;
            if( first < 0 || L.rowToChunk[ r ] < first || L.rowToChunk[ r ] > kChunksInSlice )
               return bad_layout( "ChunkedEllpack row to chunk" );
            mx = std::max( mx, ( L.rowToChunk[ r ] - first ) * c.chunkSize );
         }
         m->numberOfSlices = nsl;
         m->max_row = mx;
         alloc = L.storage;
         B2S_TRY( upload( m->rowToChunk, L.rowToChunk, s ) );
         B2S_TRY( upload( m->rowToSlice, L.rowToSlice, s ) );
         B2S_TRY( upload( m->rowPointers, L.rowPointers, s ) );
         B2S_TRY( upload( m->chunksToSeg, L.chunksToSeg, s ) );
         std::vector< ChunkSlice > sl( L.slices.begin(), L.slices.begin() + nsl );
         m->chunk_single = chunked_single( L.rowToChunk, L.rowToSlice, sl );
         B2S_TRY( upload( m->cslices, sl, s ) );
         break;
      }
      case B2S_BIELLPACK: {
         const int32_t vr = ( rows % kBiWarp ) ? rows + kBiWarp - ( rows % kBiWarp ) : rows;
         const int32_t strips = vr / kBiWarp;
         if( L.virtualRows != vr || (int32_t) L.rowPerm.size() != rows ||
             (int64_t) L.groupPointers.size() != (int64_t) strips * kBiGroups + 1 || L.groupPointers[ 0 ] != 0 )
            return bad_layout( "BiEllpack array sizes" );
         for( int32_t st = 0; st < strips; st++ )
            for( int g = 0; g < kBiGroups; g++ ) {
               const int64_t a = L.groupPointers[ st * kBiGroups + g ], b = L.groupPointers[ st * kBiGroups + g + 1 ];
               if( b < a || ( b - a ) % ( kBiWarp >> g ) != 0 )
                  return bad_layout( "BiEllpack group pointers" );
            }
         uint64_t seen = 0;  // positions taken in the current strip
         for( int32_t r = 0; r < rows; r++ ) {
            if( r % kBiWarp == 0 )
               seen = 0;
            const int32_t p = L.rowPerm[ r ] - ( r / kBiWarp ) * kBiWarp;
            if( p < 0 || p >= kBiWarp || ( seen >> p & 1u ) )
               return bad_layout( "BiEllpack row permutation" );
            seen |= uint64_t( 1 ) << p;
         }
         const int64_t addressed = L.groupPointers.back();
         if( addressed > have )
            return bad_layout( "BiEllpack storage" );
         m->virtualRows = vr;
         alloc = addressed;
         B2S_TRY( upload( m->rowPerm, L.rowPerm, s ) );
         B2S_TRY( upload( m->groupPointers, L.groupPointers, s ) );
         B2S_TRY( build_rank_row( m.get(), s ) );
         int32_t mx = 0;  // the widest strip, an upper bound of a row's length
         for( int32_t st = 0; st < strips; st++ )
            mx = std::max< int64_t >( mx, ( L.groupPointers[ ( st + 1 ) * kBiGroups ] - L.groupPointers[ st * kBiGroups ] ) );
         m->max_row = mx;
         break;
      }
      default:
         return bad_layout( "not a padded layout" );
   }
   m->alloc_elems = alloc;
   int64_t nnz = 0;
   for( int64_t k = 0; k < alloc; k++ )
      nnz += L.columns[ k ] != -1;
   m->nnz = nnz;
   m->mean_row = rows > 0 ? (double) nnz / rows : 0.0;
   B2S_TRY( m->values.alloc( (size_t) std::max< int64_t >( alloc, 1 ) * es ) );
   B2S_TRY( m->columns.alloc( (size_t) std::max< int64_t >( alloc, 1 ) * sizeof( int32_t ) ) );
   if( alloc > 0 ) {
      B2S_TRY( copy_h2d( m->values.p, L.values.data(), (size_t) alloc * es, s ) );
      B2S_TRY( copy_h2d( m->columns.p, L.columns.data(), (size_t) alloc * sizeof( int32_t ), s ) );
   }
   B2S_TRY( m->status.alloc( 4 * sizeof( int ) ) );
   B2S_TRY_CUDA( cudaMemsetAsync( m->status.p, 0, 4 * sizeof( int ), s ) );
   B2S_TRY( m->diagonal.alloc( (size_t) std::max( rows, 1 ) * es ) );
   B2S_TRY( build_diagonal( m.get(), s ) );
   if( o.keep_fp32_copy )
      B2S_TRY( ensure_fp32_copy( m.get(), s ) );
   B2S_TRY_CUDA( cudaStreamSynchronize( s ) );
   *out = m.release();
   return B2S_OK;
}

b2s_status
matrix_from_assembled( b2s_format format, b2s_dtype dtype, int32_t rows, int32_t cols, int64_t nnz, const int32_t* off,
                       const int32_t* col, const void* val, const int32_t* caps, int64_t caps_total,
                       const b2s_matrix_opts& o, cudaStream_t s, b2s_matrix* out )
{
   std::unique_ptr< b2s_matrix_t > m( new b2s_matrix_t() );
   m->format = format;
   m->dtype = dtype;
   m->rows = rows;
   m->cols = cols;
   m->device = current_device();
   b2s_status st = dtype == B2S_F64
                    ? build_from_device_csr< double >( m.get(), off, col, static_cast< const double* >( val ), nnz, o, s,
                                                       caps, true, caps_total )
                    : build_from_device_csr< float >( m.get(), off, col, static_cast< const float* >( val ), nnz, o, s,
                                                      caps, true, caps_total );
   if( st != B2S_OK )
      return st;
   if( o.symmetric )
      B2S_TRY( mark_symmetric( m.get(), s ) );
   if( o.keep_fp32_copy )
      B2S_TRY( ensure_fp32_copy( m.get(), s ) );
   *out = m.release();
   return B2S_OK;
}

// every stored column of row i is <= i
__global__ void
lower_check_kernel( const int32_t* __restrict__ off, const int32_t* __restrict__ col, int32_t rows, int* bad )
{
   for( int64_t r = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; r < rows; r += (int64_t) gridDim.x * blockDim.x )
      for( int k = off[ r ]; k < off[ r + 1 ]; k++ )
         if( col[ k ] > r ) {
            atomicExch( bad, 1 );
            break;
         }
}

__global__ void
rank_row_kernel( const int32_t* __restrict__ rowPerm, int32_t rows, int32_t* rankRow )
{
   for( int64_t r = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; r < rows; r += (int64_t) gridDim.x * blockDim.x )
      rankRow[ rowPerm[ r ] ] = (int32_t) r;
}

b2s_status
build_rank_row( b2s_matrix_t* m, cudaStream_t s )
{
   const int64_t vr = std::max( m->virtualRows, 1 );
   B2S_TRY( m->rankRow.alloc( (size_t) vr * sizeof( int32_t ) ) );
   B2S_TRY_CUDA( cudaMemsetAsync( m->rankRow.p, 0xff, (size_t) vr * sizeof( int32_t ), s ) );  // -1
   if( m->rows > 0 ) {
      rank_row_kernel<<< grid_for( m->rows ), 256, 0, s >>>( m->rowPerm.as< int32_t >(), m->rows,
                                                             m->rankRow.as< int32_t >() );
      B2S_TRY_CUDA( cudaGetLastError() );
   }
   return B2S_OK;
}

// the same check through any layout (padding slots skipped)
__global__ void
layout_lower_check_kernel( LayoutView L, int32_t rows, int32_t segmentSize, const int32_t* __restrict__ col, int* bad )
{
   for( int64_t r = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; r < rows; r += (int64_t) gridDim.x * blockDim.x ) {
      const int64_t cap = L.capacity( (int) r, segmentSize );
      for( int64_t k = 0; k < cap; k++ ) {
         const int64_t g = L.gidx( (int) r, (int) k );
         if( g < 0 )
            break;
         if( col[ g ] > r ) {
            atomicExch( bad, 1 );
            break;
         }
      }
   }
}

b2s_status
mark_symmetric( b2s_matrix_t* m, cudaStream_t s )
{
   if( m->rows != m->cols ) {
      set_error( "SymmetricMatrix must be square" );
      return B2S_INVALID_ARG;
   }
   if( m->rows > 0 ) {
      DevBuf flag;
      B2S_TRY( flag.alloc( sizeof( int ) ) );
      B2S_TRY_CUDA( cudaMemsetAsync( flag.p, 0, sizeof( int ), s ) );
      if( m->format == B2S_CSR )
         lower_check_kernel<<< grid_for( m->rows ), 256, 0, s >>>( m->offsets.as< int32_t >(),
                                                                    m->columns.as< int32_t >(), m->rows, flag.as< int >() );
      else
         layout_lower_check_kernel<<< grid_for( m->rows ), 256, 0, s >>>( view_of( m ), m->rows, m->segmentSize,
                                                                           m->columns.as< int32_t >(), flag.as< int >() );
      B2S_TRY_CUDA( cudaGetLastError() );
      int bad = 0;
      B2S_TRY( copy_d2h( &bad, flag.p, sizeof( int ), s ) );
      if( bad ) {
         set_error( "SymmetricMatrix stores the lower triangle only: an element has column > row" );
         return B2S_INVALID_ARG;
      }
   }
   m->symmetric = 1;
   return B2S_OK;
}

// triplets of L + L^T - D: element k of row i gives (i, j, v), and (j, i, v) at
// nnz + mpos[k] when j < i
template< typename Real >
__global__ void
expand_triplets_kernel( const int32_t* __restrict__ off, const int32_t* __restrict__ col, const Real* __restrict__ val,
                        int32_t rows, int64_t nnz, const int64_t* __restrict__ mpos, int32_t* ti, int32_t* tj, Real* tv )
{
   for( int64_t r = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; r < rows; r += (int64_t) gridDim.x * blockDim.x )
      for( int k = off[ r ]; k < off[ r + 1 ]; k++ ) {
         const int j = col[ k ];
         ti[ k ] = (int) r;
         tj[ k ] = j;
         tv[ k ] = val[ k ];
         if( j < r ) {
            const int64_t q = nnz + mpos[ k ];
            ti[ q ] = j;
            tj[ q ] = (int) r;
            tv[ q ] = val[ k ];
         }
      }
}

__global__ void
strict_lower_flags_kernel( const int32_t* __restrict__ off, const int32_t* __restrict__ col, int32_t rows,
                           int64_t* flags )
{
   for( int64_t r = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; r < rows; r += (int64_t) gridDim.x * blockDim.x )
      for( int k = off[ r ]; k < off[ r + 1 ]; k++ )
         flags[ k ] = col[ k ] < r ? 1 : 0;
}

b2s_status
expand_symmetric( const b2s_matrix_t* src, cudaStream_t s, b2s_matrix_t** out )
{
   *out = nullptr;
   // a padded layout's stored elements as CSR first (padding dropped, zeros kept)
   std::unique_ptr< b2s_matrix_t > csr_src;
   const b2s_matrix_t* m = src;
   if( src->format != B2S_CSR ) {
      DevBuf off, col, val;
      int64_t nz = 0;
      B2S_TRY( layout_to_csr( src, false, off, col, val, nz, s ) );
      b2s_matrix t = nullptr;
      B2S_TRY( b2s_matrix_create( B2S_CSR, (b2s_dtype) src->dtype, src->rows, src->cols, nz, off.as< int32_t >(),
                                  col.as< int32_t >(), val.p, (b2s_dtype) src->dtype, B2S_DEVICE, nullptr, s, &t ) );
      csr_src.reset( t );
      m = t;
   }
   const int64_t nnz = m->nnz;
   const size_t es = m->dtype == B2S_F64 ? 8 : 4;
   DevBuf mpos;
   B2S_TRY( mpos.alloc( (size_t) ( nnz + 1 ) * sizeof( int64_t ) ) );
   B2S_TRY_CUDA( cudaMemsetAsync( mpos.p, 0, (size_t) ( nnz + 1 ) * sizeof( int64_t ), s ) );
   if( m->rows > 0 ) {
      strict_lower_flags_kernel<<< grid_for( m->rows ), 256, 0, s >>>( m->offsets.as< int32_t >(),
                                                                        m->columns.as< int32_t >(), m->rows,
                                                                        mpos.as< int64_t >() );
      B2S_TRY_CUDA( cudaGetLastError() );
   }
   B2S_TRY( scan_exclusive_i64( mpos.as< int64_t >(), nnz + 1, s ) );
   int64_t mirrored = 0;
   B2S_TRY( copy_d2h( &mirrored, mpos.as< int64_t >() + nnz, sizeof( int64_t ), s ) );
   const int64_t count = nnz + mirrored;
   DevBuf ti, tj, tv;
   B2S_TRY( ti.alloc( (size_t) std::max< int64_t >( count, 1 ) * sizeof( int32_t ) ) );
   B2S_TRY( tj.alloc( (size_t) std::max< int64_t >( count, 1 ) * sizeof( int32_t ) ) );
   B2S_TRY( tv.alloc( (size_t) std::max< int64_t >( count, 1 ) * es ) );
   if( m->rows > 0 ) {
      if( m->dtype == B2S_F64 )
         expand_triplets_kernel< double ><<< grid_for( m->rows ), 256, 0, s >>>(
            m->offsets.as< int32_t >(), m->columns.as< int32_t >(), m->values.as< double >(), m->rows, nnz,
            mpos.as< int64_t >(), ti.as< int32_t >(), tj.as< int32_t >(), tv.as< double >() );
      else
         expand_triplets_kernel< float ><<< grid_for( m->rows ), 256, 0, s >>>(
            m->offsets.as< int32_t >(), m->columns.as< int32_t >(), m->values.as< float >(), m->rows, nnz,
            mpos.as< int64_t >(), ti.as< int32_t >(), tj.as< int32_t >(), tv.as< float >() );
      B2S_TRY_CUDA( cudaGetLastError() );
   }
   b2s_matrix_opts o;
   b2s_matrix_opts_default( &o );
   o.csr_kernel = m->csr_kernel;
   o.csr_row_groups = m->csr_group_opt;
   b2s_matrix g = nullptr;
   B2S_TRY( b2s_matrix_from_coo( B2S_CSR, (b2s_dtype) m->dtype, m->rows, m->cols, count, ti.as< int32_t >(),
                                 tj.as< int32_t >(), tv.p, (b2s_dtype) m->dtype, B2S_DEVICE, B2S_DUP_ADD, nullptr, &o,
                                 s, &g ) );
   *out = g;
   return B2S_OK;
}

b2s_status
build_diagonal( b2s_matrix_t* A, cudaStream_t s )
{
   if( A->rows == 0 )
      return B2S_OK;
   const LayoutView L = view_of( A );
   if( A->dtype == B2S_F64 )
      layout_diag_kernel< double ><<< grid_for( A->rows ), 256, 0, s >>>(
         L, A->rows, A->segmentSize, A->columns.as< int32_t >(), A->values.as< double >(), A->diagonal.as< double >() );
   else
      layout_diag_kernel< float ><<< grid_for( A->rows ), 256, 0, s >>>(
         L, A->rows, A->segmentSize, A->columns.as< int32_t >(), A->values.as< float >(), A->diagonal.as< float >() );
   B2S_TRY_CUDA( cudaGetLastError() );
   return B2S_OK;
}

b2s_status
ensure_fp32_copy( b2s_matrix_t* A, cudaStream_t s )
{
   if( A->dtype == B2S_F32 || A->values32.p )
      return B2S_OK;
   const int64_t n = A->alloc_elems;
   B2S_TRY( A->values32.alloc( (size_t) std::max< int64_t >( n, 1 ) * sizeof( float ) ) );
   if( n > 0 ) {
      cast_kernel< double, float ><<< grid_for( n ), 256, 0, s >>>( A->values.as< double >(), A->values32.as< float >(), n );
      B2S_TRY_CUDA( cudaGetLastError() );
   }
   B2S_TRY_CUDA( cudaStreamSynchronize( s ) );
   return B2S_OK;
}

}  // namespace b2s

using namespace b2s;

extern "C" {

void
b2s_matrix_opts_default( b2s_matrix_opts* o )
{
   if( ! o )
      return;
   std::memset( o, 0, sizeof( *o ) );
   o->csr_kernel = B2S_CSR_AUTO;
}

b2s_status
b2s_matrix_create( b2s_format format, b2s_dtype dtype, int32_t rows, int32_t cols, int64_t nnz, const int32_t* offsets,
                   const int32_t* columns, const void* values, b2s_dtype values_dtype, b2s_memory where,
                   const b2s_matrix_opts* opts, b2s_stream stream, b2s_matrix* out )
{
   clear_error();
   B2S_CHECK_ARG( out, "out handle is NULL" );
   *out = nullptr;
   B2S_CHECK_ARG( format >= B2S_CSR && format <= B2S_MULTIDIAGONAL, "format" );
   B2S_CHECK_ARG( dtype == B2S_F64 || dtype == B2S_F32 || dtype == B2S_BOOL, "dtype" );
   B2S_CHECK_ARG( values_dtype == B2S_F64 || values_dtype == B2S_F32, "values_dtype" );
   B2S_CHECK_ARG( where == B2S_HOST || where == B2S_DEVICE, "where" );
   B2S_CHECK_ARG( rows >= 0 && cols >= 0 && nnz >= 0, "negative size" );
   B2S_CHECK_ARG( nnz <= INT32_MAX, "nnz exceeds 32-bit indices" );
   B2S_CHECK_ARG( offsets, "offsets is NULL" );
   B2S_CHECK_ARG( nnz == 0 || ( columns && ( values || dtype == B2S_BOOL ) ), "columns/values NULL" );
   b2s_matrix_opts o;
   b2s_matrix_opts_default( &o );
   if( opts )
      o = *opts;
   if( format == B2S_MULTIDIAGONAL && ( dtype == B2S_BOOL || o.symmetric ) ) {
      set_error( "a Multidiagonal matrix holds FP64 or FP32 values of a general matrix" );
      return B2S_UNSUPPORTED;
   }
   if( dtype == B2S_BOOL )
      return create_binary( format, rows, cols, nnz, offsets, columns, values, values_dtype, where, o,
                            as_stream( stream ), out );
   std::unique_ptr< b2s_matrix_t > m( new b2s_matrix_t() );
   m->format = format;
   m->dtype = dtype;
   m->rows = rows;
   m->cols = cols;
   m->device = current_device();
   cudaStream_t s = as_stream( stream );
   b2s_status st = values_dtype == B2S_F64
                    ? build_any< double >( m.get(), offsets, columns, values, nnz, where, o, s )
                    : build_any< float >( m.get(), offsets, columns, values, nnz, where, o, s );
   if( st != B2S_OK )
      return st;
   if( o.symmetric )
      B2S_TRY( mark_symmetric( m.get(), s ) );
   if( o.keep_fp32_copy )
      B2S_TRY( ensure_fp32_copy( m.get(), s ) );
   *out = m.release();
   return B2S_OK;
}

b2s_status
b2s_matrix_convert( b2s_matrix src, b2s_format format, b2s_dtype dtype, const b2s_matrix_opts* opts, b2s_stream stream,
                    b2s_matrix* out )
{
   clear_error();
   B2S_NO_BINARY( src, "conversion" );
   B2S_CHECK_ARG( src && out, "NULL handle" );
   if( src->format != B2S_CSR && src->format == format && src->dtype == dtype &&
       ( format != B2S_SLICED_ELLPACK || ( opts ? ( opts->slice_size ? opts->slice_size : kSliceSize ) : kSliceSize ) ==
                                            src->slice_size ) ) {
      // the same matrix type: TNL's copy assignment — the same arrays
      std::unique_ptr< b2s_matrix_t > m( new b2s_matrix_t() );
      B2S_TRY( clone_matrix( src, m.get(), as_stream( stream ) ) );
      if( opts && opts->keep_fp32_copy )
         B2S_TRY( ensure_fp32_copy( m.get(), as_stream( stream ) ) );
      *out = m.release();
      return B2S_OK;
   }
   if( src->format != B2S_CSR ) {
      // padded source: TNL takes the row capacities from the source's
      // non-padding slots (SparseMatrixView::getRowCapacities) and copies the
      // nonzero values — the CSR path does exactly that from the source's rows
      // with their stored zeros (a CSR target gets the zeros dropped instead
      // of unused slots)
      cudaStream_t s = as_stream( stream );
      DevBuf off, col, val;
      int64_t nnz = 0;
      B2S_TRY( layout_to_csr( src, format == B2S_CSR, off, col, val, nnz, s ) );
      b2s_matrix_opts o;
      b2s_matrix_opts_default( &o );
      if( opts )
         o = *opts;
      if( src->symmetric )
         o.symmetric = 1;
      return b2s_matrix_create( format, dtype, src->rows, src->cols, nnz, off.as< int32_t >(), col.as< int32_t >(),
                                val.p, (b2s_dtype) src->dtype, B2S_DEVICE, &o, stream, out );
   }
   const void* vals = src->values.p;
   if( src->symmetric ) {
      // a SymmetricMatrix stays one: its lower triangle in another layout / value type
      b2s_matrix_opts o;
      b2s_matrix_opts_default( &o );
      if( opts )
         o = *opts;
      o.symmetric = 1;
      return b2s_matrix_create( format, dtype, src->rows, src->cols, src->nnz, src->offsets.as< int32_t >(),
                                src->columns.as< int32_t >(), vals, (b2s_dtype) src->dtype, B2S_DEVICE, &o, stream,
                                out );
   }
   return b2s_matrix_create( format, dtype, src->rows, src->cols, src->nnz, src->offsets.as< int32_t >(),
                             src->columns.as< int32_t >(), vals, (b2s_dtype) src->dtype, B2S_DEVICE, opts, stream, out );
}

b2s_status
b2s_matrix_destroy( b2s_matrix m )
{
   clear_error();
   delete m;
   return B2S_OK;
}

b2s_status
b2s_matrix_get_info( b2s_matrix m, b2s_matrix_info* info )
{
   clear_error();
   B2S_CHECK_ARG( m && info, "NULL argument" );
   info->format = m->format;
   info->dtype = m->dtype;
   info->rows = m->rows;
   info->cols = m->cols;
   info->nnz = m->nnz;
   info->storage_size = m->storage;
   info->device_bytes = m->device_bytes();
   info->csr_kernel = m->format == B2S_CSR ? m->csr_kernel : 0;
   info->threads_per_row = m->format == B2S_CSR ? m->tpr : 0;
   info->csr_path = m->format == B2S_CSR && m->csr_kernel == B2S_CSR_ADAPTIVE ? ( m->csr_group ? 1 : 2 ) : 0;
   info->symmetric = m->symmetric;
   return B2S_OK;
}

b2s_status
b2s_matrix_export_range( b2s_matrix m, const char* name, int64_t first, int64_t count, void* host_out )
{
   clear_error();
   B2S_CHECK_ARG( m && name && ( host_out || count == 0 ), "NULL argument" );
   const std::string n( name );
   B2S_CHECK_ARG( n == "values" || n == "columnIndexes", "export_range: only values and columnIndexes" );
   B2S_CHECK_ARG( n == "columnIndexes" || m->dtype != B2S_BOOL, "export_range: a binary matrix stores no values" );
   B2S_CHECK_ARG( first >= 0 && count >= 0 && first + count <= m->storage, "export_range: range outside the storage" );
   const bool vals = n == "values";
   const size_t es = vals ? dsize( m->dtype ) : sizeof( int32_t );
   const int64_t have = std::max< int64_t >( 0, std::min( first + count, m->alloc_elems ) - first );
   if( have > 0 )
      B2S_TRY( copy_d2h( host_out, static_cast< const char* >( vals ? m->values.p : m->columns.p ) + first * es,
                         have * es, nullptr ) );
   char* base = static_cast< char* >( host_out );
   for( int64_t i = have; i < count; i++ ) {
      if( ! vals )
         reinterpret_cast< int32_t* >( base )[ i ] = -1;
      else if( m->dtype == B2S_F64 )
         reinterpret_cast< double* >( base )[ i ] = 0.0;
      else
         reinterpret_cast< float* >( base )[ i ] = 0.0f;
   }
   return B2S_OK;
}

b2s_status
b2s_matrix_export( b2s_matrix m, const char* name, void* host_out, int64_t capacity, int64_t* count )
{
   clear_error();
   B2S_CHECK_ARG( m && name && count, "NULL argument" );
   const std::string n( name );
   cudaStream_t s = nullptr;
   auto scalar = [ & ]( int64_t v ) -> b2s_status
   {
      *count = 1;
      if( host_out ) {
         B2S_CHECK_ARG( capacity >= 1, "capacity" );
         static_cast< int64_t* >( host_out )[ 0 ] = v;
      }
      return B2S_OK;
   };
   auto array_i32 = [ & ]( const DevBuf& b, int64_t len ) -> b2s_status
   {
      *count = len;
      if( ! host_out )
         return B2S_OK;
      B2S_CHECK_ARG( capacity >= len, "capacity too small" );
      std::vector< int32_t > tmp( len );
      if( len > 0 )
         B2S_TRY( copy_d2h( tmp.data(), b.p, len * sizeof( int32_t ), s ) );
      int64_t* o = static_cast< int64_t* >( host_out );
      for( int64_t i = 0; i < len; i++ )
         o[ i ] = tmp[ i ];
      return B2S_OK;
   };
   if( n == "values" && m->dtype == B2S_BOOL ) {
      *count = 0;  // a binary matrix stores no values (SparseMatrix.hpp:297-302)
      return B2S_OK;
   }
   if( n == "values" || n == "columnIndexes" ) {
      *count = m->storage;
      if( ! host_out )
         return B2S_OK;
      B2S_CHECK_ARG( capacity >= m->storage, "capacity too small" );
      const bool vals = n == "values";
      const size_t es = vals ? dsize( m->dtype ) : sizeof( int32_t );
      if( m->alloc_elems > 0 )
         B2S_TRY( copy_d2h( host_out, vals ? m->values.p : m->columns.p, m->alloc_elems * es, s ) );
      // slots TNL allocates but never addresses (BiEllpack) read as padding
      char* base = static_cast< char* >( host_out );
      for( int64_t i = m->alloc_elems; i < m->storage; i++ ) {
         if( vals ) {
            if( m->dtype == B2S_F64 )
               reinterpret_cast< double* >( base )[ i ] = 0.0;
            else
               reinterpret_cast< float* >( base )[ i ] = 0.0f;
         }
         else
            reinterpret_cast< int32_t* >( base )[ i ] = -1;
      }
      return B2S_OK;
   }
   switch( m->format ) {
      case B2S_CSR:
         if( n == "offsets" )
            return array_i32( m->offsets, (int64_t) m->rows + 1 );
         break;
      case B2S_ELLPACK:
         if( n == "segmentSize" )
            return scalar( m->segmentSize );
         if( n == "size" )
            return scalar( m->rows );
         if( n == "alignedSize" )
            return scalar( m->alignedSize );
         break;
      case B2S_SLICED_ELLPACK:
         if( n == "sliceOffsets" )
            return array_i32( m->sliceOffsets, (int64_t) m->nslices + 1 );
         if( n == "sliceSegmentSizes" )
            return array_i32( m->sliceSegmentSizes, m->nslices );
         if( n == "size" )
            return scalar( m->cap_total );
         if( n == "alignedSize" )
            return scalar( m->storage );
         break;
      case B2S_CHUNKED_ELLPACK:
         if( n == "rowToChunkMapping" )
            return array_i32( m->rowToChunk, m->rows );
         if( n == "rowToSliceMapping" )
            return array_i32( m->rowToSlice, m->rows );
         if( n == "chunksToSegmentsMapping" )
            return array_i32( m->chunksToSeg, (int64_t) m->numberOfSlices * kChunksInSlice );
         if( n == "rowPointers" )
            return array_i32( m->rowPointers, (int64_t) m->rows + 1 );
         if( n == "slices" )
            return array_i32( m->cslices, (int64_t) m->numberOfSlices * 4 );
         if( n == "numberOfSlices" )
            return scalar( m->numberOfSlices );
         if( n == "storageSize" )
            return scalar( m->storage );
         break;
      case B2S_MULTIDIAGONAL:
         if( n == "diagonalsOffsets" )
            return array_i32( m->diagOffsets, m->segmentSize );
         if( n == "nonemptyRows" )
            return scalar( m->alignedSize );
         break;
      case B2S_BIELLPACK:
         if( n == "rowPermArray" )
            return array_i32( m->rowPerm, m->rows );
         if( n == "groupPointers" )
            return array_i32( m->groupPointers, (int64_t) ( m->virtualRows / kBiWarp ) * kBiGroups + 1 );
         if( n == "virtualRows" )
            return scalar( m->virtualRows );
         if( n == "storageSize" )
            return scalar( m->storage );
         break;
   }
   set_error( "no array '%s' for this layout", name );
   return B2S_INVALID_ARG;
}

}  // extern "C"
