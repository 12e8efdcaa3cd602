// SpMV kernels over the five segment layouts (sm_100a).
//
// Each kernel computes, for every row r in [row_begin, row_end), the sum over
// the row's stored elements of value * x[column] and hands it to a `Sink`:
//   sink.put( r, sum, acc )  — writes y (TNL's keepers, SparseMatrixView.hpp:448-471)
//                              and may add to per-thread accumulators acc[0..NR)
// When Sink::NR > 0 the kernel ends with a deterministic grid reduction of the
// accumulators and calls Sink::finish( totals ) once, from the last block —
// this is how the Krylov solvers fuse their dot products into the SpMV.
//
// Layout traversal follows TNL's Devices::Cuda segments (ColumnMajorOrder):
//   CSR             Segments/CSRView.hpp:185-200 (+ Kernels/CSR*Kernel.hpp)
//   Ellpack         Segments/EllpackView.hpp:331-372
//   SlicedEllpack   Segments/SlicedEllpackView.hpp:237-284
//   ChunkedEllpack  Segments/ChunkedEllpackView.hpp:409-530
//   BiEllpack       Segments/BiEllpackView.hpp:386-560
#pragma once

#include "b2s_internal.cuh"
#include "tma.cuh"

namespace b2s {

constexpr int kSpmvBlock = 256;

// y = alpha*s + beta*y with TNL's keeper selection (exact same arithmetic per case)
template< typename Real >
struct YSink
{
   static constexpr int NR = 0;
   Real* y;
   Real alpha, beta;
   int mode;  // 0: y=s, 1: y=alpha*s, 2: y=beta*y+s, 3: y=beta*y+alpha*s
   __device__ __forceinline__ void
   put( int row, Real s, double* ) const
   {
      switch( mode ) {
         case 0: y[ row ] = s; break;
         case 1: y[ row ] = alpha * s; break;
         case 2: y[ row ] = beta * y[ row ] + s; break;
         default: y[ row ] = beta * y[ row ] + alpha * s; break;
      }
   }
   __device__ void finish( const double* ) const {}
   __device__ bool skip() const { return false; }
};

template< typename Real >
__host__ __device__ inline int
keeper_mode( Real alpha, Real beta )
{
   if( beta == Real( 0 ) )
      return alpha == Real( 1 ) ? 0 : 1;
   return alpha == Real( 1 ) ? 2 : 3;
}

// Common epilogue: reduce the sink accumulators when the sink asks for it.
template< class Sink, int BLOCK >
__device__ __forceinline__ void
spmv_epilogue( const Sink& sink, double* acc, RedScratch rs )
{
   if constexpr( Sink::NR > 0 ) {
      double a[ Sink::NR ], t[ Sink::NR ];
#pragma unroll
      for( int k = 0; k < Sink::NR; k++ )
         a[ k ] = acc[ k ];
      if( grid_reduce< Sink::NR, BLOCK >( a, rs, t ) && threadIdx.x == 0 )
         sink.finish( t );
   }
}

template< class Sink >
struct AccOf
{
   double v[ Sink::NR > 0 ? Sink::NR : 1 ];
};

// Read-only global loads that do not allocate in L1 (matrix data is streamed once).
template< typename T >
__device__ __forceinline__ T
ld_stream( const T* p )
{
   return __ldcs( p );
}

// ---------------------------------------------------------------------------
// CSR, TPR threads per row (TPR = 1: one thread per row, summing in the
// row's element order exactly like TNL's CSRScalar kernel; TPR > 1: strided
// partial sums combined with a fixed butterfly).
template< typename Real, int TPR, class Sink >
__global__ void __launch_bounds__( kSpmvBlock )
csr_vector_kernel( const int32_t* __restrict__ off, const int32_t* __restrict__ col, const Real* __restrict__ val,
                   const Real* __restrict__ x, int32_t row_begin, int32_t row_end, Sink sink, RedScratch rs )
{
   if( sink.skip() )
      return;  // uniform over the grid: the solve this launch belongs to is finished
   AccOf< Sink > acc{};
   constexpr int RPW = 32 / TPR;  // rows per warp and step
   const int lane = threadIdx.x & 31;
   const int sub = lane % TPR;
   const int64_t warp_global = ( blockIdx.x * (int64_t) kSpmvBlock + threadIdx.x ) >> 5;
   const int64_t nwarps = ( (int64_t) gridDim.x * kSpmvBlock ) >> 5;
   // the loop bound is warp-uniform so the shuffles below always see the full warp
   for( int64_t base = row_begin + warp_global * RPW; base < row_end; base += nwarps * RPW ) {
      const int64_t r = base + lane / TPR;
      const bool active = r < row_end;
      Real s = 0;
      if( active ) {
         const int b = __ldg( off + r ), e = __ldg( off + r + 1 );
         for( int k = b + sub; k < e; k += TPR )
            s += ld_stream( val + k ) * __ldg( x + ld_stream( col + k ) );
      }
      if constexpr( TPR > 1 ) {
#pragma unroll
         for( int o = TPR / 2; o > 0; o >>= 1 )
            s += __shfl_xor_sync( 0xffffffffu, s, o, TPR );
      }
      if( active && sub == 0 )
         sink.put( (int) r, s, acc.v );
   }
   spmv_epilogue< Sink, kSpmvBlock >( sink, acc.v, rs );
}

// ---------------------------------------------------------------------------
// CSR, nnz-balanced tiles ("adaptive" row binning without a host pass).
// Tile t owns the rows whose first nonzero lies in the window
// [t*kTileNnz, (t+1)*kTileNnz) of the nonzero array (tile_rows[t] = first such
// row, found by binary search when the matrix is built). A CTA
//   1. streams the tile's nonzeros with 128-bit loads of columns and values,
//      multiplies by the gathered x and keeps the products in shared memory;
//   2. sums each row from shared memory with `tpr` threads per row (chosen
//      per tile from its mean row length; tpr = 1 adds in the row's element
//      order, exactly like TNL's CSRScalar kernel);
//   3. if the tile's last row is too long for the buffer, reduces it with the
//      whole CTA straight from global memory.
// Every tile moves about kTileNnz nonzeros, whatever the row lengths.
constexpr int kTileBlock = 256;

template< typename Real >
struct Vec4;
template<>
struct Vec4< double >
{
   __device__ __forceinline__ static void
   load( const double* p, double ( &v )[ 4 ] )
   {
      const double2 a = __ldcs( reinterpret_cast< const double2* >( p ) );
      const double2 b = __ldcs( reinterpret_cast< const double2* >( p ) + 1 );
      v[ 0 ] = a.x;
      v[ 1 ] = a.y;
      v[ 2 ] = b.x;
      v[ 3 ] = b.y;
   }
};
template<>
struct Vec4< float >
{
   __device__ __forceinline__ static void
   load( const float* p, float ( &v )[ 4 ] )
   {
      const float4 a = __ldcs( reinterpret_cast< const float4* >( p ) );
      v[ 0 ] = a.x;
      v[ 1 ] = a.y;
      v[ 2 ] = a.z;
      v[ 3 ] = a.w;
   }
};

template< typename Real, int TPR, class Sink >
__device__ __forceinline__ void
tile_rows_from_smem( const Real* prod, const int32_t* __restrict__ off, int r0, int rlast, int a, const Sink& sink,
                     double* acc )
{
   constexpr int RPW = 32 / TPR;
   constexpr int WARPS = kTileBlock / 32;
   const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
   const int sub = lane % TPR;
   for( int base = r0 + warp * RPW; base < rlast; base += WARPS * RPW ) {
      const int r = base + lane / TPR;
      const bool active = r < rlast;
      Real s = 0;
      if( active ) {
         const int e = __ldg( off + r + 1 ) - a;
         for( int k = __ldg( off + r ) - a + sub; k < e; k += TPR )
            s += prod[ k ];
      }
      if constexpr( TPR > 1 ) {
#pragma unroll
         for( int o = TPR / 2; o > 0; o >>= 1 )
            s += __shfl_xor_sync( 0xffffffffu, s, o, TPR );
      }
      if( active && sub == 0 )
         sink.put( r, s, acc );
   }
}

// Persistent, TMA-fed version: tile t is exactly the window
// [t*kTileNnz, (t+1)*kTileNnz) of the nonzero arrays. One thread streams the
// columns and values of upcoming windows into a kTmaStages-deep ring of
// shared-memory buffers with bulk asynchronous copies (cp.async.bulk,
// completing on an mbarrier per stage) while the CTA works on the current
// window:
//   1. products value*x[column] of the window, in place in shared memory;
//   2. the rows owned by the tile (those starting in the window) are summed
//      from shared memory; the part of the last row that runs past the window
//      is read from global memory (L2-warm: the next window holds it);
//   3. the stage is released and refilled with the window kTmaStages ahead.
// Dynamic shared memory: kTmaStages * kTileNnz * (4 + sizeof(Real)) bytes.
constexpr int kTmaStages = 3;

template< typename Real >
constexpr size_t
tma_smem_bytes()
{
   return (size_t) kTmaStages * kTileNnz * ( sizeof( int32_t ) + sizeof( Real ) ) + kTmaStages * sizeof( uint64_t );
}

template< typename Real, int TPR, class Sink >
__device__ __forceinline__ void
tma_rows( const Real* prod, const int32_t* __restrict__ off, const int32_t* __restrict__ col,
          const Real* __restrict__ val, const Real* __restrict__ x, int r0, int r1, int64_t w0, int len,
          const Sink& sink, double* acc )
{
   constexpr int RPW = 32 / TPR;
   constexpr int WARPS = kTileBlock / 32;
   const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
   const int sub = lane % TPR;
   for( int base = r0 + warp * RPW; base < r1; base += WARPS * RPW ) {
      const int r = base + lane / TPR;
      const bool active = r < r1;
      Real s = 0;
      if( active ) {
         const int64_t b = __ldg( off + r ), e = __ldg( off + r + 1 );
         const int in_end = (int) min( e - w0, (int64_t) len );
         for( int k = (int) ( b - w0 ) + sub; k < in_end; k += TPR )
            s += prod[ k ];
         for( int64_t k = w0 + len + sub; k < e; k += TPR )  // overhang past the window
            s += __ldg( val + k ) * __ldg( x + __ldg( col + k ) );
      }
      if constexpr( TPR > 1 ) {
#pragma unroll
         for( int o = TPR / 2; o > 0; o >>= 1 )
            s += __shfl_xor_sync( 0xffffffffu, s, o, TPR );
      }
      if( active && sub == 0 )
         sink.put( r, s, acc );
   }
}

template< typename Real, class Sink >
__global__ void __launch_bounds__( kTileBlock )
csr_tma_kernel( const int32_t* __restrict__ off, const int32_t* __restrict__ col, const Real* __restrict__ val,
                const Real* __restrict__ x, const int32_t* __restrict__ tile_rows, int32_t ntiles, int64_t nnz,
                Sink sink, RedScratch rs, int* err )
{
   if( sink.skip() )
      return;  // uniform over the grid: the solve this launch belongs to is finished
   extern __shared__ __align__( 128 ) unsigned char tma_smem[];
   int32_t* scol = reinterpret_cast< int32_t* >( tma_smem );
   Real* sval = reinterpret_cast< Real* >( tma_smem + (size_t) kTmaStages * kTileNnz * sizeof( int32_t ) );
   uint64_t* bar = reinterpret_cast< uint64_t* >( tma_smem + (size_t) kTmaStages * kTileNnz
                                                                * ( sizeof( int32_t ) + sizeof( Real ) ) );
   AccOf< Sink > acc{};
   if( threadIdx.x == 0 ) {
      for( int s = 0; s < kTmaStages; s++ )
         mbar_init( bar + s, 1 );
      fence_mbar_init();
   }
   __syncthreads();

   // thread 0: fill stage (k % S) with the window of this CTA's k-th tile
   auto issue = [ & ]( int k )
   {
      const int64_t t = blockIdx.x + (int64_t) k * gridDim.x;
      if( t >= ntiles )
         return;
      const int s = k % kTmaStages;
      const int64_t w0 = t * kTileNnz;
      const int64_t len = min( (int64_t) kTileNnz, nnz - w0 );
      if( len <= 0 ) {
         mbar_arrive( bar + s );  // empty window (trailing empty rows): complete the phase
         return;
      }
      const uint32_t bc = (uint32_t) ( ( len * sizeof( int32_t ) + 15 ) & ~15ll );
      const uint32_t bv = (uint32_t) ( ( len * sizeof( Real ) + 15 ) & ~15ll );
      mbar_arrive_expect_tx( bar + s, bc + bv );
      bulk_g2s( scol + (size_t) s * kTileNnz, col + w0, bc, bar + s );
      bulk_g2s( sval + (size_t) s * kTileNnz, val + w0, bv, bar + s );
   };
   if( threadIdx.x == 0 )
      for( int k = 0; k < kTmaStages; k++ )
         issue( k );

   bool failed = false;
   int k = 0;
   for( ; blockIdx.x + (int64_t) k * gridDim.x < ntiles; k++ ) {
      const int t = blockIdx.x + k * gridDim.x;
      const int s = k % kTmaStages;
      const bool ok = mbar_wait_bounded( bar + s, ( k / kTmaStages ) & 1 );
      if( __syncthreads_or( ! ok ) ) {
         failed = true;
         break;
      }
      const int64_t w0 = (int64_t) t * kTileNnz;
      const int len = (int) max( (int64_t) 0, min( (int64_t) kTileNnz, nnz - w0 ) );
      const int32_t* c = scol + (size_t) s * kTileNnz;
      Real* p = sval + (size_t) s * kTileNnz;
      {
         // all gathers of x issued before any is used (kTileNnz / kTileBlock per thread)
         constexpr int PER = kTileNnz / kTileBlock;
         Real xv[ PER ];
#pragma unroll
         for( int j = 0; j < PER; j++ ) {
            const int i = threadIdx.x + j * kTileBlock;
            xv[ j ] = i < len ? __ldg( x + c[ i ] ) : Real( 0 );
         }
#pragma unroll
         for( int j = 0; j < PER; j++ ) {
            const int i = threadIdx.x + j * kTileBlock;
            if( i < len )
               p[ i ] = p[ i ] * xv[ j ];
         }
      }
      __syncthreads();
      const int r0 = __ldg( tile_rows + t ), r1 = __ldg( tile_rows + t + 1 );
      if( r1 > r0 ) {
         const int mean = (int) ( ( (int64_t) __ldg( off + r1 ) - __ldg( off + r0 ) ) / ( r1 - r0 ) );
         if( mean <= 4 )
            tma_rows< Real, 1, Sink >( p, off, col, val, x, r0, r1, w0, len, sink, acc.v );
         else if( mean <= 12 )
            tma_rows< Real, 2, Sink >( p, off, col, val, x, r0, r1, w0, len, sink, acc.v );
         else if( mean <= 32 )
            tma_rows< Real, 4, Sink >( p, off, col, val, x, r0, r1, w0, len, sink, acc.v );
         else if( mean <= 96 )
            tma_rows< Real, 8, Sink >( p, off, col, val, x, r0, r1, w0, len, sink, acc.v );
         else if( mean <= 256 )
            tma_rows< Real, 16, Sink >( p, off, col, val, x, r0, r1, w0, len, sink, acc.v );
         else
            tma_rows< Real, 32, Sink >( p, off, col, val, x, r0, r1, w0, len, sink, acc.v );
      }
      // every thread is done with stage s; order its generic-proxy accesses of
      // the stage before the bulk copy that refills it
      fence_proxy_async_smem();
      __syncthreads();
      if( threadIdx.x == 0 )
         issue( k + kTmaStages );
   }
   if( failed ) {
      // a copy never completed: record it, then wait (bounded) for this CTA's
      // copies still in flight before leaving
      if( threadIdx.x == 0 ) {
         atomicExch( err, 1 );
         for( int j = k; j < k + kTmaStages && blockIdx.x + (int64_t) j * gridDim.x < ntiles; j++ )
            mbar_wait_bounded( bar + ( j % kTmaStages ), ( j / kTmaStages ) & 1 );
      }
      __syncthreads();
   }
   spmv_epilogue< Sink, kTileBlock >( sink, acc.v, rs );
}

// ---------------------------------------------------------------------------
// Ellpack (ColumnMajor): one thread per row; element k of row r sits at
// r + alignedSize*k, so consecutive threads read consecutive slots.
template< typename Real, class Sink >
__global__ void __launch_bounds__( kSpmvBlock )
ellpack_kernel( const int32_t* __restrict__ col, const Real* __restrict__ val, int32_t segmentSize, int32_t alignedSize,
                const Real* __restrict__ x, int32_t row_begin, int32_t row_end, Sink sink, RedScratch rs )
{
   if( sink.skip() )
      return;  // uniform over the grid: the solve this launch belongs to is finished
   AccOf< Sink > acc{};
   for( int64_t r = row_begin + blockIdx.x * (int64_t) kSpmvBlock + threadIdx.x; r < row_end;
        r += (int64_t) gridDim.x * kSpmvBlock ) {
      // every slot of the row is read (padding sits inside the allocation and
      // contributes 0), so the loads of all iterations are independent
      Real s = 0;
      int64_t g = r;
#pragma unroll 4
      for( int k = 0; k < segmentSize; k++, g += alignedSize ) {
         const int c = ld_stream( col + g );
         const Real v = ld_stream( val + g );
         if( c >= 0 )
            s += v * __ldg( x + c );
      }
      sink.put( (int) r, s, acc.v );
   }
   spmv_epilogue< Sink, kSpmvBlock >( sink, acc.v, rs );
}

// ---------------------------------------------------------------------------
// SlicedEllpack (ColumnMajor, slice 32): one thread per row; a warp covers one
// slice and reads 32 consecutive slots per step.
template< typename Real, class Sink >
__global__ void __launch_bounds__( kSpmvBlock )
sliced_kernel( const int32_t* __restrict__ col, const Real* __restrict__ val, const int32_t* __restrict__ sliceOffsets,
               const Real* __restrict__ x, int32_t row_begin, int32_t row_end, Sink sink, RedScratch rs )
{
   if( sink.skip() )
      return;  // uniform over the grid: the solve this launch belongs to is finished
   AccOf< Sink > acc{};
   for( int64_t r = row_begin + blockIdx.x * (int64_t) kSpmvBlock + threadIdx.x; r < row_end;
        r += (int64_t) gridDim.x * kSpmvBlock ) {
      const int slice = (int) ( r / kSliceSize );
      const int b = __ldg( sliceOffsets + slice ) + (int) ( r % kSliceSize );
      const int e = __ldg( sliceOffsets + slice + 1 );
      Real s = 0;
#pragma unroll 4
      for( int g = b; g < e; g += kSliceSize ) {
         const int c = ld_stream( col + g );
         const Real v = ld_stream( val + g );
         if( c >= 0 )
            s += v * __ldg( x + c );
      }
      sink.put( (int) r, s, acc.v );
   }
   spmv_epilogue< Sink, kSpmvBlock >( sink, acc.v, rs );
}

// ---------------------------------------------------------------------------
// ChunkedEllpack (ColumnMajor): one block of 256 threads per slice, one
// thread per chunk; chunk sums are combined per row in chunk order.
template< typename Real, class Sink >
__global__ void __launch_bounds__( kChunksInSlice )
chunked_kernel( const int32_t* __restrict__ col, const Real* __restrict__ val, const ChunkSlice* __restrict__ slices,
                const int32_t* __restrict__ rowToChunk, const int32_t* __restrict__ rowToSlice,
                const Real* __restrict__ x, int32_t row_begin, int32_t row_end, Sink sink, RedScratch rs )
{
   __shared__ Real part[ kChunksInSlice ];
   if( sink.skip() )
      return;  // uniform over the grid: the solve this launch belongs to is finished
   AccOf< Sink > acc{};
   const int s_first = __ldg( rowToSlice + row_begin );
   const int s_last = __ldg( rowToSlice + row_end - 1 );
   for( int sidx = s_first + blockIdx.x; sidx <= s_last; sidx += gridDim.x ) {
      const ChunkSlice sl = slices[ sidx ];
      Real s = 0;
      int64_t g = (int64_t) sl.pointer + threadIdx.x;
#pragma unroll 4
      for( int o = 0; o < sl.chunkSize; o++, g += kChunksInSlice ) {
         const int c = ld_stream( col + g );
         const Real v = ld_stream( val + g );
         if( c >= 0 )
            s += v * __ldg( x + c );
      }
      part[ threadIdx.x ] = s;
      __syncthreads();
      if( (int) threadIdx.x < sl.size ) {
         const int row = sl.firstSegment + threadIdx.x;
         int ch = threadIdx.x == 0 ? 0 : __ldg( rowToChunk + row - 1 );
         const int last = __ldg( rowToChunk + row );
         Real r = 0;
         for( ; ch < last; ch++ )
            r += part[ ch ];
         if( row >= row_begin && row < row_end )
            sink.put( row, r, acc.v );
      }
      __syncthreads();
   }
   spmv_epilogue< Sink, kChunksInSlice >( sink, acc.v, rs );
}

// ---------------------------------------------------------------------------
// BiEllpack (ColumnMajor, warp 32): one thread per row; the row's strip rank
// selects how many groups it spans (detail/BiEllpack.h:48-64) and group g
// stores element i of rank p at groupPointer + p + i*(32>>g).
template< typename Real, class Sink >
__global__ void __launch_bounds__( kSpmvBlock )
biell_kernel( const int32_t* __restrict__ col, const Real* __restrict__ val, const int32_t* __restrict__ rowPerm,
              const int32_t* __restrict__ groupPointers, const Real* __restrict__ x, int32_t row_begin,
              int32_t row_end, Sink sink, RedScratch rs )
{
   if( sink.skip() )
      return;  // uniform over the grid: the solve this launch belongs to is finished
   AccOf< Sink > acc{};
   for( int64_t r = row_begin + blockIdx.x * (int64_t) kSpmvBlock + threadIdx.x; r < row_end;
        r += (int64_t) gridDim.x * kSpmvBlock ) {
      const int strip = (int) ( r / kBiWarp );
      const int gb = strip * kBiGroups;
      const int p = __ldg( rowPerm + r ) - strip * kBiWarp;
      const int groups = p == 0 ? 6 : ( p < 2 ? 5 : ( p < 4 ? 4 : ( p < 8 ? 3 : ( p < 16 ? 2 : 1 ) ) ) );
      Real s = 0;
      int h = kBiWarp;
      int gp = __ldg( groupPointers + gb );
      for( int k = 0; k < groups; k++ ) {
         const int gn = __ldg( groupPointers + gb + k + 1 );
         const int w = ( gn - gp ) / h;
         int64_t g = (int64_t) gp + p;
#pragma unroll 4
         for( int i = 0; i < w; i++, g += h ) {
            const int c = ld_stream( col + g );
            const Real v = ld_stream( val + g );
            if( c >= 0 )
               s += v * __ldg( x + c );
         }
         gp = gn;
         h >>= 1;
      }
      sink.put( (int) r, s, acc.v );
   }
   spmv_epilogue< Sink, kSpmvBlock >( sink, acc.v, rs );
}

// ---------------------------------------------------------------------------
// Dispatch over layouts for a given sink.
inline int
spmv_grid( int64_t threads_needed, int block )
{
   const int64_t g = ( threads_needed + block - 1 ) / block;
   const int64_t cap = (int64_t) num_sms() * 16;
   return (int) std::max< int64_t >( 1, std::min< int64_t >( g, std::min< int64_t >( cap, kMaxReduceGrid ) ) );
}

template< typename Real, class Sink >
inline b2s_status
spmv_dispatch( const b2s_matrix_t* A, const Real* values, const Real* x, int32_t rb, int32_t re, const Sink& sink,
               RedScratch rs, cudaStream_t s )
{
   const int32_t* col = A->columns.as< int32_t >();
   const int64_t nr = (int64_t) re - rb;
   if( nr <= 0 )
      return B2S_OK;
   switch( A->format ) {
      case B2S_CSR: {
         const int32_t* off = A->offsets.as< int32_t >();
         if( A->csr_kernel == B2S_CSR_ADAPTIVE && rb == 0 && re == A->rows ) {
            constexpr size_t smem = tma_smem_bytes< Real >();
            static int attr_set[ 64 ] = { 0 };
            const int dev = current_device();
            if( dev >= 0 && dev < 64 && ! attr_set[ dev ] ) {
               B2S_TRY_CUDA( cudaFuncSetAttribute( csr_tma_kernel< Real, Sink >,
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem ) );
               attr_set[ dev ] = 1;
            }
            const int per_sm = (int) std::min< size_t >( 8, ( 227u * 1024u ) / ( smem + 1024u ) );
            const int grid = (int) std::max< int64_t >(
               1, std::min< int64_t >( A->n_blocks,
                                       std::min< int64_t >( (int64_t) num_sms() * per_sm, kMaxReduceGrid ) ) );
            csr_tma_kernel< Real, Sink ><<< grid, kTileBlock, smem, s >>>(
               off, col, values, x, A->csr_blocks.as< int32_t >(), A->n_blocks, A->nnz, sink, rs,
               A->status.as< int >() );
            break;
         }
         const int tpr = A->tpr;
         const int grid = spmv_grid( nr * tpr, kSpmvBlock );
#define B2S_CSR_CASE( T )                                                                                   \
   case T:                                                                                                  \
      csr_vector_kernel< Real, T, Sink ><<< grid, kSpmvBlock, 0, s >>>( off, col, values, x, rb, re, sink, rs ); \
      break;
         switch( tpr ) {
            B2S_CSR_CASE( 1 )
            B2S_CSR_CASE( 2 )
            B2S_CSR_CASE( 4 )
            B2S_CSR_CASE( 8 )
            B2S_CSR_CASE( 16 )
            B2S_CSR_CASE( 32 )
            default:
               set_error( "bad threads per row %d", tpr );
               return B2S_INVALID_ARG;
         }
#undef B2S_CSR_CASE
         break;
      }
      case B2S_ELLPACK:
         ellpack_kernel< Real, Sink ><<< spmv_grid( nr, kSpmvBlock ), kSpmvBlock, 0, s >>>(
            col, values, A->segmentSize, A->alignedSize, x, rb, re, sink, rs );
         break;
      case B2S_SLICED_ELLPACK:
         sliced_kernel< Real, Sink ><<< spmv_grid( nr, kSpmvBlock ), kSpmvBlock, 0, s >>>(
            col, values, A->sliceOffsets.as< int32_t >(), x, rb, re, sink, rs );
         break;
      case B2S_CHUNKED_ELLPACK: {
         const int grid = (int) std::min< int64_t >( std::max( A->numberOfSlices, 1 ),
                                                     std::min< int64_t >( (int64_t) num_sms() * 8, kMaxReduceGrid ) );
         chunked_kernel< Real, Sink ><<< grid, kChunksInSlice, 0, s >>>(
            col, values, A->cslices.as< ChunkSlice >(), A->rowToChunk.as< int32_t >(), A->rowToSlice.as< int32_t >(), x,
            rb, re, sink, rs );
         break;
      }
      case B2S_BIELLPACK:
         biell_kernel< Real, Sink ><<< spmv_grid( nr, kSpmvBlock ), kSpmvBlock, 0, s >>>(
            col, values, A->rowPerm.as< int32_t >(), A->groupPointers.as< int32_t >(), x, rb, re, sink, rs );
         break;
      default:
         set_error( "unknown format" );
         return B2S_INVALID_ARG;
   }
   B2S_TRY_CUDA( cudaGetLastError() );
   return B2S_OK;
}

}  // namespace b2s
