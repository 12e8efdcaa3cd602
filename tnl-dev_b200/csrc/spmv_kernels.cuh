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

#include <type_traits>

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
// CSR, nnz-balanced warp windows (the "adaptive" kernel; row binning without
// a host pass). Window w is the range [w*WIN, (w+1)*WIN) of the nonzero
// arrays, WIN = 32*E (E = 8 for FP64, 12 for FP32); it owns the rows whose
// first nonzero lies in it (win_rows[w] = first such row, found by binary
// search when the matrix is built). One warp per window:
//   1. lane l owns elements l, l+32, l+64, ... of the window: coalesced
//      streaming loads of columns and values (evict-first in L2, so x stays
//      resident) and gathers of x that cover a few consecutive rows per
//      instruction; the offsets of the window's first 32 rows are loaded
//      alongside;
//   2. the products are parked in the warp's slice of shared memory (one
//      conflict-free store per element);
//   3. every owned row is summed from shared memory by one lane in the row's
//      element order (TNL's CSRScalar order, CSRScalarKernel.hpp); the part of
//      a row that runs past the window is read from global memory. Rows longer
//      than kCsrLongRow, or running far past the window, are summed by the
//      whole warp instead.
// PIPE (matrices whose rows are all short): the next window's columns and row
// range are loaded while the current window is summed, so a window waits on
// one gather round trip only.
// Grid: resident CTAs only, striding over the windows.
constexpr int kCsrWarpsPerCta = 4;
constexpr int kCsrBlock = 32 * kCsrWarpsPerCta;
constexpr int kLongOverhang = 8;

template< typename Real >
struct CsrWin
{
   static constexpr int E = sizeof( Real ) == 8 ? kWinElemsF64 : kWinElemsF32;
   static constexpr int W = 32 * E;
   static constexpr int table = sizeof( Real ) == 8 ? 0 : 1;
};

// L2 policy for data read exactly once per product
__device__ __forceinline__ uint64_t
l2_evict_first()
{
   uint64_t pol;
   asm( "createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"( pol ) );
   return pol;
}

// streaming loads that bypass L1 and leave L2 first in line for eviction
__device__ __forceinline__ int
ld_stream_ef( const int32_t* p, uint64_t pol )
{
   int v;
   asm( "ld.global.nc.L1::no_allocate.L2::cache_hint.b32 %0, [%1], %2;" : "=r"( v ) : "l"( p ), "l"( pol ) );
   return v;
}
__device__ __forceinline__ float
ld_stream_ef( const float* p, uint64_t pol )
{
   float v;
   asm( "ld.global.nc.L1::no_allocate.L2::cache_hint.f32 %0, [%1], %2;" : "=f"( v ) : "l"( p ), "l"( pol ) );
   return v;
}
__device__ __forceinline__ double
ld_stream_ef( const double* p, uint64_t pol )
{
   double v;
   asm( "ld.global.nc.L1::no_allocate.L2::cache_hint.f64 %0, [%1], %2;" : "=d"( v ) : "l"( p ), "l"( pol ) );
   return v;
}

// 8 consecutive elements, 32-byte aligned, as 256-bit loads that bypass L1
__device__ __forceinline__ void
ld_stream8( const int32_t* p, int ( &c )[ 8 ], uint64_t pol )
{
   asm( "ld.global.nc.L1::no_allocate.L2::cache_hint.v8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8], %9;"
        : "=r"( c[ 0 ] ), "=r"( c[ 1 ] ), "=r"( c[ 2 ] ), "=r"( c[ 3 ] ), "=r"( c[ 4 ] ), "=r"( c[ 5 ] ), "=r"( c[ 6 ] ),
          "=r"( c[ 7 ] )
        : "l"( p ), "l"( pol ) );
}
__device__ __forceinline__ void
ld_stream8( const float* p, float ( &v )[ 8 ], uint64_t pol )
{
   asm( "ld.global.nc.L1::no_allocate.L2::cache_hint.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8], %9;"
        : "=f"( v[ 0 ] ), "=f"( v[ 1 ] ), "=f"( v[ 2 ] ), "=f"( v[ 3 ] ), "=f"( v[ 4 ] ), "=f"( v[ 5 ] ), "=f"( v[ 6 ] ),
          "=f"( v[ 7 ] )
        : "l"( p ), "l"( pol ) );
}
__device__ __forceinline__ void
ld_stream8( const double* p, double ( &v )[ 8 ], uint64_t pol )
{
   asm( "ld.global.nc.L1::no_allocate.L2::cache_hint.v4.f64 {%0,%1,%2,%3}, [%4], %5;"
        : "=d"( v[ 0 ] ), "=d"( v[ 1 ] ), "=d"( v[ 2 ] ), "=d"( v[ 3 ] )
        : "l"( p ), "l"( pol ) );
   asm( "ld.global.nc.L1::no_allocate.L2::cache_hint.v4.f64 {%0,%1,%2,%3}, [%4], %5;"
        : "=d"( v[ 4 ] ), "=d"( v[ 5 ] ), "=d"( v[ 6 ] ), "=d"( v[ 7 ] )
        : "l"( p + 4 ), "l"( pol ) );
}

// Sum of value*x over the 8 elements [q, q+8) clipped to [q, end), loaded
// with 256-bit loads when all 8 are inside (q is 8-aligned).
template< typename Real >
__device__ __forceinline__ Real
dot8( const int32_t* __restrict__ col, const Real* __restrict__ val, const Real* __restrict__ x, int64_t q,
      int64_t end, uint64_t pol )
{
   Real t = 0;
   if( q + 8 <= end ) {
      int c[ 8 ];
      Real v[ 8 ];
      ld_stream8( col + q, c, pol );
      ld_stream8( val + q, v, pol );
      Real xv[ 8 ];
#pragma unroll
      for( int i = 0; i < 8; i++ )
         xv[ i ] = __ldg( x + c[ i ] );
#pragma unroll
      for( int i = 0; i < 8; i++ )
         t += v[ i ] * xv[ i ];
   }
   else {
      for( int64_t k = q; k < end; k++ )
         t += __ldg( val + k ) * __ldg( x + __ldg( col + k ) );
   }
   return t;
}

// resident blocks per SM asked of the compiler: the variant for matrices with
// long rows fits 10 (48 registers, no spills), the pipelined one 8
#ifndef B2S_WARP_MIN_BLOCKS
#define B2S_WARP_MIN_BLOCKS 10
#endif
template< typename Real, bool PIPE, class Sink >
__global__ void __launch_bounds__( kCsrBlock, PIPE ? 8 : B2S_WARP_MIN_BLOCKS )
csr_warp_kernel( const int32_t* __restrict__ off, const int32_t* __restrict__ col, const Real* __restrict__ val,
                 const Real* __restrict__ x, const int32_t* __restrict__ win_rows, int64_t nwin, int64_t nnz, Sink sink,
                 RedScratch rs )
{
   constexpr int E = CsrWin< Real >::E;
   constexpr int W = CsrWin< Real >::W;
   __shared__ __align__( 16 ) Real prod[ kCsrWarpsPerCta ][ W ];
   if( sink.skip() )
      return;  // uniform over the grid: the solve this launch belongs to is finished
   AccOf< Sink > acc{};
   const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
   Real* p = prod[ warp ];
   const uint64_t pol = l2_evict_first();
   const int64_t stride = (int64_t) gridDim.x * kCsrWarpsPerCta;
   int64_t w = (int64_t) blockIdx.x * kCsrWarpsPerCta + warp;
   // columns of window ww (zeros outside the matrix)
   auto load_cols = [ & ]( int64_t ww, int( &cc )[ E ] )
   {
      const int64_t b0 = ww * W;
      if( ww < nwin && b0 + W <= nnz ) {
#pragma unroll
         for( int i = 0; i < E; i++ )
            cc[ i ] = ld_stream_ef( col + b0 + lane + 32 * i, pol );
      }
      else {
#pragma unroll
         for( int i = 0; i < E; i++ ) {
            const int64_t k = b0 + lane + 32 * i;
            cc[ i ] = ( ww < nwin && k < nnz ) ? __ldcs( col + k ) : 0;
         }
      }
   };
   int c[ E ];
   int r0 = 0, r1 = 0;
   if( PIPE && w < nwin ) {
      load_cols( w, c );
      r0 = __ldg( win_rows + w );
      r1 = __ldg( win_rows + w + 1 );
   }
   for( ; w < nwin; w += stride ) {
      if( ! PIPE ) {
         load_cols( w, c );
         r0 = __ldg( win_rows + w );
         r1 = __ldg( win_rows + w + 1 );
      }
      const int64_t w0 = w * W, wend = w0 + W;
      // 1. values and gathers of this window, offsets of its first 32 rows
      Real v[ E ], xv[ E ];
      if( wend <= nnz ) {
#pragma unroll
         for( int i = 0; i < E; i++ ) {
            v[ i ] = ld_stream_ef( val + w0 + lane + 32 * i, pol );
            xv[ i ] = __ldg( x + c[ i ] );
         }
      }
      else {
#pragma unroll
         for( int i = 0; i < E; i++ ) {
            const int64_t k = w0 + lane + 32 * i;
            v[ i ] = k < nnz ? __ldcs( val + k ) : Real( 0 );
            xv[ i ] = k < nnz ? __ldg( x + c[ i ] ) : Real( 0 );
         }
      }
      const int ob = __ldg( off + min( r0 + lane, r1 ) );
      const int ob32 = ( lane == 31 && r0 + 32 <= r1 ) ? __ldg( off + r0 + 32 ) : 0;
      int r0n = 0, r1n = 0;
      if constexpr( PIPE ) {
         // the next window's columns and rows go out before this one is summed
         const int64_t wn = w + stride;
         if( wn < nwin ) {
            r0n = __ldg( win_rows + wn );
            r1n = __ldg( win_rows + wn + 1 );
         }
         load_cols( wn, c );
      }
      // 2. products, one conflict-free store each
#pragma unroll
      for( int i = 0; i < E; i++ )
         p[ lane + 32 * i ] = v[ i ] * xv[ i ];
      __syncwarp();
      // 3. the owned rows, 32 at a time
      for( int rb = r0; rb < r1; rb += 32 ) {
         const int r = rb + lane;
         const bool active = r < r1;
         int b, e;
         if( rb == r0 ) {
            b = ob;
            e = __shfl_down_sync( 0xffffffffu, ob, 1 );
            if( lane == 31 )
               e = ob32;
         }
         else {
            b = __ldg( off + min( r, r1 ) );
            e = __shfl_down_sync( 0xffffffffu, b, 1 );
            if( lane == 31 && active )
               e = __ldg( off + r + 1 );
         }
         bool coop = false;
         if( active ) {
            coop = e - b > kCsrLongRow || (int64_t) e - wend > kLongOverhang;
            if( ! coop ) {
               Real s = 0;
               const int le = (int) ( min( (int64_t) e, wend ) - w0 );
               for( int k = (int) ( b - w0 ); k < le; k++ )
                  s += p[ k ];
               for( int64_t k = wend; k < e; k++ )
                  s += __ldg( val + k ) * __ldg( x + __ldg( col + k ) );
               sink.put( r, s, acc.v );
            }
         }
         // long rows: the whole warp, one row at a time
         unsigned cm = __ballot_sync( 0xffffffffu, coop );
         while( cm ) {
            const int src = __ffs( cm ) - 1;
            cm &= cm - 1;
            const int cb = __shfl_sync( 0xffffffffu, b, src ), ce = __shfl_sync( 0xffffffffu, e, src );
            Real t = 0;
            const int le = (int) ( min( (int64_t) ce, wend ) - w0 );
            for( int k = (int) ( cb - w0 ) + lane; k < le; k += 32 )
               t += p[ k ];
            for( int64_t base = wend; base < ce; base += 256 )
               t += dot8< Real >( col, val, x, base + 8 * lane, ce, pol );
            t = warp_sum( t );
            if( lane == src )
               sink.put( rb + src, t, acc.v );
         }
      }
      __syncwarp();  // the slice is refilled by the next window
      if constexpr( PIPE ) {
         r0 = r0n;
         r1 = r1n;
      }
   }
   spmv_epilogue< Sink, kCsrBlock >( sink, acc.v, rs );
}

// ---------------------------------------------------------------------------
// CSR, groups of 32 consecutive rows staged in shared memory (matrices whose
// every group of 32 rows holds at most kCsrGroupCap nonzeros — stencils and
// other short, even rows; the window kernel above takes the rest).
// One warp per group, persistent over the groups, csr_group_stages() shared
// buffers per warp:
//   * the group's columns and values are copied to shared memory by cp.async
//     in 16-byte chunks (coalesced, no registers held) while the earlier
//     groups are summed; the row offsets run one more group ahead;
//   * lane l sums row 32g + l from shared memory in the row's element order
//     (TNL's CSRScalar order, CSRScalarKernel.hpp), one rounded product per
//     element. Neighbouring lanes hold neighbouring rows, so for banded
//     matrices the gathers of x at one element position are contiguous.
// Chunks are aligned down/up to 16 bytes: up to 12 bytes past the last
// nonzero are read (every device allocation carries >= 256 bytes of padding).
constexpr int kCsrGroupRows = 32;
constexpr int kCsrGroupWarps = 4;
constexpr int kCsrGroupBlock = 32 * kCsrGroupWarps;

__device__ __forceinline__ void
cp_async16( void* dst, const void* src, uint64_t pol )
{
   const unsigned d = (unsigned) __cvta_generic_to_shared( dst );
   asm volatile( "cp.async.cg.shared.global.L2::cache_hint [%0], [%1], 16, %2;" ::"r"( d ), "l"( src ), "l"( pol )
                 : "memory" );
}
__device__ __forceinline__ void
cp_async_commit()
{
   asm volatile( "cp.async.commit_group;" ::: "memory" );
}
template< int N >
__device__ __forceinline__ void
cp_async_wait()
{
   asm volatile( "cp.async.wait_group %0;" ::"n"( N ) : "memory" );
}

// a product rounded on its own (no fused multiply-add), as a serial host loop computes it
__device__ __forceinline__ double
mul_rn( double a, double b )
{
   return __dmul_rn( a, b );
}
__device__ __forceinline__ float
mul_rn( float a, float b )
{
   return __fmul_rn( a, b );
}

// Stages of the copy pipeline. Two for both value types: a third FP32 stage
// (as many bytes in flight per warp as FP64) measured 9 % slower on the 128^3
// Laplacian (0.644 against 0.705 of the copy bandwidth).
template< typename Real >
constexpr int csr_group_stages()
{
   return 2;
}

// RPL rows per lane: groups of 32 RPL rows (lane l sums rows l, l + 32, ...)
// with at most RPL * kCsrGroupCap nonzeros, which every such group of a
// matrix whose 32-row groups fit the cap satisfies.
template< typename Real, int RPL, class Sink >
__global__ void __launch_bounds__( kCsrGroupBlock, 8 / RPL )
csr_group_kernel( const int32_t* __restrict__ off, const int32_t* __restrict__ col, const Real* __restrict__ val,
                  const Real* __restrict__ x, int32_t row_begin, int32_t row_end, Sink sink, RedScratch rs )
{
   constexpr int VPC = 16 / sizeof( Real );    // values per 16-byte chunk
   constexpr int GR = kCsrGroupRows * RPL;     // rows per group
   constexpr int SC = kCsrGroupCap * RPL + 8;  // room for the alignment slack
   constexpr int NS = csr_group_stages< Real >();
   __shared__ __align__( 16 ) int32_t scol[ kCsrGroupWarps ][ NS ][ SC ];
   __shared__ __align__( 16 ) Real sval[ kCsrGroupWarps ][ NS ][ SC ];
   if( sink.skip() )
      return;  // uniform over the grid: the solve this launch belongs to is finished
   AccOf< Sink > acc{};
   const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
   const uint64_t pol = l2_evict_first();
   // groups of GR rows from row_begin (a multiple of GR, so they are unions of
   // the 32-row groups the nonzero cap was checked on)
   const int64_t ngroups = ( (int64_t) row_end - row_begin + GR - 1 ) / GR;
   const int64_t stride = (int64_t) gridDim.x * kCsrGroupWarps;
   int64_t g = (int64_t) blockIdx.x * kCsrGroupWarps + warp;
   // lo[j] = off[row], hi[j] = off[row + 1] of this lane's row j in group gg
   auto load_off = [ & ]( int64_t gg, int( &lo )[ RPL ], int( &hi )[ RPL ] )
   {
#pragma unroll
      for( int j = 0; j < RPL; j++ ) {
         lo[ j ] = hi[ j ] = 0;
         if( gg < ngroups ) {
            const int64_t r = row_begin + gg * GR + 32 * j + lane;
            lo[ j ] = __ldg( off + ( r < row_end ? r : row_end ) );
            hi[ j ] = __ldg( off + ( r + 1 < row_end ? r + 1 : row_end ) );
         }
      }
   };
   auto stage = [ & ]( int64_t gg, const int( &lo )[ RPL ], const int( &hi )[ RPL ], int buf )
   {
      if( gg < ngroups ) {
         const int base = __shfl_sync( 0xffffffffu, lo[ 0 ], 0 );
         const int end = __shfl_sync( 0xffffffffu, hi[ RPL - 1 ], 31 );
         const int a0 = base & ~3, a1 = ( end + 3 ) & ~3;
         for( int q = 4 * lane; q < a1 - a0; q += 128 )
            cp_async16( &scol[ warp ][ buf ][ q ], col + a0 + q, pol );
         const int v0 = base & ~( VPC - 1 ), v1 = ( end + VPC - 1 ) & ~( VPC - 1 );
         for( int q = VPC * lane; q < v1 - v0; q += 32 * VPC )
            cp_async16( &sval[ warp ][ buf ][ q ], val + v0 + q, pol );
      }
      cp_async_commit();  // an empty group past the end keeps the wait counts uniform
   };
   // offsets of groups g, g + stride, ..., g + (NS - 1) stride; the copies of
   // the first NS - 1 of them are in flight when the loop starts
   int olo[ NS ][ RPL ], ohi[ NS ][ RPL ];
#pragma unroll
   for( int i = 0; i < NS; i++ )
      load_off( g + i * stride, olo[ i ], ohi[ i ] );
#pragma unroll
   for( int i = 0; i < NS - 1; i++ )
      stage( g + i * stride, olo[ i ], ohi[ i ], i );
   int buf = 0;
   for( ; g < ngroups; g += stride ) {
      stage( g + ( NS - 1 ) * stride, olo[ NS - 1 ], ohi[ NS - 1 ], ( buf + NS - 1 ) % NS );
      int nlo[ RPL ], nhi[ RPL ];
      load_off( g + NS * stride, nlo, nhi );
      cp_async_wait< NS - 1 >();  // this group's copies have landed
      __syncwarp();
      const int base = __shfl_sync( 0xffffffffu, olo[ 0 ][ 0 ], 0 );
      const int32_t* sc = scol[ warp ][ buf ] - ( base & ~3 );
      const Real* sv = sval[ warp ][ buf ] - ( base & ~( VPC - 1 ) );
#pragma unroll
      for( int j = 0; j < RPL; j++ ) {
         const int lo = olo[ 0 ][ j ], hi = ohi[ 0 ][ j ];
         Real sum = 0;
         for( int k = lo; k < hi; k += 8 ) {
            Real v[ 8 ], xv[ 8 ];
#pragma unroll
            for( int i = 0; i < 8; i++ ) {
               const int q = k + i < hi ? k + i : k;  // past the row: a repeated in-row element, not summed
               v[ i ] = sv[ q ];
               xv[ i ] = __ldg( x + sc[ q ] );
            }
#pragma unroll
            for( int i = 0; i < 8; i++ )
               if( k + i < hi )
                  sum = sum + mul_rn( v[ i ], xv[ i ] );
         }
         const int64_t r = row_begin + g * GR + 32 * j + lane;
         if( r < row_end )
            sink.put( (int) r, sum, acc.v );
      }
      __syncwarp();  // the buffer is refilled NS groups later
#pragma unroll
      for( int i = 0; i < NS - 1; i++ )
#pragma unroll
         for( int j = 0; j < RPL; j++ ) {
            olo[ i ][ j ] = olo[ i + 1 ][ j ];
            ohi[ i ][ j ] = ohi[ i + 1 ][ j ];
         }
#pragma unroll
      for( int j = 0; j < RPL; j++ ) {
         olo[ NS - 1 ][ j ] = nlo[ j ];
         ohi[ NS - 1 ][ j ] = nhi[ j ];
      }
      buf = buf + 1 == NS ? 0 : buf + 1;
   }
   cp_async_wait< 0 >();
   spmv_epilogue< Sink, kCsrGroupBlock >( sink, acc.v, rs );
}

// ---------------------------------------------------------------------------
// One slot of a padded layout into s. With SKIP the value of a padding slot
// (column -1, value 0) is never read: where padding dominates (irregular rows
// in Ellpack-like layouts) that removes most of the value bytes. Without it
// the value load is issued alongside the column load (no dependency), which
// is faster when there is little padding.
template< typename Real, bool SKIP >
__device__ __forceinline__ void
slot_fma( const int32_t* __restrict__ col, const Real* __restrict__ val, const Real* __restrict__ x, int64_t g, Real& s )
{
   const int c = ld_stream( col + g );
   if constexpr( SKIP ) {
      if( c >= 0 )
         s += ld_stream( val + g ) * __ldg( x + c );
   }
   else {
      const Real v = ld_stream( val + g );
      if( c >= 0 )
         s += v * __ldg( x + c );
   }
}

// Two adjacent rows r (even) and r + 1: in the ColumnMajor layouts their slots
// k are neighbours, so one 8-byte column load and one two-element value load
// serve both rows; each row's sum keeps its slot order (same results as one
// row per thread).
template< typename Real >
struct PairOf;
template<>
struct PairOf< float >
{
   using type = float2;
};
template<>
struct PairOf< double >
{
   using type = double2;
};

template< typename Real, bool SKIP >
__device__ __forceinline__ void
slot_fma2( const int32_t* __restrict__ col, const Real* __restrict__ val, const Real* __restrict__ x, int64_t g,
           Real& s0, Real& s1 )
{
   using P = typename PairOf< Real >::type;
   const int2 c = ld_stream( reinterpret_cast< const int2* >( col + g ) );
   if constexpr( SKIP ) {
      if( c.x >= 0 || c.y >= 0 ) {
         const P v = ld_stream( reinterpret_cast< const P* >( val + g ) );
         if( c.x >= 0 )
            s0 += v.x * __ldg( x + c.x );
         if( c.y >= 0 )
            s1 += v.y * __ldg( x + c.y );
      }
   }
   else {
      const P v = ld_stream( reinterpret_cast< const P* >( val + g ) );
      if( c.x >= 0 )
         s0 += v.x * __ldg( x + c.x );
      if( c.y >= 0 )
         s1 += v.y * __ldg( x + c.y );
   }
}

// ---------------------------------------------------------------------------
// Ellpack (ColumnMajor): one thread per row; element k of row r sits at
// r + alignedSize*k, so consecutive threads read consecutive slots.
template< typename Real, bool SKIP, class Sink >
__global__ void __launch_bounds__( kSpmvBlock )
ellpack_kernel( const int32_t* __restrict__ col, const Real* __restrict__ val, int32_t segmentSize, int32_t alignedSize,
                const Real* __restrict__ x, int32_t row_begin, int32_t row_end, Sink sink, RedScratch rs )
{
   if( sink.skip() )
      return;  // uniform over the grid: the solve this launch belongs to is finished
   AccOf< Sink > acc{};
   for( int64_t r = row_begin + blockIdx.x * (int64_t) kSpmvBlock + threadIdx.x; r < row_end;
        r += (int64_t) gridDim.x * kSpmvBlock ) {
      // every slot of the row is visited (padding sits inside the allocation
      // and contributes nothing), so the loads of all iterations are independent
      Real s = 0;
      int64_t g = r;
#pragma unroll 4
      for( int k = 0; k < segmentSize; k++, g += alignedSize ) {
         slot_fma< Real, SKIP >( col, val, x, g, s );
      }
      sink.put( (int) r, s, acc.v );
   }
   spmv_epilogue< Sink, kSpmvBlock >( sink, acc.v, rs );
}

// Ellpack, two adjacent rows per thread (row_begin and alignedSize even: every
// pair load is aligned; the slots of row r + 1 exist up to alignedSize).
template< typename Real, bool SKIP, class Sink >
__global__ void __launch_bounds__( kSpmvBlock )
ellpack2_kernel( const int32_t* __restrict__ col, const Real* __restrict__ val, int32_t segmentSize,
                 int32_t alignedSize, const Real* __restrict__ x, int32_t row_begin, int32_t row_end, Sink sink,
                 RedScratch rs )
{
   if( sink.skip() )
      return;
   AccOf< Sink > acc{};
   for( int64_t r = row_begin + 2 * ( blockIdx.x * (int64_t) kSpmvBlock + threadIdx.x ); r < row_end;
        r += 2 * (int64_t) gridDim.x * kSpmvBlock ) {
      Real s0 = 0, s1 = 0;
      int64_t g = r;
#pragma unroll 4
      for( int k = 0; k < segmentSize; k++, g += alignedSize )
         slot_fma2< Real, SKIP >( col, val, x, g, s0, s1 );
      sink.put( (int) r, s0, acc.v );
      if( r + 1 < row_end )
         sink.put( (int) r + 1, s1, acc.v );
   }
   spmv_epilogue< Sink, kSpmvBlock >( sink, acc.v, rs );
}

// ---------------------------------------------------------------------------
// SlicedEllpack (ColumnMajor, slice S = 8, 16, 32 or 64): one thread per row;
// element k of row r sits at sliceOffset + r%S + S*k, so a warp reads
// 32/S runs of S consecutive slots per step (S >= 32: one run).
template< typename Real, int S, bool SKIP, class Sink >
__global__ void __launch_bounds__( kSpmvBlock )
sliced_kernel( const int32_t* __restrict__ col, const Real* __restrict__ val, const int32_t* __restrict__ sliceOffsets,
               const Real* __restrict__ x, int32_t row_begin, int32_t row_end, Sink sink, RedScratch rs )
{
   if( sink.skip() )
      return;  // uniform over the grid: the solve this launch belongs to is finished
   AccOf< Sink > acc{};
   for( int64_t r = row_begin + blockIdx.x * (int64_t) kSpmvBlock + threadIdx.x; r < row_end;
        r += (int64_t) gridDim.x * kSpmvBlock ) {
      const int slice = (int) ( r / S );
      const int b = __ldg( sliceOffsets + slice ) + (int) ( r % S );
      const int e = __ldg( sliceOffsets + slice + 1 );
      Real s = 0;
#pragma unroll 4
      for( int g = b; g < e; g += S ) {
         slot_fma< Real, SKIP >( col, val, x, g, s );
      }
      sink.put( (int) r, s, acc.v );
   }
   spmv_epilogue< Sink, kSpmvBlock >( sink, acc.v, rs );
}

// SlicedEllpack, two adjacent rows per thread (row_begin even): both rows lie in
// one slice (S even), slice offsets are multiples of S, so the pair loads are
// aligned; a slice holds the slots of all its S rows.
template< typename Real, int S, bool SKIP, class Sink >
__global__ void __launch_bounds__( kSpmvBlock )
sliced2_kernel( const int32_t* __restrict__ col, const Real* __restrict__ val, const int32_t* __restrict__ sliceOffsets,
                const Real* __restrict__ x, int32_t row_begin, int32_t row_end, Sink sink, RedScratch rs )
{
   if( sink.skip() )
      return;
   AccOf< Sink > acc{};
   for( int64_t r = row_begin + 2 * ( blockIdx.x * (int64_t) kSpmvBlock + threadIdx.x ); r < row_end;
        r += 2 * (int64_t) gridDim.x * kSpmvBlock ) {
      const int slice = (int) ( r / S );
      const int b = __ldg( sliceOffsets + slice ) + (int) ( r % S );
      const int e = __ldg( sliceOffsets + slice + 1 );
      Real s0 = 0, s1 = 0;
#pragma unroll 4
      for( int g = b; g < e; g += S )
         slot_fma2< Real, SKIP >( col, val, x, g, s0, s1 );
      sink.put( (int) r, s0, acc.v );
      if( r + 1 < row_end )
         sink.put( (int) r + 1, s1, acc.v );
   }
   spmv_epilogue< Sink, kSpmvBlock >( sink, acc.v, rs );
}

// FP32: four adjacent rows r (a multiple of 4) .. r + 3 per thread — one 16-byte
// column load and one 16-byte value load serve the four (the FP64 pairs move 16
// bytes of values per load too). Each row's sum keeps its slot order.
__device__ __forceinline__ void
slot_fma4( const int32_t* __restrict__ col, const float* __restrict__ val, const float* __restrict__ x, int64_t g,
           float ( &s )[ 4 ] )
{
   const int4 c = ld_stream( reinterpret_cast< const int4* >( col + g ) );
   const float4 v = ld_stream( reinterpret_cast< const float4* >( val + g ) );
   if( c.x >= 0 )
      s[ 0 ] += v.x * __ldg( x + c.x );
   if( c.y >= 0 )
      s[ 1 ] += v.y * __ldg( x + c.y );
   if( c.z >= 0 )
      s[ 2 ] += v.z * __ldg( x + c.z );
   if( c.w >= 0 )
      s[ 3 ] += v.w * __ldg( x + c.w );
}

// FP64: the four values as one 32-byte load (g a multiple of 4). The load
// needs `val + g` on a 32-byte boundary (the column load: `col + g` on 16):
// spmv_dispatch chooses the quad kernels only for base pointers aligned so
// (every array the library allocates starts on a 256-byte boundary).
__device__ __forceinline__ void
slot_fma4( const int32_t* __restrict__ col, const double* __restrict__ val, const double* __restrict__ x, int64_t g,
           double ( &s )[ 4 ] )
{
   const int4 c = ld_stream( reinterpret_cast< const int4* >( col + g ) );
   double v0, v1, v2, v3;
   asm( "ld.global.nc.L1::no_allocate.v4.f64 {%0,%1,%2,%3}, [%4];"
        : "=d"( v0 ), "=d"( v1 ), "=d"( v2 ), "=d"( v3 )
        : "l"( val + g ) );
   if( c.x >= 0 )
      s[ 0 ] += v0 * __ldg( x + c.x );
   if( c.y >= 0 )
      s[ 1 ] += v1 * __ldg( x + c.y );
   if( c.z >= 0 )
      s[ 2 ] += v2 * __ldg( x + c.z );
   if( c.w >= 0 )
      s[ 3 ] += v3 * __ldg( x + c.w );
}

// Multidiagonal (MultidiagonalMatrixView.hpp:488-528, ColumnMajor as on
// Devices::Cuda): no column indices — element d of row r is A(r, r + offsets[d])
// at d * ne + r (ne: nonemptyRows; rows from ne on are empty), and columns
// outside [0, cols) are skipped. Each thread takes R = 16 / sizeof( Real )
// adjacent rows (FP64 pairs, FP32 quads): with VEC (ne and row_begin multiples
// of R, values 16-byte aligned) the R values of a diagonal are one 16-byte
// load — measured on the 128^3 Laplacian pattern against 32-byte FP64 quads and
// one row per thread. Each row sums in increasing diagonal order, which is
// its increasing column order.
template< typename Real, bool VEC, class Sink >
__global__ void __launch_bounds__( kSpmvBlock )
mdiag_kernel( const int32_t* __restrict__ doff, int32_t ndiag, const Real* __restrict__ val, int32_t ne, int32_t cols,
              const Real* __restrict__ x, int32_t row_begin, int32_t row_end, Sink sink, RedScratch rs )
{
   constexpr int R = 16 / sizeof( Real );
   using Vec = typename std::conditional< std::is_same< Real, double >::value, double2, float4 >::type;
   if( sink.skip() )
      return;
   __shared__ int32_t so[ kMaxDiagonals ];
   for( int d = threadIdx.x; d < ndiag; d += kSpmvBlock )
      so[ d ] = doff[ d ];
   __syncthreads();
   AccOf< Sink > acc{};
   for( int64_t r = row_begin + R * ( blockIdx.x * (int64_t) kSpmvBlock + threadIdx.x ); r < row_end;
        r += R * (int64_t) gridDim.x * kSpmvBlock ) {
      Real s[ R ];
#pragma unroll
      for( int j = 0; j < R; j++ )
         s[ j ] = 0;
      if( r < ne ) {
         const bool inner = r + R - 1 < ne;
#pragma unroll 2
         for( int d = 0; d < ndiag; d++ ) {
            const int64_t g = (int64_t) d * ne + r;
            Real v[ R ];
            if constexpr( VEC ) {
               const Vec q = ld_stream( reinterpret_cast< const Vec* >( val + g ) );
               static_assert( sizeof( Vec ) == R * sizeof( Real ), "one 16-byte load" );
               memcpy( v, &q, sizeof( Vec ) );
            }
            else {
#pragma unroll
               for( int j = 0; j < R; j++ )
                  v[ j ] = ( inner || r + j < ne ) ? ld_stream( val + g + j ) : Real( 0 );
            }
            const int64_t c = r + so[ d ];
            if( c >= 0 && c + R - 1 < cols && inner ) {
#pragma unroll
               for( int j = 0; j < R; j++ )
                  s[ j ] += v[ j ] * __ldg( x + c + j );
            }
            else {
#pragma unroll
               for( int j = 0; j < R; j++ )
                  if( c + j >= 0 && c + j < cols && r + j < ne )
                     s[ j ] += v[ j ] * __ldg( x + c + j );
            }
         }
      }
#pragma unroll
      for( int j = 0; j < R; j++ )
         if( r + j < row_end )
            sink.put( (int) r + j, s[ j ], acc.v );
   }
   spmv_epilogue< Sink, kSpmvBlock >( sink, acc.v, rs );
}

// Ellpack, four rows per thread (row_begin and alignedSize multiples of 4)
template< typename Real, class Sink >
__global__ void __launch_bounds__( kSpmvBlock )
ellpack4_kernel( const int32_t* __restrict__ col, const Real* __restrict__ val, int32_t segmentSize,
                 int32_t alignedSize, const Real* __restrict__ x, int32_t row_begin, int32_t row_end, Sink sink,
                 RedScratch rs )
{
   if( sink.skip() )
      return;
   AccOf< Sink > acc{};
   for( int64_t r = row_begin + 4 * ( blockIdx.x * (int64_t) kSpmvBlock + threadIdx.x ); r < row_end;
        r += 4 * (int64_t) gridDim.x * kSpmvBlock ) {
      Real s[ 4 ] = { 0, 0, 0, 0 };
      int64_t g = r;
#pragma unroll 4
      for( int k = 0; k < segmentSize; k++, g += alignedSize )
         slot_fma4( col, val, x, g, s );
#pragma unroll
      for( int j = 0; j < 4; j++ )
         if( r + j < row_end )
            sink.put( (int) r + j, s[ j ], acc.v );
   }
   spmv_epilogue< Sink, kSpmvBlock >( sink, acc.v, rs );
}

// SlicedEllpack, four rows per thread (row_begin a multiple of 4; S and the
// slice offsets are multiples of 8)
template< typename Real, int S, class Sink >
__global__ void __launch_bounds__( kSpmvBlock )
sliced4_kernel( const int32_t* __restrict__ col, const Real* __restrict__ val, const int32_t* __restrict__ sliceOffsets,
                const Real* __restrict__ x, int32_t row_begin, int32_t row_end, Sink sink, RedScratch rs )
{
   if( sink.skip() )
      return;
   AccOf< Sink > acc{};
   for( int64_t r = row_begin + 4 * ( blockIdx.x * (int64_t) kSpmvBlock + threadIdx.x ); r < row_end;
        r += 4 * (int64_t) gridDim.x * kSpmvBlock ) {
      const int slice = (int) ( r / S );
      const int b = __ldg( sliceOffsets + slice ) + (int) ( r % S );
      const int e = __ldg( sliceOffsets + slice + 1 );
      Real s[ 4 ] = { 0, 0, 0, 0 };
#pragma unroll 4
      for( int g = b; g < e; g += S )
         slot_fma4( col, val, x, g, s );
#pragma unroll
      for( int j = 0; j < 4; j++ )
         if( r + j < row_end )
            sink.put( (int) r + j, s[ j ], acc.v );
   }
   spmv_epilogue< Sink, kSpmvBlock >( sink, acc.v, rs );
}

// ---------------------------------------------------------------------------
// ChunkedEllpack (ColumnMajor): one block of 256 threads per slice, one
// thread per chunk; chunk sums are combined per row in chunk order.
template< typename Real, bool SKIP, class Sink >
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
         slot_fma< Real, SKIP >( col, val, x, g, s );
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

// ChunkedEllpack whose rows have exactly one chunk each: chunk t of a slice is
// row firstSegment + t, so its thread sums the row's slots (column-major inside
// the slice) and stores the row — no shared-memory combine and no barrier per
// slice. The row's value is 0 + its chunk's sum, as the general kernel forms it.
template< typename Real, bool SKIP, class Sink >
__global__ void __launch_bounds__( kChunksInSlice )
chunked1_kernel( const int32_t* __restrict__ col, const Real* __restrict__ val, const ChunkSlice* __restrict__ slices,
                 const int32_t* __restrict__ rowToSlice, const Real* __restrict__ x, int32_t row_begin,
                 int32_t row_end, Sink sink, RedScratch rs )
{
   if( sink.skip() )
      return;  // uniform over the grid: the solve this launch belongs to is finished
   AccOf< Sink > acc{};
   const int s_first = __ldg( rowToSlice + row_begin );
   const int s_last = __ldg( rowToSlice + row_end - 1 );
   for( int sidx = s_first + blockIdx.x; sidx <= s_last; sidx += gridDim.x ) {
      const ChunkSlice sl = slices[ sidx ];
      const int row = sl.firstSegment + (int) threadIdx.x;
      if( (int) threadIdx.x < sl.size && row >= row_begin && row < row_end ) {
         Real s = 0;
         int64_t g = (int64_t) sl.pointer + threadIdx.x;
#pragma unroll 4
         for( int o = 0; o < sl.chunkSize; o++, g += kChunksInSlice )
            slot_fma< Real, SKIP >( col, val, x, g, s );
         Real r = 0;
         r += s;
         sink.put( row, r, acc.v );
      }
   }
   spmv_epilogue< Sink, kChunksInSlice >( sink, acc.v, rs );
}

// ---------------------------------------------------------------------------
// BiEllpack (ColumnMajor, warp 32): one thread per row; the row's strip rank
// selects how many groups it spans (detail/BiEllpack.h:48-64) and group g
// stores element i of rank p at groupPointer + p + i*(32>>g).
template< typename Real, bool SKIP, class Sink >
__global__ void __launch_bounds__( kSpmvBlock )
biell_kernel( const int32_t* __restrict__ col, const Real* __restrict__ val, const int32_t* __restrict__ rowPerm,
              const int32_t* __restrict__ groupPointers, const Real* __restrict__ x, int32_t row_begin,
              int32_t row_end, Sink sink, RedScratch rs )
{
   if( sink.skip() )
      return;  // uniform over the grid: the solve this launch belongs to is finished
   AccOf< Sink > acc{};
   const int lane = threadIdx.x & 31;
   const int64_t warp_global = ( blockIdx.x * (int64_t) kSpmvBlock + threadIdx.x ) >> 5;
   const int64_t nwarps = ( (int64_t) gridDim.x * kSpmvBlock ) >> 5;
   // warp-uniform loop: a warp takes 32 consecutive rows, normally one strip
   for( int64_t base = row_begin + warp_global * 32; base < row_end; base += nwarps * 32 ) {
      const int64_t r = base + lane;
      const bool active = r < row_end;
      const int strip = (int) ( ( active ? r : base ) / kBiWarp );
      const int gb = strip * kBiGroups;
      // the strip's seven group pointers, loaded once by lanes 0..6 when the
      // whole warp is in one strip (one round trip instead of up to seven)
      const bool one_strip = __all_sync( 0xffffffffu, strip == __shfl_sync( 0xffffffffu, strip, 0 ) );
      int gpl = 0;
      if( one_strip && lane <= kBiGroups )
         gpl = __ldg( groupPointers + gb + lane );
      int gpk[ kBiGroups + 1 ];
#pragma unroll
      for( int k = 0; k <= kBiGroups; k++ )
         gpk[ k ] = __shfl_sync( 0xffffffffu, gpl, k );
      if( active ) {
         const int p = __ldg( rowPerm + r ) - strip * kBiWarp;
         const int groups = p == 0 ? 6 : ( p < 2 ? 5 : ( p < 4 ? 4 : ( p < 8 ? 3 : ( p < 16 ? 2 : 1 ) ) ) );
         Real s = 0;
         int h = kBiWarp;
         int gp = one_strip ? gpk[ 0 ] : __ldg( groupPointers + gb );
#pragma unroll
         for( int k = 0; k < kBiGroups; k++ ) {  // unrolled: gpk stays in registers
            if( k < groups ) {
               const int gn = one_strip ? gpk[ k + 1 ] : __ldg( groupPointers + gb + k + 1 );
               const int w = ( gn - gp ) / h;
               int64_t g = (int64_t) gp + p;
#pragma unroll 4
               for( int i = 0; i < w; i++, g += h )
                  slot_fma< Real, SKIP >( col, val, x, g, s );
               gp = gn;
               h >>= 1;
            }
         }
         sink.put( (int) r, s, acc.v );
      }
   }
   spmv_epilogue< Sink, kSpmvBlock >( sink, acc.v, rs );
}

// BiEllpack by strip rank: lane p of a warp takes rank p of one strip, so its
// slots gp + p + i*(32>>g) need no permutation lookup first, and the row it
// stores (rankRow, the inverse of rowPerm) is loaded alongside the slots. The
// sum runs over the same slots in the same order as biell_kernel.
template< typename Real, bool SKIP, class Sink >
__global__ void __launch_bounds__( kSpmvBlock )
biell_rank_kernel( const int32_t* __restrict__ col, const Real* __restrict__ val, const int32_t* __restrict__ rankRow,
                   const int32_t* __restrict__ groupPointers, const Real* __restrict__ x, int32_t row_begin,
                   int32_t row_end, Sink sink, RedScratch rs )
{
   if( sink.skip() )
      return;  // uniform over the grid: the solve this launch belongs to is finished
   AccOf< Sink > acc{};
   const int p = threadIdx.x & 31;
   const int groups = p == 0 ? 6 : ( p < 2 ? 5 : ( p < 4 ? 4 : ( p < 8 ? 3 : ( p < 16 ? 2 : 1 ) ) ) );
   const int64_t warp_global = ( blockIdx.x * (int64_t) kSpmvBlock + threadIdx.x ) >> 5;
   const int64_t nwarps = ( (int64_t) gridDim.x * kSpmvBlock ) >> 5;
   const int64_t first = row_begin / kBiWarp, last = ( (int64_t) row_end - 1 ) / kBiWarp;
   for( int64_t strip = first + warp_global; strip <= last; strip += nwarps ) {
      int gpl = 0;
      if( p <= kBiGroups )
         gpl = __ldg( groupPointers + strip * kBiGroups + p );
      const int row = __ldg( rankRow + strip * kBiWarp + p );
      int gpk[ kBiGroups + 1 ];
#pragma unroll
      for( int k = 0; k <= kBiGroups; k++ )
         gpk[ k ] = __shfl_sync( 0xffffffffu, gpl, k );
      if( row >= row_begin && row < row_end ) {
         Real s = 0;
#pragma unroll
         for( int k = 0; k < kBiGroups; k++ ) {
            if( k < groups ) {
               const int w = ( gpk[ k + 1 ] - gpk[ k ] ) >> ( 5 - k );  // group k: 32 >> k ranks wide
               int64_t g = (int64_t) gpk[ k ] + p;
#pragma unroll 4
               for( int i = 0; i < w; i++, g += ( kBiWarp >> k ) )
                  slot_fma< Real, SKIP >( col, val, x, g, s );
            }
         }
         sink.put( row, s, acc.v );
      }
   }
   spmv_epilogue< Sink, kSpmvBlock >( sink, acc.v, rs );
}

// BiEllpack by rank pairs: a half-warp takes one strip, lane q its ranks 2q and
// 2q + 1, whose group-0 slots are neighbours — one 8-byte column load and one
// two-element value load serve both where the strip's group 0 starts at an even
// slot (otherwise, and in the higher groups, the ranks load one by one). Each
// rank's sum keeps the slot order of biell_rank_kernel.
template< typename Real, bool SKIP, class Sink >
__global__ void __launch_bounds__( kSpmvBlock )
biell_pair_kernel( const int32_t* __restrict__ col, const Real* __restrict__ val, const int32_t* __restrict__ rankRow,
                   const int32_t* __restrict__ groupPointers, const Real* __restrict__ x, int32_t row_begin,
                   int32_t row_end, Sink sink, RedScratch rs )
{
   if( sink.skip() )
      return;  // uniform over the grid: the solve this launch belongs to is finished
   AccOf< Sink > acc{};
   const int lane = threadIdx.x & 31, half = lane >> 4, q = lane & 15;
   const int p0 = 2 * q, p1 = 2 * q + 1;
   auto groups_of = []( int p ) { return p == 0 ? 6 : ( p < 2 ? 5 : ( p < 4 ? 4 : ( p < 8 ? 3 : ( p < 16 ? 2 : 1 ) ) ) ); };
   const int g0 = groups_of( p0 ), g1 = groups_of( p1 );
   const int64_t warp_global = ( blockIdx.x * (int64_t) kSpmvBlock + threadIdx.x ) >> 5;
   const int64_t nwarps = ( (int64_t) gridDim.x * kSpmvBlock ) >> 5;
   const int64_t first = row_begin / kBiWarp, last = ( (int64_t) row_end - 1 ) / kBiWarp;
   for( int64_t pair = warp_global; first + 2 * pair <= last; pair += nwarps ) {
      const int64_t strip = first + 2 * pair + half;
      const bool live = strip <= last;
      int gpl = 0;
      if( live && q <= kBiGroups )
         gpl = __ldg( groupPointers + strip * kBiGroups + q );
      int row0 = -1, row1 = -1;
      if( live ) {
         row0 = __ldg( rankRow + strip * kBiWarp + p0 );
         row1 = __ldg( rankRow + strip * kBiWarp + p1 );
      }
      int gpk[ kBiGroups + 1 ];
#pragma unroll
      for( int k = 0; k <= kBiGroups; k++ )
         gpk[ k ] = __shfl_sync( 0xffffffffu, gpl, ( lane & 16 ) + k );
      const bool in0 = row0 >= row_begin && row0 < row_end, in1 = row1 >= row_begin && row1 < row_end;
      if( in0 || in1 ) {
         Real s0 = 0, s1 = 0;
         // group 0: all 32 ranks, 32 slots per element position
         const int w0 = ( gpk[ 1 ] - gpk[ 0 ] ) >> 5;
         int64_t g = (int64_t) gpk[ 0 ] + p0;
         if( ( gpk[ 0 ] & 1 ) == 0 ) {
#pragma unroll 4
            for( int i = 0; i < w0; i++, g += kBiWarp )
               slot_fma2< Real, SKIP >( col, val, x, g, s0, s1 );
         }
         else {
#pragma unroll 4
            for( int i = 0; i < w0; i++, g += kBiWarp ) {
               slot_fma< Real, SKIP >( col, val, x, g, s0 );
               slot_fma< Real, SKIP >( col, val, x, g + 1, s1 );
            }
         }
#pragma unroll
         for( int k = 1; k < kBiGroups; k++ ) {
            const int w = ( gpk[ k + 1 ] - gpk[ k ] ) >> ( 5 - k );  // group k: 32 >> k ranks wide
            if( k < g0 ) {
               int64_t h = (int64_t) gpk[ k ] + p0;
               for( int i = 0; i < w; i++, h += ( kBiWarp >> k ) )
                  slot_fma< Real, SKIP >( col, val, x, h, s0 );
            }
            if( k < g1 ) {
               int64_t h = (int64_t) gpk[ k ] + p1;
               for( int i = 0; i < w; i++, h += ( kBiWarp >> k ) )
                  slot_fma< Real, SKIP >( col, val, x, h, s1 );
            }
         }
         if( in0 )
            sink.put( row0, s0, acc.v );
         if( in1 )
            sink.put( row1, s1, acc.v );
      }
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

// Four rows per thread where padding is rare, by measurement on the 128^3
// Laplacian: Ellpack in both value types (FP64 0.81 -> 0.85 of the copy
// bandwidth with 32-byte value loads), SlicedEllpack in FP32 only (FP64 fell
// from 0.85 with row pairs to 0.79)
template< typename Real >
constexpr bool kQuadRowsEllpack = true;
template< typename Real >
constexpr bool kQuadRowsSliced = sizeof( Real ) == 4;

// Rows per lane of the row-group kernel. One for both value types: two FP32
// rows per lane (64-row groups, 6 resident blocks per SM) measured 12 % slower
// on the 3D Laplacians (128^3: 0.62 against 0.705 of the copy bandwidth;
// 160^3: 0.71 against 0.80) — more warps beat more work per warp.
#ifndef B2S_CSR_GROUP_RPL_F32
#define B2S_CSR_GROUP_RPL_F32 1
#endif
template< typename Real >
constexpr int csr_group_rows_per_lane()
{
   return sizeof( Real ) == 4 ? B2S_CSR_GROUP_RPL_F32 : 1;
}

// the row-group kernel on the rows [rb, re) (rb a multiple of 32 RPL), over
// the resident blocks only
template< typename Real, int RPL, class Sink >
inline b2s_status
launch_csr_group( const int32_t* off, const int32_t* col, const Real* values, const Real* x, int32_t rb, int32_t re,
                  const Sink& sink, RedScratch rs, cudaStream_t s )
{
   auto kern = csr_group_kernel< Real, RPL, Sink >;
   static int per_sm[ 64 ] = {};
   const int dev = current_device();
   int occ = dev >= 0 && dev < 64 ? per_sm[ dev ] : 0;
   if( occ == 0 ) {
      B2S_TRY_CUDA( cudaOccupancyMaxActiveBlocksPerMultiprocessor( &occ, kern, kCsrGroupBlock, 0 ) );
      occ = std::max( occ, 1 );
      if( dev >= 0 && dev < 64 )
         per_sm[ dev ] = occ;
   }
   const int64_t nr = (int64_t) re - rb;
   const int64_t groups = ( nr + kCsrGroupRows * RPL - 1 ) / ( kCsrGroupRows * RPL );
   const int64_t want = ( groups + kCsrGroupWarps - 1 ) / kCsrGroupWarps;
   const int grid = (int) std::max< int64_t >(
      1, std::min< int64_t >( want, std::min< int64_t >( (int64_t) num_sms() * occ, kMaxReduceGrid ) ) );
   kern<<< grid, kCsrGroupBlock, 0, s >>>( off, col, values, x, rb, re, sink, rs );
   B2S_TRY_CUDA( cudaGetLastError() );
   return B2S_OK;
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
   // padded layouts: skip the value loads of padding slots when padding is
   // more than a quarter of the slots
   const bool skip = (double) A->alloc_elems > 1.25 * (double) std::max< int64_t >( A->nnz, 1 );
   // the row-quad and row-pair kernels load 4 (2) neighbouring slots at once:
   // their base pointers must be aligned to those loads
   const bool quad_aligned = reinterpret_cast< uintptr_t >( values ) % ( 4 * sizeof( Real ) ) == 0
                             && reinterpret_cast< uintptr_t >( col ) % 16 == 0;
   const bool pair_aligned = reinterpret_cast< uintptr_t >( values ) % ( 2 * sizeof( Real ) ) == 0
                             && reinterpret_cast< uintptr_t >( col ) % 8 == 0;
   switch( A->format ) {
      case B2S_CSR: {
         const int32_t* off = A->offsets.as< int32_t >();
         if( A->csr_kernel == B2S_CSR_ADAPTIVE && A->csr_group && rb % kCsrGroupRows == 0 ) {
            constexpr int R2 = csr_group_rows_per_lane< Real >();
            if( R2 > 1 && rb % ( kCsrGroupRows * R2 ) == 0 )
               B2S_TRY( ( launch_csr_group< Real, R2, Sink >( off, col, values, x, rb, re, sink, rs, s ) ) );
            else
               B2S_TRY( ( launch_csr_group< Real, 1, Sink >( off, col, values, x, rb, re, sink, rs, s ) ) );
            break;
         }
         if( A->csr_kernel == B2S_CSR_ADAPTIVE && rb == 0 && re == A->rows ) {
            auto kern = A->csr_pipe ? csr_warp_kernel< Real, true, Sink > : csr_warp_kernel< Real, false, Sink >;
            static int per_sm[ 64 ][ 2 ] = {};
            const int dev = current_device();
            int occ = dev >= 0 && dev < 64 ? per_sm[ dev ][ A->csr_pipe ] : 0;
            if( occ == 0 ) {
               B2S_TRY_CUDA( cudaOccupancyMaxActiveBlocksPerMultiprocessor( &occ, kern, kCsrBlock, 0 ) );
               occ = std::max( occ, 1 );
               if( dev >= 0 && dev < 64 )
                  per_sm[ dev ][ A->csr_pipe ] = occ;
            }
            constexpr int t = CsrWin< Real >::table;
            const int64_t nwin = A->n_win[ t ];
            const int64_t want = ( nwin + kCsrWarpsPerCta - 1 ) / kCsrWarpsPerCta;
            const int grid = (int) std::max< int64_t >(
               1, std::min< int64_t >( want, std::min< int64_t >( (int64_t) num_sms() * occ, kMaxReduceGrid ) ) );
            kern<<< grid, kCsrBlock, 0, s >>>( off, col, values, x, A->csr_win[ t ].as< int32_t >(), nwin, A->nnz, sink,
                                              rs );
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
         // row pairs where padding is rare (with much padding the pair's
         // shorter row would load values of its padding slots)
         if constexpr( kQuadRowsEllpack< Real > ) {
            if( ! skip && quad_aligned && rb % 4 == 0 && A->alignedSize % 4 == 0 ) {
               ellpack4_kernel< Real, Sink ><<< spmv_grid( ( nr + 3 ) / 4, kSpmvBlock ), kSpmvBlock, 0, s >>>(
                  col, values, A->segmentSize, A->alignedSize, x, rb, re, sink, rs );
               break;
            }
         }
         if( ! skip && pair_aligned && rb % 2 == 0 && A->alignedSize % 2 == 0 )
            ellpack2_kernel< Real, false, Sink ><<< spmv_grid( ( nr + 1 ) / 2, kSpmvBlock ), kSpmvBlock, 0, s >>>(
               col, values, A->segmentSize, A->alignedSize, x, rb, re, sink, rs );
         else if( skip )
            ellpack_kernel< Real, true, Sink ><<< spmv_grid( nr, kSpmvBlock ), kSpmvBlock, 0, s >>>(
               col, values, A->segmentSize, A->alignedSize, x, rb, re, sink, rs );
         else
            ellpack_kernel< Real, false, Sink ><<< spmv_grid( nr, kSpmvBlock ), kSpmvBlock, 0, s >>>(
               col, values, A->segmentSize, A->alignedSize, x, rb, re, sink, rs );
         break;
      case B2S_SLICED_ELLPACK: {
         const bool quad = kQuadRowsSliced< Real > && ! skip && quad_aligned && rb % 4 == 0;
         const bool pair = ! quad && ! skip && pair_aligned && rb % 2 == 0;
         const int grid = spmv_grid( quad ? ( nr + 3 ) / 4 : ( pair ? ( nr + 1 ) / 2 : nr ), kSpmvBlock );
         const int32_t* so = A->sliceOffsets.as< int32_t >();
#define B2S_SLICED( SS )                                                                                            \
   if constexpr( kQuadRowsSliced< Real > ) {                                                                       \
      if( quad ) {                                                                                                  \
         sliced4_kernel< Real, SS, Sink ><<< grid, kSpmvBlock, 0, s >>>( col, values, so, x, rb, re, sink, rs );    \
         break;                                                                                                     \
      }                                                                                                             \
   }                                                                                                                \
   if( pair )                                                                                                       \
      sliced2_kernel< Real, SS, false, Sink ><<< grid, kSpmvBlock, 0, s >>>( col, values, so, x, rb, re, sink, rs ); \
   else if( skip )                                                                                                  \
      sliced_kernel< Real, SS, true, Sink ><<< grid, kSpmvBlock, 0, s >>>( col, values, so, x, rb, re, sink, rs );   \
   else                                                                                                             \
      sliced_kernel< Real, SS, false, Sink ><<< grid, kSpmvBlock, 0, s >>>( col, values, so, x, rb, re, sink, rs );
         switch( A->slice_size ) {
            case 8:
               B2S_SLICED( 8 )
               break;
            case 16:
               B2S_SLICED( 16 )
               break;
            case 64:
               B2S_SLICED( 64 )
               break;
            default:
               B2S_SLICED( 32 )
               break;
         }
#undef B2S_SLICED
         break;
      }
      case B2S_CHUNKED_ELLPACK: {
         const int grid = (int) std::min< int64_t >( std::max( A->numberOfSlices, 1 ),
                                                     std::min< int64_t >( (int64_t) num_sms() * 8, kMaxReduceGrid ) );
         if( A->chunk_single ) {
            if( skip )
               chunked1_kernel< Real, true, Sink ><<< grid, kChunksInSlice, 0, s >>>(
                  col, values, A->cslices.as< ChunkSlice >(), A->rowToSlice.as< int32_t >(), x, rb, re, sink, rs );
            else
               chunked1_kernel< Real, false, Sink ><<< grid, kChunksInSlice, 0, s >>>(
                  col, values, A->cslices.as< ChunkSlice >(), A->rowToSlice.as< int32_t >(), x, rb, re, sink, rs );
         }
         else if( skip )
            chunked_kernel< Real, true, Sink ><<< grid, kChunksInSlice, 0, s >>>(
               col, values, A->cslices.as< ChunkSlice >(), A->rowToChunk.as< int32_t >(), A->rowToSlice.as< int32_t >(), x,
               rb, re, sink, rs );
         else
            chunked_kernel< Real, false, Sink ><<< grid, kChunksInSlice, 0, s >>>(
               col, values, A->cslices.as< ChunkSlice >(), A->rowToChunk.as< int32_t >(), A->rowToSlice.as< int32_t >(), x,
               rb, re, sink, rs );
         break;
      }
      case B2S_BIELLPACK:
         if( A->rankRow.p && ! skip && pair_aligned ) {
            // rank pairs where padding is rare (a pair loads both ranks' values)
            const int64_t lanes = ( ( (int64_t) re - 1 ) / kBiWarp - rb / kBiWarp + 2 ) / 2 * kBiWarp;
            biell_pair_kernel< Real, false, Sink ><<< spmv_grid( lanes, kSpmvBlock ), kSpmvBlock, 0, s >>>(
               col, values, A->rankRow.as< int32_t >(), A->groupPointers.as< int32_t >(), x, rb, re, sink, rs );
         }
         else if( A->rankRow.p ) {
            const int64_t lanes = ( ( (int64_t) re - 1 ) / kBiWarp - rb / kBiWarp + 1 ) * kBiWarp;
            if( skip )
               biell_rank_kernel< Real, true, Sink ><<< spmv_grid( lanes, kSpmvBlock ), kSpmvBlock, 0, s >>>(
                  col, values, A->rankRow.as< int32_t >(), A->groupPointers.as< int32_t >(), x, rb, re, sink, rs );
            else
               biell_rank_kernel< Real, false, Sink ><<< spmv_grid( lanes, kSpmvBlock ), kSpmvBlock, 0, s >>>(
                  col, values, A->rankRow.as< int32_t >(), A->groupPointers.as< int32_t >(), x, rb, re, sink, rs );
         }
         else if( skip )
            biell_kernel< Real, true, Sink ><<< spmv_grid( nr, kSpmvBlock ), kSpmvBlock, 0, s >>>(
               col, values, A->rowPerm.as< int32_t >(), A->groupPointers.as< int32_t >(), x, rb, re, sink, rs );
         else
            biell_kernel< Real, false, Sink ><<< spmv_grid( nr, kSpmvBlock ), kSpmvBlock, 0, s >>>(
               col, values, A->rowPerm.as< int32_t >(), A->groupPointers.as< int32_t >(), x, rb, re, sink, rs );
         break;
      case B2S_MULTIDIAGONAL: {
         // one 16-byte value load per diagonal and thread: r and ne multiples
         // of the rows per thread, the values 16-byte aligned
         constexpr int R = 16 / sizeof( Real );
         const int32_t ne = A->alignedSize;
         const bool vec = rb % R == 0 && ne % R == 0 && reinterpret_cast< uintptr_t >( values ) % 16 == 0;
         const int grid = spmv_grid( ( nr + R - 1 ) / R, kSpmvBlock );
         const int32_t* doff = A->diagOffsets.as< int32_t >();
         if( vec )
            mdiag_kernel< Real, true, Sink ><<< grid, kSpmvBlock, 0, s >>>( doff, A->segmentSize, values, ne, A->cols, x,
                                                                           rb, re, sink, rs );
         else
            mdiag_kernel< Real, false, Sink ><<< grid, kSpmvBlock, 0, s >>>( doff, A->segmentSize, values, ne, A->cols, x,
                                                                            rb, re, sink, rs );
         break;
      }
      default:
         set_error( "unknown format" );
         return B2S_INVALID_ARG;
   }
   B2S_TRY_CUDA( cudaGetLastError() );
   return B2S_OK;
}

}  // namespace b2s
