// The stationary solvers Solvers::Linear::Jacobi (Jacobi.hpp:67-128) and SOR
// (SOR.hpp:66-118) with the iteration control of IterativeSolver.
//
// Jacobi: each sweep is one SpMV whose sink writes
//    out_i = in_i + (omega / a_ii) (b_i - row_i . in),
// two sweeps per loop pass (x -> aux -> x); the residue ||A x - b|| / ||b||
// is an SpMV with a reduction, launched after every sweep and skipped on the
// device unless the iteration count is a multiple of the residue period, as
// in TNL (whose first check of a pass reads x before the second sweep).
//
// SOR: TNL's Devices::Host sweep is the sequential forward sweep
//    x_i += (omega / a_ii) (b_i - row_i . x)
// with the rows before i already updated. Here it runs as one dependency
// kernel per sweep, the scheme of the ILU(0) substitutions: a warp takes the
// next row from a ticket counter in the level order of the strict lower
// triangle's dependency graph, its lanes wait (bounded) for the rows j < i of
// the row to publish their new values, and the row publishes its own. The
// new values go to a second vector (rows j > i read the previous sweep's
// values whatever the pattern), and the two vectors swap roles every sweep.
//
// Arithmetic follows the reference build (g++ -O3 -march=x86-64-v3) of TNL's
// host loops: FP64 row sums are fused multiply-adds in element order; FP32
// rows sum their rounded FP32 products in FP64 (the reduction's identity is
// the double 0.0) and round the sum to FP32; SOR adds the rounded update
// (x += t u, an atomic addition in TNL), Jacobi fuses it (in + t u).
#pragma once

#include "ilu.cuh"
#include "krylov_kernels.cuh"

#include <algorithm>
#include <vector>

namespace b2s {

// nextIteration at the start of a pass (mode 0); mode 1 counts the second
// sweep of a Jacobi pass without a check (Jacobi.hpp:103-107)
__global__ void
stat_ctl_kernel( Ctl* ctl, int mode )
{
   Ctl& c = *ctl;
   if( c.done )
      return;
   if( mode == 0 )
      next_iteration( c );
   else
      c.it++;
}

// ||b|| as LinearResidueGetter divides by it (no guard against zero)
struct StatNormbFin
{
   static constexpr bool active = true;
   __device__ void operator()( Ctl& c, const double* t ) const { c.normb = sqrt( t[ 0 ] ); }
};

// residue = ||A x - b|| / ||b|| (LinearResidueGetter.hpp:16-28); `always`: the
// final one after the loop, otherwise only when it % period == 0
template< typename Real >
struct StatResG
{
   static constexpr int NR = 1;
   const Real* b;
   Ctl* ctl;
   long long period;
   int always;
   __device__ bool
   skip() const
   {
      if( always )
         return false;
      const Ctl& c = *ctl;
      return c.done != 0 || c.it % period != 0;
   }
   __device__ __forceinline__ void
   put( int row, Real s, double* acc ) const
   {
      const double d = (double) s - (double) b[ row ];
      acc[ 0 ] += d * d;
   }
   __device__ void
   finish( const double* t ) const
   {
      Ctl& c = *ctl;
      c.residue = sqrt( t[ 0 ] ) / c.normb;
   }
};

__device__ __forceinline__ double
fused( double a, double b, double c )
{
   return __fma_rn( a, b, c );
}
__device__ __forceinline__ float
fused( float a, float b, float c )
{
   return __fmaf_rn( a, b, c );
}

// one Jacobi sweep: out = in + (omega / diag) (b - A in)   (Jacobi.hpp:112-128)
template< typename Real >
struct JacobiG
{
   static constexpr int NR = 0;
   const Real* in;
   Real* out;
   const Real* b;
   const Real* diag;
   Real omega;
   const Ctl* ctl;
   __device__ bool skip() const { return ctl->done != 0; }
   __device__ __forceinline__ void
   put( int row, Real s, double* ) const
   {
      const Real t = omega / diag[ row ];
      out[ row ] = fused( t, b[ row ] - s, in[ row ] );
   }
   __device__ void finish( const double* ) const {}
};

template< typename Real >
struct SorView
{
   int32_t n;
   const int32_t* off;
   const int32_t* col;
   const Real* val;
   const int32_t* ord;  // rows by level of the strict lower triangle
   int32_t nord;
   int32_t* flags;
   IluState* st;
};

// a row's sum in the reference build's evaluation
__device__ __forceinline__ double
sor_acc( double acc, double v, double x )
{
   return __fma_rn( v, x, acc );
}
__device__ __forceinline__ double
sor_acc( double acc, float v, float x )
{
   return __dadd_rn( acc, (double) __fmul_rn( v, x ) );
}
__device__ __forceinline__ double
sor_keep( double xo, double t, double u )
{
   return __dadd_rn( xo, __dmul_rn( t, u ) );
}
__device__ __forceinline__ float
sor_keep( float xo, float t, float u )
{
   return __fadd_rn( xo, __fmul_rn( t, u ) );
}

// one forward SOR sweep xo -> xn (SOR.hpp:101-118), one warp per row in
// level order; x may not alias
template< typename Real >
__global__ void __launch_bounds__( kIluBlock )
sor_sweep_kernel( SorView< Real > P, const Real* __restrict__ b, const Real* __restrict__ diag, const Real* xo, Real* xn,
                  Real omega, const Ctl* ctl )
{
   if( ctl->done )
      return;
   const int lane = threadIdx.x & 31;
   IluState* st = P.st;
   const int epoch = *(volatile int*) &st->epoch;
   for( ;; ) {
      unsigned t = 0;
      if( lane == 0 )
         t = atomicAdd( &st->ticket, 1u );
      t = __shfl_sync( 0xffffffffu, t, 0 );
      if( t >= (unsigned) P.nord )
         return;
      const int i = P.ord[ t ];
      if( i < 0 )
         continue;  // padding of a level
      const int b0 = P.off[ i ], b1 = P.off[ i + 1 ];
      double acc = 0.0;
      for( int base = b0; base < b1; base += 32 ) {
         const int k = base + lane;
         Real v = 0, xv = 0;
         int ok = 1;
         if( k < b1 ) {
            const int j = P.col[ k ];
            v = P.val[ k ];
            if( j < i ) {
               ok = ilu_wait( P.flags + j, epoch, st );
               if( ok )
                  xv = __ldcg( xn + j );
            }
            else
               xv = xo[ j ];
         }
         if( ! __all_sync( 0xffffffffu, ok ) )
            return;
         const int cnt = min( 32, b1 - base );
         for( int q = 0; q < cnt; q++ )
            acc = sor_acc( acc, __shfl_sync( 0xffffffffu, v, q ), __shfl_sync( 0xffffffffu, xv, q ) );
      }
      if( lane == 0 ) {
         const Real value = (Real) acc;
         const Real tt = omega / diag[ i ];
         xn[ i ] = sor_keep( xo[ i ], tt, b[ i ] - value );
         __threadfence();
         st_release( P.flags + i, epoch );
      }
      __syncwarp();
   }
}

// The sweep's plan: the matrix rows in storage order (a padded layout's
// rows without padding), the level order of the strict lower triangle, and
// the pass state.
template< typename Real >
struct SorPlan
{
   int32_t n = 0;
   DevBuf off_own, col_own, val_own;
   const int32_t* off = nullptr;
   const int32_t* col = nullptr;
   const Real* val = nullptr;
   DevBuf ord, flags, state;
   int32_t nord = 0;
   int levels = 0;
   int grid = 0;

   SorView< Real > view() const
   {
      return SorView< Real >{ n, off, col, val, ord.as< int32_t >(), nord, flags.as< int32_t >(), state.as< IluState >() };
   }

   b2s_status
   build( const b2s_matrix_t* A, cudaStream_t s )
   {
      n = A->rows;
      int64_t nnz = A->nnz;
      if( A->format == B2S_CSR ) {
         off = A->offsets.as< int32_t >();
         col = A->columns.as< int32_t >();
         val = A->values.as< Real >();
      }
      else {
         B2S_TRY( layout_to_csr( A, false, off_own, col_own, val_own, nnz, s ) );
         off = off_own.as< int32_t >();
         col = col_own.as< int32_t >();
         val = val_own.as< Real >();
      }
      B2S_TRY( flags.alloc( (size_t) std::max( n, 1 ) * sizeof( int32_t ) ) );
      B2S_TRY( state.alloc( sizeof( IluState ) ) );
      B2S_TRY_CUDA( cudaMemsetAsync( flags.p, 0, (size_t) std::max( n, 1 ) * sizeof( int32_t ), s ) );
      B2S_TRY_CUDA( cudaMemsetAsync( state.p, 0, sizeof( IluState ), s ) );
      // level of a row: one more than the deepest earlier row it reads
      std::vector< int32_t > hoff( (size_t) n + 1, 0 ), hcol( (size_t) std::max< int64_t >( nnz, 1 ) );
      if( n > 0 )
         B2S_TRY( copy_d2h( hoff.data(), off, hoff.size() * sizeof( int32_t ), s ) );
      if( nnz > 0 )
         B2S_TRY( copy_d2h( hcol.data(), col, (size_t) nnz * sizeof( int32_t ), s ) );
      std::vector< int32_t > lev( (size_t) std::max( n, 1 ), 0 );
      int depth = 0;
      for( int32_t i = 0; i < n; i++ ) {
         int l = 0;
         for( int32_t k = hoff[ i ]; k < hoff[ i + 1 ]; k++ )
            if( hcol[ k ] < i )
               l = std::max( l, lev[ hcol[ k ] ] + 1 );
         lev[ i ] = l;
         depth = std::max( depth, l + 1 );
      }
      levels = depth;
      std::vector< int64_t > start( (size_t) depth + 1, 0 );
      for( int32_t i = 0; i < n; i++ )
         start[ lev[ i ] + 1 ]++;
      for( int l = 0; l < depth; l++ )
         start[ l + 1 ] += start[ l ];
      nord = n;
      std::vector< int32_t > h( (size_t) n + 32, -1 );
      for( int32_t i = 0; i < n; i++ )
         h[ start[ lev[ i ] ]++ ] = i;
      B2S_TRY( ord.alloc( h.size() * sizeof( int32_t ) ) );
      B2S_TRY( copy_h2d( ord.p, h.data(), h.size() * sizeof( int32_t ), s ) );
      grid = num_sms() * ( 2048 / kIluBlock );
      return B2S_OK;
   }

   // xn = one sweep from xo on `s`, skipped when the solve is done
   b2s_status
   sweep( const Real* b, const Real* diag, const Real* xo, Real* xn, Real omega, Ctl* ctl, cudaStream_t s ) const
   {
      if( n == 0 )
         return B2S_OK;
      const SorView< Real > v = view();
      ilu_begin_kernel< DoneGate ><<< 1, 1, 0, s >>>( v.st, DoneGate{ ctl } );
      sor_sweep_kernel< Real ><<< grid, kIluBlock, 0, s >>>( v, b, diag, xo, xn, omega, ctl );
      B2S_TRY_CUDA( cudaGetLastError() );
      return B2S_OK;
   }

   // B2S_TIMEOUT when a bounded wait gave up (the word is reset)
   b2s_status
   check( cudaStream_t s ) const
   {
      if( n == 0 )
         return B2S_OK;
      IluState h{};
      B2S_TRY( copy_d2h( &h, state.p, sizeof( IluState ), s ) );
      if( h.error ) {
         const int zero = 0;
         B2S_TRY( copy_h2d( reinterpret_cast< char* >( state.p ) + offsetof( IluState, error ), &zero, sizeof( int ), s ) );
         set_error( "SOR: a bounded wait for an earlier row gave up" );
         return B2S_TIMEOUT;
      }
      return B2S_OK;
   }
};

}  // namespace b2s
