// ILU(0) on the device: Preconditioners::ILU0 (Solvers/Linear/Preconditioners/ILU0.hpp:23-144)
// with its triangular solves (Solvers/Linear/Utils/TriangularSolve.h:24-110).
//
// The factors live in the pattern of A (CSR, rows sorted by column, diagonal
// stored): L with a unit diagonal strictly below, U on and above it.
//
// Both the factorization and the substitutions are sequential along
// dependency chains. They run as "sync-free" persistent kernels: a warp takes
// the next row from a ticket counter, waits until every row it depends on has
// published its result (a per-row flag holding the current pass's epoch),
// computes, and publishes its own row. Tickets hand the rows out level by
// level (the level of a row is one more than the deepest row it depends on,
// computed once when the factors are built), so every awaited row was claimed
// earlier by a warp that is already running, and all rows of a level are in
// flight together — the critical path is the number of levels, not the
// number of rows. Every wait is bounded: after kIluSpinLimit polls the warp
// raises the error word and returns, and the others leave as soon as they see
// it; the host turns the word into B2S_TIMEOUT.
//
// Arithmetic follows TNL's loops element by element: for row i and each of
// its L entries k in increasing order, L_ik = L_ik / U_kk and every later
// entry j of the row takes L_ik * U_kj off (U_kj = 0 when absent); the
// substitutions subtract L_ij x_j (U_ij x_j) in increasing j and divide by
// U_ii last. The reference build (g++ -O3 -march=x86-64-v3) contracts the
// factorization updates into fused multiply-adds, leaves the FP64
// substitution sums uncontracted and vectorizes the FP32 ones by four with a
// fused remainder; the kernels evaluate every term the same way, so the
// results are TNL's bit for bit.
#pragma once

#include "b2s_internal.cuh"

#include <cstddef>
#include <type_traits>
#include <vector>

namespace b2s {

constexpr int kIluBlock = 256;
constexpr int kIluSpinLimit = 1 << 21;

struct IluState
{
   unsigned int ticket;  // next row to claim
   int epoch;            // the current pass; a row is done when its flag equals it
   int error;            // 1: a bounded wait gave up
   int pad;
};

template< typename Real >
struct IluView
{
   int32_t n;
   const int32_t* off;
   const int32_t* col;
   const int32_t* diag;  // position of A_ii in each row
   const int32_t* ord_l; // rows by level of L (the factorization and L^-1), -1 padded
   const int32_t* ord_u; // rows by level of U (U^-1), -1 padded
   int32_t n_l, n_u;     // lengths of the padded lists
   Real* lu;
   int32_t* flags;
   IluState* st;
};

struct NoGate
{
   __device__ bool skip() const { return false; }
};

// a multiply-subtract the way the reference build evaluates it
template< bool FUSED >
__device__ __forceinline__ double
msub( double a, double l, double u )
{
   return FUSED ? __fma_rn( -l, u, a ) : __dsub_rn( a, __dmul_rn( l, u ) );
}
template< bool FUSED >
__device__ __forceinline__ float
msub( float a, float l, float u )
{
   return FUSED ? __fmaf_rn( -l, u, a ) : __fsub_rn( a, __fmul_rn( l, u ) );
}
// Term q of the m terms of a substitution row, as the reference build sums
// it: FP64 products rounded, then subtracted; FP32 vectorized by four
// (rounded products subtracted in order) with the m mod 4 remaining terms
// fused.
template< typename Real >
__device__ __forceinline__ Real
sum_term( Real acc, Real v, Real xv, int q, int m )
{
   if constexpr( std::is_same< Real, float >::value ) {
      if( q >= m / 4 * 4 )
         return msub< true >( acc, v, xv );
   }
   return msub< false >( acc, v, xv );
}

__device__ __forceinline__ int
ld_acquire( const int32_t* p )
{
   int v;
   asm volatile( "ld.acquire.gpu.global.b32 %0, [%1];" : "=r"( v ) : "l"( p ) : "memory" );
   return v;
}
__device__ __forceinline__ void
st_release( int32_t* p, int v )
{
   asm volatile( "st.release.gpu.global.b32 [%0], %1;" ::"l"( p ), "r"( v ) : "memory" );
}

// bounded wait until row `j` has published in this epoch
__device__ __forceinline__ bool
ilu_wait( const int32_t* flag, int epoch, IluState* st )
{
   for( int it = 0; it < kIluSpinLimit; it++ ) {
      if( ld_acquire( flag ) == epoch )
         return true;
      if( ( it & 255 ) == 255 && *(volatile int*) &st->error )
         return false;
   }
   atomicExch( &st->error, 1 );
   return false;
}

// a new pass: tickets from 0, a fresh epoch
template< class Gate >
__global__ void
ilu_begin_kernel( IluState* st, Gate gate )
{
   if( gate.skip() )
      return;
   st->ticket = 0;
   st->epoch += 1;
}

// Rows per level are padded with -1 to a multiple of kIluRows in the
// level-ordered lists (1: no padding; the kernels skip -1 entries).
constexpr int kIluRows = 1;

// the factorization, one warp per row, in level order
template< typename Real >
__global__ void __launch_bounds__( kIluBlock )
ilu_factor_kernel( IluView< Real > L )
{
   const int lane = threadIdx.x & 31;
   IluState* st = L.st;
   const int epoch = *(volatile int*) &st->epoch;
   for( ;; ) {
      unsigned t = 0;
      if( lane == 0 )
         t = atomicAdd( &st->ticket, 1u );
      t = __shfl_sync( 0xffffffffu, t, 0 );
      if( t >= (unsigned) L.n_l )
         return;
      const int i = L.ord_l[ t ];
      if( i < 0 )
         continue;  // padding of a level
      const int b = L.off[ i ], e = L.off[ i + 1 ], d = L.diag[ i ];
      for( int ck = b; ck < d; ck++ ) {
         const int k = L.col[ ck ];  // k < i, an earlier level
         int ok = 1;
         if( lane == 0 )
            ok = ilu_wait( L.flags + k, epoch, st );
         if( ! __shfl_sync( 0xffffffffu, ok, 0 ) )
            return;
         const int dk = L.diag[ k ], ek = L.off[ k + 1 ];
         Real lik = 0;
         if( lane == 0 ) {
            lik = __ldcg( L.lu + ck ) / __ldcg( L.lu + dk );
            L.lu[ ck ] = lik;
         }
         lik = __shfl_sync( 0xffffffffu, lik, 0 );
         for( int cj = ck + 1 + lane; cj < e; cj += 32 ) {
            const int j = L.col[ cj ];
            int lo = dk, hi = ek;  // U part of row k: columns >= k, sorted
            while( lo < hi ) {
               const int mid = ( lo + hi ) >> 1;
               if( L.col[ mid ] < j )
                  lo = mid + 1;
               else
                  hi = mid;
            }
            const Real u = ( lo < ek && L.col[ lo ] == j ) ? __ldcg( L.lu + lo ) : Real( 0 );
            L.lu[ cj ] = msub< true >( __ldcg( L.lu + cj ), lik, u );
         }
         __syncwarp();
      }
      __threadfence();
      __syncwarp();
      if( lane == 0 )
         st_release( L.flags + i, epoch );
   }
}

// x = L^-1 b (UPPER = false, unit diagonal) or x = U^-1 b (UPPER = true),
// one warp per row in level order (lanes wait for the row's dependencies in
// parallel; the sum runs in TNL's order through shuffles); x may be b.
// PLAIN: every term a rounded product subtracted in order (the ILUT
// substitutions, whose loops the reference build does not vectorize).
template< typename Real, bool UPPER, class Gate, bool PLAIN = false >
__global__ void __launch_bounds__( kIluBlock )
ilu_trsv_kernel( IluView< Real > L, const Real* b, Real* x, Gate gate )
{
   if( gate.skip() )
      return;
   const int lane = threadIdx.x & 31;
   IluState* st = L.st;
   const int epoch = *(volatile int*) &st->epoch;
   const int32_t* ord = UPPER ? L.ord_u : L.ord_l;
   const int32_t nord = UPPER ? L.n_u : L.n_l;
   for( ;; ) {
      unsigned t = 0;
      if( lane == 0 )
         t = atomicAdd( &st->ticket, 1u );
      t = __shfl_sync( 0xffffffffu, t, 0 );
      if( t >= (unsigned) nord )
         return;
      const int i = ord[ t ];
      if( i < 0 )
         continue;  // padding of a level
      const int d = L.diag[ i ];
      const int b0 = UPPER ? d + 1 : L.off[ i ], b1 = UPPER ? L.off[ i + 1 ] : d;
      Real acc = b[ i ];
      for( int base = b0; base < b1; base += 32 ) {
         const int k = base + lane;
         Real v = 0, xv = 0;
         int ok = 1;
         if( k < b1 ) {
            const int j = L.col[ k ];
            v = L.lu[ k ];
            ok = ilu_wait( L.flags + j, epoch, st );
            if( ok )
               xv = __ldcg( x + j );
         }
         if( ! __all_sync( 0xffffffffu, ok ) )
            return;
         const int cnt = min( 32, b1 - base );
         for( int q = 0; q < cnt; q++ ) {
            const Real vq = __shfl_sync( 0xffffffffu, v, q ), xq = __shfl_sync( 0xffffffffu, xv, q );
            acc = PLAIN ? msub< false >( acc, vq, xq ) : sum_term< Real >( acc, vq, xq, base - b0 + q, b1 - b0 );
         }
      }
      if( UPPER )
         acc = acc / L.lu[ d ];
      if( lane == 0 ) {
         x[ i ] = acc;
         __threadfence();
         st_release( L.flags + i, epoch );
      }
      __syncwarp();
   }
}

// The factors of one matrix in one value type, with their pass state.
template< typename Real >
struct IluFactors
{
   int32_t n = 0;
   DevBuf off_own, col_own;  // the CSR pattern when A is not CSR
   const int32_t* off = nullptr;
   const int32_t* col = nullptr;
   DevBuf diag, ord_l, ord_u, lu, flags, state;
   int grid = 0;
   int levels_l = 0, levels_u = 0;  // depth of the dependency chains
   int32_t n_ord_l = 0, n_ord_u = 0;
   bool plain_sum = false;  // ILUT factors: substitution terms subtracted one by one

   IluView< Real > view() const
   {
      return IluView< Real >{ n,         off,       col, diag.as< int32_t >(), ord_l.as< int32_t >(), ord_u.as< int32_t >(),
                              n_ord_l,   n_ord_u,   lu.as< Real >(),      flags.as< int32_t >(),  state.as< IluState >() };
   }

   // x = U^-1 L^-1 b on `s` (no synchronization; x may be b)
   template< class Gate = NoGate >
   b2s_status apply( const Real* b, Real* x, cudaStream_t s, Gate gate = Gate() ) const
   {
      if( n == 0 )
         return B2S_OK;
      const IluView< Real > v = view();
      ilu_begin_kernel< Gate ><<< 1, 1, 0, s >>>( v.st, gate );
      if( plain_sum )
         ilu_trsv_kernel< Real, false, Gate, true ><<< grid, kIluBlock, 0, s >>>( v, b, x, gate );
      else
         ilu_trsv_kernel< Real, false, Gate ><<< grid, kIluBlock, 0, s >>>( v, b, x, gate );
      ilu_begin_kernel< Gate ><<< 1, 1, 0, s >>>( v.st, gate );
      if( plain_sum )
         ilu_trsv_kernel< Real, true, Gate, true ><<< grid, kIluBlock, 0, s >>>( v, x, x, gate );
      else
         ilu_trsv_kernel< Real, true, Gate ><<< grid, kIluBlock, 0, s >>>( v, x, x, gate );
      B2S_TRY_CUDA( cudaGetLastError() );
      return B2S_OK;
   }

   // B2S_TIMEOUT when a bounded wait gave up since the last check (the word is reset)
   b2s_status check( cudaStream_t s ) const
   {
      if( n == 0 )
         return B2S_OK;
      IluState h{};
      B2S_TRY( copy_d2h( &h, state.p, sizeof( IluState ), s ) );
      if( h.error ) {
         const int zero = 0;
         B2S_TRY( copy_h2d( reinterpret_cast< char* >( state.p ) + offsetof( IluState, error ), &zero, sizeof( int ), s ) );
         set_error( "ILU(0): a bounded wait for a dependency gave up" );
         return B2S_TIMEOUT;
      }
      return B2S_OK;
   }
};

// Factorize A (values in Real: A's own or its FP32 copy). Defined in ilu.cu.
template< typename Real >
b2s_status ilu_factorize( const b2s_matrix_t* A, const Real* values, IluFactors< Real >& F, cudaStream_t s );

// The level orders of F's L and U dependency graphs from the host copy of its
// pattern (hdiag: the first U position of each row), and the pass state.
template< typename Real >
b2s_status ilu_levels( IluFactors< Real >& F, const std::vector< int32_t >& hoff, const std::vector< int32_t >& hcol,
                       const std::vector< int32_t >& hdiag, cudaStream_t s );

// ILUT( p, tau ) factors of A in the ILU(0) factor structure, applied by the
// same kernels with PLAIN sums (ilut.cu).
template< typename Real >
b2s_status ilut_factorize( const b2s_matrix_t* A, int32_t p, double tau, IluFactors< Real >& F, cudaStream_t s );

}  // namespace b2s
