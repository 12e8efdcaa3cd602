// Krylov solvers: TNL's Solvers::Linear::CG (CG.hpp:11-104), BICGStab
// (BICGStab.hpp:33-145), GMRES (GMRES.hpp:72-346, 641-763), TFQMR
// (TFQMR.hpp:18-114) and BICGStabL (BICGStabL.hpp:42-250), with the
// iteration control of IterativeSolver (IterativeSolver.hpp:98-146).
//
// Differences from the reference's Devices::Cuda execution, all of them
// B200-motivated and result-preserving up to rounding:
//  * scalars (dot products, alpha/beta, Givens, residue) stay on the device;
//    TNL copies every reduction to the host (Algorithms/detail/Reduction.hpp:303-340);
//  * dot products are fused into the producing SpMV or vector update;
//  * iterations run as captured CUDA graphs; the host polls one flag per chunk
//    of iterations (GMRES: once per restart cycle);
//  * dot products accumulate in FP64 for every value type;
//  * mixed precision: FP32 matrix and vectors inside FP64 iterative refinement.
#include "krylov_kernels.cuh"
#include "tfqmr_bicgstabl.cuh"
#include "ilu.cuh"
#include "stationary.cuh"

#include <algorithm>
#include <cfloat>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <type_traits>

namespace b2s {

// ---------------------------------------------------------------------------
// Vector ops shared by the solvers
template< typename Real >
struct NormOp
{
   static constexpr int NR = 1;
   const Real* v;
   const Real* diag;
   __device__ __forceinline__ void load( const Ctl& ) {}
   __device__ __forceinline__ void
   operator()( int64_t i, double* acc ) const
   {
      Real t = v[ i ];
      if( diag )
         t = t / diag[ i ];
      acc[ 0 ] += (double) t * (double) t;
   }
};

// normb = ||M^-1 b|| (1 when zero): CG.hpp:22-32, BICGStab.hpp:42-51, GMRES.hpp:94-103
struct NormbFin
{
   static constexpr bool active = true;
   __device__ void
   operator()( Ctl& c, const double* t ) const
   {
      c.normb = sqrt( t[ 0 ] );
      if( c.normb == 0.0 )
         c.normb = 1.0;
   }
};

template< typename Real >
struct CopyCastOp
{
   static constexpr int NR = 1;
   Real* dst;
   const Real* src;
   __device__ __forceinline__ void load( const Ctl& ) {}
   __device__ __forceinline__ void operator()( int64_t i, double* ) const { dst[ i ] = src[ i ]; }
};

// ---------------------------------------------------------------------------
// Gated sinks: skip the SpMV launch when the solve (or the optional step) is off.
template< typename Real >
struct CgInitG : CgInitSink< Real >
{
   __device__ bool skip() const { return false; }
};
template< typename Real >
struct CgApG : CgApSink< Real >
{
   __device__ bool skip() const { return this->ctl->done != 0; }
};
template< typename Real >
struct BiResG : BiResSink< Real >
{
   int exact;
   __device__ bool
   skip() const
   {
      const Ctl& c = *this->ctl;
      if( this->mode == 0 )
         return false;
      if( c.done )
         return true;
      if( this->mode == 1 )
         return c.restart_flag == 0;
      return false;
   }
   __device__ void
   finish( const double* t ) const
   {
      BiResSink< Real >::finish( t );
      if( this->mode == 1 && ! exact ) {
         // after a restart the residue is ||r|| / ||b|| with the fresh r (BICGStab.hpp:106-111)
         Ctl& c = *this->ctl;
         c.residue = sqrt( t[ 0 ] ) / c.normb;
         next_iteration( c );
      }
   }
};
template< typename Real >
struct BiMatvecG : BiMatvecSink< Real >
{
   __device__ bool skip() const { return this->ctl->done != 0; }
};

// ---------------------------------------------------------------------------
// GMRES device pieces. Small arrays live in `GmArrays` (FP64, device).
struct GmArrays
{
   double *H, *sv, *cs, *sn, *y, *hl;
   int ldH;  // m_max + 1 ... H is indexed H[k + i*(m+1)] as in GMRES.hpp with the cycle's m
};

// TNL's Givens helpers (GMRES.hpp:722-750)
__host__ __device__ __forceinline__ void
gen_plane_rotation( double dx, double dy, double& cs, double& sn )
{
   if( dy == 0.0 ) {
      cs = 1.0;
      sn = 0.0;
   }
   else if( fabs( dy ) > fabs( dx ) ) {
      const double t = dx / dy;
      sn = 1.0 / sqrt( 1.0 + t * t );
      cs = t * sn;
   }
   else {
      const double t = dy / dx;
      cs = 1.0 / sqrt( 1.0 + t * t );
      sn = t * cs;
   }
}

__host__ __device__ __forceinline__ void
apply_plane_rotation( double& dx, double& dy, double cs, double sn )
{
   const double t = cs * dx + sn * dy;
   dy = cs * dy - sn * dx;
   dx = t;
}

// r = M^-1 (b - A x), acc += r.r ; mode 0: initial residual, 1: after a cycle
template< typename Real >
struct GmResSink
{
   static constexpr int NR = 1;
   const Real* b;
   Real* r;
   const Real* diag;
   Ctl* ctl;
   int mode;
   int pre = 0;  // 1: s is already M^-1 (b - A x)
   __device__ bool
   skip() const
   {
      if( mode == 0 )
         return false;
      const Ctl& c = *ctl;
      return c.done != 0 || c.o_steps < c.m;
   }
   __device__ __forceinline__ void
   put( int row, Real s, double* acc ) const
   {
      Real rr = pre ? s : b[ row ] - s;
      if( diag && ! pre )
         rr = rr / diag[ row ];
      r[ row ] = rr;
      acc[ 0 ] += (double) rr * (double) rr;
   }
   __device__ void
   finish( const double* t ) const
   {
      Ctl& c = *ctl;
      if( mode == 0 ) {
         c.gm_beta = sqrt( t[ 0 ] );
         c.it = 0;
      }
      else {
         c.beta_old = c.gm_beta;
         c.gm_beta = sqrt( t[ 0 ] );
      }
      c.residue = c.gm_beta / c.normb;
   }
};

// w = M^-1 A v_i ; MGS also forms the first projection (w, v_0)
template< typename Real, bool MGS >
struct GmWSink
{
   static constexpr int NR = MGS ? 1 : 0;
   Real* w;
   const Real* v0;
   const Real* diag;
   Ctl* ctl;
   GmArrays g;
   int i, m;
   int pre = 0;  // 1: s is already M^-1 A v_i
   __device__ bool skip() const { return ctl->cycle_stop != 0; }
   __device__ __forceinline__ void
   put( int row, Real s, double* acc ) const
   {
      if( diag && ! pre )
         s = s / diag[ row ];
      w[ row ] = s;
      if constexpr( MGS )
         acc[ 0 ] += (double) s * (double) v0[ row ];
   }
   __device__ void
   finish( const double* t ) const
   {
      if constexpr( MGS ) {
         g.hl[ 0 ] = t[ 0 ];
         g.H[ 0 + i * ( m + 1 ) ] += t[ 0 ];
      }
   }
};

// Cycle start: v_0 = (1/beta) r, H = 0, s = (beta, 0, ...), first nextIteration
template< typename Real >
__global__ void
gm_start_kernel( int64_t n, Real* __restrict__ v0, const Real* __restrict__ r, Ctl* ctl, GmArrays g, int m )
{
   Ctl& c = *ctl;
   if( c.done )
      return;
   const double beta = c.gm_beta;
   const Real scale = (Real) ( 1.0 / beta );
   for( int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x )
      v0[ i ] = scale * r[ i ];
   if( blockIdx.x == 0 && threadIdx.x == 0 ) {
      for( int k = 0; k < ( m + 1 ) * m; k++ )
         g.H[ k ] = 0.0;
      for( int k = 0; k <= m; k++ )
         g.sv[ k ] = 0.0;
      g.sv[ 0 ] = beta;
      c.m = m;
      c.o_steps = m;
      c.cycle_stop = 0;
      // head of step 0: nextIteration() (GMRES.hpp:297)
      const bool go = check_next( c );
      c.it++;
      if( ! go ) {
         c.cycle_stop = 1;
         c.o_steps = 0;
      }
   }
}

// Givens rotations for column i, residue, and the tail check of step i
// (GMRES.hpp:330-344, 751-763). Runs in one thread.
__device__ void
gm_finish_step( Ctl& c, GmArrays g, int i, int m, double normw )
{
   double* Hc = g.H + i * ( m + 1 );
   Hc[ i + 1 ] = normw;
   c.normw = normw;
   for( int k = 0; k < i; k++ )
      apply_plane_rotation( Hc[ k ], Hc[ k + 1 ], g.cs[ k ], g.sn[ k ] );
   if( Hc[ i + 1 ] != 0.0 ) {
      gen_plane_rotation( Hc[ i ], Hc[ i + 1 ], g.cs[ i ], g.sn[ i ] );
      apply_plane_rotation( Hc[ i ], Hc[ i + 1 ], g.cs[ i ], g.sn[ i ] );
      apply_plane_rotation( g.sv[ i ], g.sv[ i + 1 ], g.cs[ i ], g.sn[ i ] );
   }
   c.residue = fabs( g.sv[ i + 1 ] ) / c.normb;
   if( ! check_next( c ) ) {
      c.cycle_stop = 1;
      c.o_steps = i;
      return;
   }
   if( i + 1 < m ) {
      // head of step i+1: nextIteration() — the check has just passed
      c.it++;
   }
   else {
      c.cycle_stop = 1;  // the for-loop ends by i < m
      c.o_steps = m;
   }
}

// MGS projection step k of pass l: w -= h_prev v_prev ; acc += (w, v_k)
template< typename Real >
struct GmMgsOp
{
   static constexpr int NR = 1;
   Real* w;
   const Real *vprev, *vk;
   const double* hprev_ptr;
   Real hprev;
   __device__ __forceinline__ void load( const Ctl& ) { hprev = vprev ? (Real) *hprev_ptr : Real( 0 ); }
   __device__ __forceinline__ void
   operator()( int64_t j, double* acc ) const
   {
      Real t = w[ j ];
      if( vprev ) {
         t = t - hprev * vprev[ j ];
         w[ j ] = t;
      }
      acc[ 0 ] += (double) t * (double) vk[ j ];
   }
};

struct GmMgsFin
{
   static constexpr bool active = true;
   GmArrays g;
   int k, i, m;
   __device__ void
   operator()( Ctl&, const double* t ) const
   {
      g.hl[ k ] = t[ 0 ];
      g.H[ k + i * ( m + 1 ) ] += t[ 0 ];
   }
};

// last MGS step: w -= h_i v_i ; acc += (w, w) -> normw, Givens, tail check
template< typename Real >
struct GmMgsLastOp
{
   static constexpr int NR = 1;
   Real* w;
   const Real* vi;
   const double* h_ptr;
   Real h;
   __device__ __forceinline__ void load( const Ctl& ) { h = (Real) *h_ptr; }
   __device__ __forceinline__ void
   operator()( int64_t j, double* acc ) const
   {
      const Real t = w[ j ] - h * vi[ j ];
      w[ j ] = t;
      acc[ 0 ] += (double) t * (double) t;
   }
};

struct GmNormFin
{
   static constexpr bool active = true;
   GmArrays g;
   int i, m;
   __device__ void operator()( Ctl& c, const double* t ) const { gm_finish_step( c, g, i, m, sqrt( t[ 0 ] ) ); }
};

// Gated vector kernel for the Arnoldi loop (skips when the cycle stopped).
template< typename Real, class Op, class Fin >
__global__ void __launch_bounds__( kReduceBlock )
arn_kernel( int64_t n, Ctl* ctl, Op op, Fin fin, RedScratch rs )
{
   if( ctl->cycle_stop || ctl->done )
      return;
   op.load( *ctl );
   double acc[ Op::NR ];
#pragma unroll
   for( int k = 0; k < Op::NR; k++ )
      acc[ k ] = 0.0;
   for( int64_t i = blockIdx.x * (int64_t) kReduceBlock + threadIdx.x; i < n; i += (int64_t) gridDim.x * kReduceBlock )
      op( i, acc );
   if constexpr( Fin::active ) {
      double tot[ Op::NR ];
      if( grid_reduce< Op::NR, kReduceBlock >( acc, rs, tot ) && threadIdx.x == 0 )
         fin( *ctl, tot );
   }
}

// Four elements of a column per thread step: 32 bytes (FP64) or 16 bytes
// (FP32; eight FP32 elements per step needed 122 registers in the projection
// kernel and measured slower). Columns start on 128-byte boundaries.
template< typename Real >
struct GsStep
{
   static constexpr int W = 4;
   Real v[ W ];
};
__device__ __forceinline__ GsStep< double >
ld_step( const double* p )
{
   const double2 a = reinterpret_cast< const double2* >( p )[ 0 ], b = reinterpret_cast< const double2* >( p )[ 1 ];
   return { { a.x, a.y, b.x, b.y } };
}
__device__ __forceinline__ GsStep< float >
ld_step( const float* p )
{
   const float4 a = *reinterpret_cast< const float4* >( p );
   return { { a.x, a.y, a.z, a.w } };
}
__device__ __forceinline__ void
st_step( double* p, const GsStep< double >& a )
{
   reinterpret_cast< double2* >( p )[ 0 ] = make_double2( a.v[ 0 ], a.v[ 1 ] );
   reinterpret_cast< double2* >( p )[ 1 ] = make_double2( a.v[ 2 ], a.v[ 3 ] );
}
__device__ __forceinline__ void
st_step( float* p, const GsStep< float >& a )
{
   *reinterpret_cast< float4* >( p ) = make_float4( a.v[ 0 ], a.v[ 1 ], a.v[ 2 ], a.v[ 3 ] );
}

// sum of the four products of one step in pairs, in FP64
template< int W >
__device__ __forceinline__ double
step_dot( const double* a, const double* b )
{
   static_assert( W == 4, "four elements per step" );
   return ( a[ 0 ] * b[ 0 ] + a[ 1 ] * b[ 1 ] ) + ( a[ 2 ] * b[ 2 ] + a[ 3 ] * b[ 3 ] );
}

// four FP32 products summed in FP32 (fused), one FP64 conversion per step:
// FP32 basis passes that converted every product were bound by FP64-pipe
// instructions at half the bytes of the FP64 passes
__device__ __forceinline__ float
step_dot32( const float* a, const float* b )
{
   float s = a[ 0 ] * b[ 0 ];
   s = __fmaf_rn( a[ 1 ], b[ 1 ], s );
   s = __fmaf_rn( a[ 2 ], b[ 2 ], s );
   return __fmaf_rn( a[ 3 ], b[ 3 ], s );
}

// CGS projections: hl[k0+c] = (V_{k0+c}, w) for c < nk (<= NK <= 16 per launch),
// accumulated in FP64 (FP32 storage: in FP64 over four-element FP32 partial sums).
// NK (1, 2, 4, 8 or 16) sizes the accumulators and the block reduction to the
// columns of the launch: the early steps of a cycle project on one to a few
// columns, where a 16-value reduction per block had cost more than the loads.
// At least three resident blocks per SM (at most 85 registers): the batched
// column loads had taken the FP32 kernel to 128 registers and two blocks.
constexpr int kMd = 16;
template< typename Real, int NK >
__global__ void __launch_bounds__( kReduceBlock, 3 )
gm_multidot_kernel( int64_t n, int64_t ld, Ctl* ctl, const Real* __restrict__ V, const Real* __restrict__ w, int k0,
                    int nk, GmArrays g, int i, int m, RedScratch rs )
{
   static_assert( NK >= 1 && NK <= kMd, "columns per launch" );
   if( ctl->cycle_stop || ctl->done )
      return;
   constexpr int W = GsStep< Real >::W;
   double acc[ NK ];
#pragma unroll
   for( int c = 0; c < NK; c++ )
      acc[ c ] = 0.0;
   // four elements of w and of every column per step; the column base pointers stay in registers
   const Real* Vb = V + (int64_t) k0 * ld;
   const int64_t nw = n / W, t0 = blockIdx.x * (int64_t) kReduceBlock + threadIdx.x,
                 step = (int64_t) gridDim.x * kReduceBlock;
   for( int64_t q = t0; q < nw; q += step ) {
      const GsStep< Real > wv = ld_step( w + W * q );
      if constexpr( std::is_same< Real, float >::value ) {
         // up to eight columns' steps are loaded before their products, so a
         // thread keeps up to nine loads in flight (one column at a time left
         // the FP32 pass latency-bound: 38 long-scoreboard stalls per issue)
#pragma unroll
         for( int c0 = 0; c0 < NK; c0 += 8 ) {
            GsStep< Real > vv[ 8 ];
#pragma unroll
            for( int cc = 0; cc < 8; cc++ )
               if( c0 + cc < NK && c0 + cc < nk )
                  vv[ cc ] = ld_step( Vb + ( c0 + cc ) * ld + W * q );
#pragma unroll
            for( int cc = 0; cc < 8; cc++ )
               if( c0 + cc < NK && c0 + cc < nk )
                  acc[ c0 + cc ] += (double) step_dot32( vv[ cc ].v, wv.v );
         }
      }
      else {
         double wd[ W ];
#pragma unroll
         for( int u = 0; u < W; u++ )
            wd[ u ] = (double) wv.v[ u ];
         // columns in batches of four loads in flight
#pragma unroll
         for( int c0 = 0; c0 < NK; c0 += 4 ) {
            GsStep< Real > vv[ 4 ];
#pragma unroll
            for( int cc = 0; cc < 4; cc++ )
               if( c0 + cc < NK && c0 + cc < nk )
                  vv[ cc ] = ld_step( Vb + ( c0 + cc ) * ld + W * q );
#pragma unroll
            for( int cc = 0; cc < 4; cc++ )
               if( c0 + cc < NK && c0 + cc < nk ) {
                  double vd[ W ];
#pragma unroll
                  for( int u = 0; u < W; u++ )
                     vd[ u ] = (double) vv[ cc ].v[ u ];
                  acc[ c0 + cc ] += step_dot< W >( vd, wd );
               }
         }
      }
   }
   for( int64_t j = W * nw + t0; j < n; j += step ) {
      const double wj = (double) w[ j ];
#pragma unroll
      for( int c = 0; c < NK; c++ )
         if( c < nk )
            acc[ c ] += (double) Vb[ c * ld + j ] * wj;
   }
   double tot[ NK ];
   if( grid_reduce< NK, kReduceBlock >( acc, rs, tot ) && threadIdx.x == 0 ) {
      for( int c = 0; c < nk; c++ ) {
         g.hl[ k0 + c ] = tot[ c ];
         g.H[ k0 + c + i * ( m + 1 ) ] += tot[ c ];
      }
   }
}

// CGS update: w = w - V_i hl (gemv with alpha = -1, beta = 1, MatrixOperations.h:46-120),
// summed in FP64 (FP32 storage: over FP32 partial sums of four columns) and
// rounded once to the storage type; on the last pass also ||w||^2 -> normw,
// Givens, tail check.
// One step of the update: w[4q .. 4q+3] -= V_i hl (coef = -hl, coef32 its
// FP32 copy), stored and returned
template< typename Real >
__device__ __forceinline__ GsStep< Real >
gs_update_step( const Real* __restrict__ V, int64_t ld, Real* __restrict__ w, int64_t q, int i, const double* coef,
                const float* coef32 )
{
   constexpr int W = GsStep< Real >::W;
   double aux[ W ];
#pragma unroll
   for( int u = 0; u < W; u++ )
      aux[ u ] = 0.0;
   if constexpr( std::is_same< Real, float >::value ) {
      // eight columns' loads in flight, then their two four-column FP32 partial sums
      for( int k0 = 0; k0 <= i; k0 += 8 ) {
         GsStep< Real > vv[ 8 ];
#pragma unroll
         for( int kk = 0; kk < 8; kk++ )
            if( k0 + kk <= i )
               vv[ kk ] = ld_step( V + ( k0 + kk ) * ld + W * q );
#pragma unroll
         for( int h = 0; h < 2; h++ ) {
            float part[ W ] = { 0.f, 0.f, 0.f, 0.f };
#pragma unroll
            for( int kk = 4 * h; kk < 4 * h + 4; kk++ )
               if( k0 + kk <= i ) {
                  const float ck = coef32[ k0 + kk ];
#pragma unroll
                  for( int u = 0; u < W; u++ )
                     part[ u ] = __fmaf_rn( vv[ kk ].v[ u ], ck, part[ u ] );
               }
#pragma unroll
            for( int u = 0; u < W; u++ )
               aux[ u ] += (double) part[ u ];
         }
      }
   }
   else {
      // four columns' loads in flight, then their products in column order
      for( int k0 = 0; k0 <= i; k0 += 4 ) {
         GsStep< Real > vv[ 4 ];
#pragma unroll
         for( int kk = 0; kk < 4; kk++ )
            if( k0 + kk <= i )
               vv[ kk ] = ld_step( V + ( k0 + kk ) * ld + W * q );
#pragma unroll
         for( int kk = 0; kk < 4; kk++ )
            if( k0 + kk <= i ) {
               const double ck = coef[ k0 + kk ];
#pragma unroll
               for( int u = 0; u < W; u++ )
                  aux[ u ] += (double) vv[ kk ].v[ u ] * ck;
            }
      }
   }
   GsStep< Real > wv = ld_step( w + W * q );
#pragma unroll
   for( int u = 0; u < W; u++ )
      wv.v[ u ] = (Real) ( aux[ u ] + (double) wv.v[ u ] );
   st_step( w + W * q, wv );
   return wv;
}

// one element of the update (the n % 4 tail)
template< typename Real >
__device__ __forceinline__ Real
gs_update_elem( const Real* __restrict__ V, int64_t ld, Real* __restrict__ w, int64_t j, int i, const double* coef )
{
   double aux = 0;
   for( int k = 0; k <= i; k++ )
      aux += (double) V[ k * ld + j ] * coef[ k ];
   const Real t = (Real) ( aux + (double) w[ j ] );
   w[ j ] = t;
   return t;
}

template< typename Real >
__device__ __forceinline__ void
gs_load_coef( const GmArrays& g, int i, double* coef, float* coef32 )
{
   for( int k = threadIdx.x; k <= i; k += kReduceBlock ) {
      coef[ k ] = -g.hl[ k ];
      coef32[ k ] = (float) coef[ k ];
   }
   __syncthreads();
}

template< typename Real, bool LAST >
__global__ void __launch_bounds__( kReduceBlock )
gm_cgs_update_kernel( int64_t n, int64_t ld, Ctl* ctl, const Real* __restrict__ V, Real* __restrict__ w, int i, int m,
                      GmArrays g, RedScratch rs )
{
   if( ctl->cycle_stop || ctl->done )
      return;
   constexpr int W = GsStep< Real >::W;
   __shared__ double coef[ 256 ];
   __shared__ float coef32[ 256 ];
   gs_load_coef< Real >( g, i, coef, coef32 );
   double acc[ 1 ] = { 0.0 };
   // four elements of every basis column per step
   const int64_t nw = n / W, t0 = blockIdx.x * (int64_t) kReduceBlock + threadIdx.x,
                 step = (int64_t) gridDim.x * kReduceBlock;
   for( int64_t q = t0; q < nw; q += step ) {
      const GsStep< Real > wv = gs_update_step< Real >( V, ld, w, q, i, coef, coef32 );
#pragma unroll
      for( int u = 0; u < W; u++ )
         acc[ 0 ] += (double) wv.v[ u ] * (double) wv.v[ u ];
   }
   for( int64_t j = W * nw + t0; j < n; j += step ) {
      const Real t = gs_update_elem< Real >( V, ld, w, j, i, coef );
      acc[ 0 ] += (double) t * (double) t;
   }
   if constexpr( LAST ) {
      double tot[ 1 ];
      if( grid_reduce< 1, kReduceBlock >( acc, rs, tot ) && threadIdx.x == 0 )
         gm_finish_step( *ctl, g, i, m, sqrt( tot[ 0 ] ) );
   }
}

// CGSR: the first pass's update w -= V_i hl fused with the second pass's
// projections on columns 0 .. nk-1 (nk <= NK <= 16): each step of the updated
// w is dotted with those columns as soon as it is formed. The columns were
// just read for the update, so the second read is served by the caches and
// the pass over V that the second projections would make from HBM goes away
// (for i >= 16 the remaining columns get their own projection launch). The
// pass-0 coefficients are read from hl into shared memory before any block
// arrives at the grid reduction, whose last block then writes the pass-1
// projections into hl and adds them to H.
template< typename Real, int NK >
__global__ void __launch_bounds__( kReduceBlock )
gm_cgs_update_dot_kernel( int64_t n, int64_t ld, Ctl* ctl, const Real* __restrict__ V, Real* __restrict__ w, int i,
                          int nk, int m, GmArrays g, RedScratch rs )
{
   static_assert( NK >= 1 && NK <= kMd, "columns per launch" );
   if( ctl->cycle_stop || ctl->done )
      return;
   constexpr int W = GsStep< Real >::W;
   __shared__ double coef[ 256 ];
   __shared__ float coef32[ 256 ];
   gs_load_coef< Real >( g, i, coef, coef32 );
   double acc[ NK ];
#pragma unroll
   for( int c = 0; c < NK; c++ )
      acc[ c ] = 0.0;
   const int64_t nw = n / W, t0 = blockIdx.x * (int64_t) kReduceBlock + threadIdx.x,
                 step = (int64_t) gridDim.x * kReduceBlock;
   for( int64_t q = t0; q < nw; q += step ) {
      const GsStep< Real > wv = gs_update_step< Real >( V, ld, w, q, i, coef, coef32 );
      if constexpr( std::is_same< Real, float >::value ) {
         // the columns come back from the caches: batches of four loads keep
         // the registers (and the resident blocks) of the update
#pragma unroll
         for( int c0 = 0; c0 < NK; c0 += 4 ) {
            GsStep< Real > vv[ 4 ];
#pragma unroll
            for( int cc = 0; cc < 4; cc++ )
               if( c0 + cc < NK && c0 + cc < nk )
                  vv[ cc ] = ld_step( V + ( c0 + cc ) * ld + W * q );
#pragma unroll
            for( int cc = 0; cc < 4; cc++ )
               if( c0 + cc < NK && c0 + cc < nk )
                  acc[ c0 + cc ] += (double) step_dot32( vv[ cc ].v, wv.v );
         }
      }
      else {
         double wd[ W ];
#pragma unroll
         for( int u = 0; u < W; u++ )
            wd[ u ] = (double) wv.v[ u ];
         // columns in batches of four loads in flight
#pragma unroll
         for( int c0 = 0; c0 < NK; c0 += 4 ) {
            GsStep< Real > vv[ 4 ];
#pragma unroll
            for( int cc = 0; cc < 4; cc++ )
               if( c0 + cc < NK && c0 + cc < nk )
                  vv[ cc ] = ld_step( V + ( c0 + cc ) * ld + W * q );
#pragma unroll
            for( int cc = 0; cc < 4; cc++ )
               if( c0 + cc < NK && c0 + cc < nk ) {
                  double vd[ W ];
#pragma unroll
                  for( int u = 0; u < W; u++ )
                     vd[ u ] = (double) vv[ cc ].v[ u ];
                  acc[ c0 + cc ] += step_dot< W >( vd, wd );
               }
         }
      }
   }
   for( int64_t j = W * nw + t0; j < n; j += step ) {
      const double wj = (double) gs_update_elem< Real >( V, ld, w, j, i, coef );
#pragma unroll
      for( int c = 0; c < NK; c++ )
         if( c < nk )
            acc[ c ] += (double) V[ c * ld + j ] * wj;
   }
   double tot[ NK ];
   if( grid_reduce< NK, kReduceBlock >( acc, rs, tot ) && threadIdx.x == 0 ) {
      for( int c = 0; c < nk; c++ ) {
         g.hl[ c ] = tot[ c ];
         g.H[ c + i * ( m + 1 ) ] += tot[ c ];
      }
   }
}

// v_{i+1} = (1 / normw) w
template< typename Real >
__global__ void
gm_normalize_kernel( int64_t n, Ctl* ctl, Real* __restrict__ vn, const Real* __restrict__ w )
{
   const Ctl& c = *ctl;
   if( c.cycle_stop || c.done )
      return;
   const Real scale = (Real) ( 1.0 / c.normw );
   for( int64_t j = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; j < n; j += (int64_t) gridDim.x * blockDim.x )
      vn[ j ] = scale * w[ j ];
}

// Back substitution of the update (GMRES.hpp:641-664); one thread.
__global__ void
gm_backsolve_kernel( Ctl* ctl, GmArrays g )
{
   Ctl& c = *ctl;
   if( c.done || threadIdx.x != 0 || blockIdx.x != 0 )
      return;
   const int m = c.m;
   const int k = c.o_steps < m ? c.o_steps : m - 1;
   for( int i = 0; i <= m; i++ )
      g.y[ i ] = g.sv[ i ];
   for( int i = k; i >= 0; i-- ) {
      const double d = g.H[ i + i * ( m + 1 ) ];
      if( d == 0.0 ) {
         c.reason = 3;
         c.done = 1;
         return;
      }
      g.y[ i ] /= d;
      for( int j = i - 1; j >= 0; j-- )
         g.y[ j ] -= g.H[ j + i * ( m + 1 ) ] * g.y[ i ];
   }
}

// x = V_{0..k} y + x
template< typename Real >
__global__ void
gm_xupdate_kernel( int64_t n, int64_t ld, Ctl* ctl, const Real* __restrict__ V, Real* __restrict__ x, GmArrays g )
{
   const Ctl& c = *ctl;
   if( c.done )
      return;
   const int m = c.m;
   const int k = c.o_steps < m ? c.o_steps : m - 1;
   __shared__ Real coef[ 256 ];
   for( int q = threadIdx.x; q <= k; q += blockDim.x )
      coef[ q ] = (Real) g.y[ q ];
   __syncthreads();
   for( int64_t j = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; j < n; j += (int64_t) gridDim.x * blockDim.x ) {
      Real aux = 0;
      for( int q = 0; q <= k; q++ )
         aux += V[ q * ld + j ] * coef[ q ];
      x[ j ] = aux + x[ j ];
   }
}

}  // namespace b2s

using namespace b2s;

// ---------------------------------------------------------------------------
// Solver handle
struct b2s_solver_t
{
   b2s_matrix_t* A = nullptr;
   b2s_matrix_t* expanded = nullptr;  // owned: L + L^T - D when the caller's matrix is a SymmetricMatrix
   b2s_solve_opts o{};
   cudaStream_t cs = nullptr;
   bool owns_stream = true;  // false: stream and events lent by a server worker
   bool mixed = false;
   int n = 0;

   DevBuf ctl_buf;
   Ctl* h_ctl = nullptr;  // host mirror of the control block
   bool h_ctl_pinned = false;
   Scratch scr;           // reduction scratch (slots)
   DevBuf md_partials;    // multi-dot partials (16 per block)
   DevBuf md_counter;

   // working vectors in the Krylov precision
   DevBuf vecs;
   DevBuf diag32;
   // ILU(0) factors (preconditioner B2S_PRECOND_ILU0), in the matrix's value type
   IluFactors< double > ilu64;
   IluFactors< float > ilu32;
   // SOR sweep plan (solver B2S_SOR), in the matrix's value type
   SorPlan< double > sor64;
   SorPlan< float > sor32;
   // FP64 outer vectors (mixed)
   DevBuf outer;

   // GMRES
   DevBuf gm;
   DevBuf V;
   int64_t ld = 0;
   int mmax = 0;

   std::map< long long, cudaGraphExec_t > graphs;
   std::map< long long, cudaGraph_t > graph_defs;
   cudaEvent_t ev0 = nullptr, ev1 = nullptr;
   std::chrono::steady_clock::time_point t_start;

   ~b2s_solver_t()
   {
      for( auto& kv : graphs )
         cudaGraphExecDestroy( kv.second );
      for( auto& kv : graph_defs )
         cudaGraphDestroy( kv.second );
      if( h_ctl && h_ctl_pinned )
         cudaFreeHost( h_ctl );
      else
         delete h_ctl;
      delete expanded;
      if( owns_stream ) {
         if( ev0 )
            cudaEventDestroy( ev0 );
         if( ev1 )
            cudaEventDestroy( ev1 );
         if( cs )
            cudaStreamDestroy( cs );
      }
   }
};

namespace b2s {

static int
vgrid( int64_t n )
{
   return reduce_grid( n, 4 );
}

// The grid-stride vector and reduction kernels run one wave of resident
// blocks (at most vgrid( n )): every block takes the same share of the
// vector and does one block-level reduction, with no partial last wave —
// for kernels whose registers allow fewer than eight blocks per SM (the
// four-accumulator updates, the 16-column projections) a grid of 8 per SM
// ran in two to four waves. Measured on GMRES(30) in FP32: projections at
// 4 blocks per SM (one wave) 96 ms against 103 ms (8 per SM) and 112 ms
// (2 per SM).
template< typename K >
static int
wave_grid( K kernel, int64_t n )
{
   const int per_sm = resident_blocks( reinterpret_cast< const void* >( kernel ), kReduceBlock );
   return std::max( 1, std::min( vgrid( n ), num_sms() * per_sm ) );
}

template< typename Real >
struct KrylovVecs
{
   Real *b, *x, *r, *p, *Ap, *z, *r_ast, *s, *As, *w;
};

template< typename Real >
static KrylovVecs< Real >
vec_layout( b2s_solver_t* S )
{
   const int64_t ln = ( (int64_t) S->n + 63 ) / 64 * 64;
   Real* base = S->vecs.as< Real >();
   KrylovVecs< Real > v;
   Real** slots[] = { &v.b, &v.x, &v.r, &v.p, &v.Ap, &v.z, &v.r_ast, &v.s, &v.As, &v.w };
   for( int i = 0; i < 10; i++ )
      *slots[ i ] = base + i * ln;
   return v;
}

// Capture `body` into a graph (cached under `key`) and launch it on the solver stream.
// the solver's ILU(0) factors in Real, or NULL (no ILU preconditioner)
template< typename Real >
static const IluFactors< Real >*
ilu_of( const b2s_solver_t* S )
{
   if( S->o.preconditioner != B2S_PRECOND_ILU0 && S->o.preconditioner != B2S_PRECOND_ILUT )
      return nullptr;
   if constexpr( std::is_same< Real, double >::value )
      return &S->ilu64;
   else
      return &S->ilu32;
}

// An SpMV through `sink` with M = ILU(0) applied in between: the SpMV stores
// b - A x (b != NULL) or A x into `out`, M^-1 is applied in place, and the
// sink's own pass (pre = 1) runs on the result; every step is skipped with
// the sink.
template< typename Real, class Sink >
static b2s_status
prec_spmv( b2s_solver_t* S, const IluFactors< Real >& ilu, const Real* vals, const Real* xin, const Real* b, Real* out,
           Sink sink, RedScratch rs )
{
   sink.pre = 1;
   StoreSink< Real, Sink > st{ out, b, sink };
   B2S_TRY( ( spmv_dispatch< Real, StoreSink< Real, Sink > >( S->A, vals, xin, 0, S->A->rows, st, RedScratch{}, S->cs ) ) );
   B2S_TRY( ilu.apply( out, out, S->cs, sink ) );
   sink_post_kernel< Real, Sink ><<< wave_grid( sink_post_kernel< Real, Sink >, S->n ), kReduceBlock, 0, S->cs >>>( S->n, out, sink, rs );
   B2S_TRY_CUDA( cudaGetLastError() );
   return B2S_OK;
}

template< class F >
static b2s_status
run_graph( b2s_solver_t* S, long long key, F&& body )
{
   if( S->o.graphs == 1 )
      return body();  // direct launches on the solver stream
   auto it = S->graphs.find( key );
   if( it == S->graphs.end() ) {
      cudaGraph_t g = nullptr;
      B2S_TRY_CUDA( cudaStreamBeginCapture( S->cs, cudaStreamCaptureModeThreadLocal ) );
      b2s_status st = body();
      cudaError_t e = cudaStreamEndCapture( S->cs, &g );
      if( st != B2S_OK ) {
         if( g )
            cudaGraphDestroy( g );
         return st;
      }
      B2S_TRY_CUDA( e );
      cudaGraphExec_t ge = nullptr;
      B2S_TRY_CUDA( cudaGraphInstantiate( &ge, g, 0 ) );
      S->graph_defs[ key ] = g;
      it = S->graphs.emplace( key, ge ).first;
   }
   B2S_TRY_CUDA( cudaGraphLaunch( it->second, S->cs ) );
   return B2S_OK;
}

// Host-side bound on one solve: the polling loops end with B2S_TIMEOUT
// instead of running forever if the device never reports completion.
constexpr double kMaxSolveSeconds = 1800.0;

static b2s_status
check_wall( b2s_solver_t* S )
{
   const double s = std::chrono::duration< double >( std::chrono::steady_clock::now() - S->t_start ).count();
   if( s > kMaxSolveSeconds ) {
      set_error( "solve exceeded %.0f s without the device reporting completion", kMaxSolveSeconds );
      return B2S_TIMEOUT;
   }
   return B2S_OK;
}

static b2s_status
read_ctl( b2s_solver_t* S )
{
   B2S_TRY_CUDA( cudaMemcpyAsync( S->h_ctl, S->ctl_buf.p, sizeof( Ctl ), cudaMemcpyDeviceToHost, S->cs ) );
   B2S_TRY_CUDA( cudaStreamSynchronize( S->cs ) );
   return B2S_OK;
}

static b2s_status
read_done( b2s_solver_t* S, int& done )
{
   Ctl* d = S->ctl_buf.as< Ctl >();
   B2S_TRY_CUDA( cudaMemcpyAsync( &S->h_ctl->done, &d->done, sizeof( int ), cudaMemcpyDeviceToHost, S->cs ) );
   B2S_TRY_CUDA( cudaStreamSynchronize( S->cs ) );
   done = S->h_ctl->done;
   return B2S_OK;
}

static b2s_status
init_ctl( b2s_solver_t* S, double tol, long long maxit )
{
   Ctl c{};
   c.tol = tol;
   c.div_tol = S->o.divergence_residue;
   c.maxit = maxit;
   c.minit = S->o.min_iterations;
   *S->h_ctl = c;
   B2S_TRY_CUDA( cudaMemcpyAsync( S->ctl_buf.p, S->h_ctl, sizeof( Ctl ), cudaMemcpyHostToDevice, S->cs ) );
   return B2S_OK;
}

// IterativeSolver::checkConvergence (IterativeSolver.hpp:121-146) as a status
static b2s_status
convergence_status( const Ctl& c )
{
   if( c.reason == 3 )
      return B2S_BREAKDOWN;
   if( std::isnan( c.residue ) )
      return B2S_NAN;
   if( c.residue > c.div_tol && c.it > c.minit )
      return B2S_DIVERGED;
   if( c.it >= c.maxit )
      return B2S_NOT_CONVERGED;
   if( c.residue > c.tol )
      return B2S_NOT_CONVERGED;
   return B2S_OK;
}

static bool
host_check_next( const Ctl& c )
{
   return ! ( std::isnan( c.residue ) || c.it > c.maxit || ( c.residue > c.div_tol && c.it >= c.minit )
              || ( c.residue < c.tol && c.it >= c.minit ) );
}

static int
chunk_of( const b2s_solver_t* S )
{
   if( S->o.check_interval > 0 )
      return S->o.check_interval;
   const int64_t work = S->A->nnz + 10LL * S->n;
   if( work < 2000000 )
      return 32;
   if( work < 20000000 )
      return 8;
   return 4;
}

// ---------------------------------------------------------------------------
// The Krylov loops. `vals` are A's values in Real, `diag` the Jacobi diagonal
// in Real (NULL: unpreconditioned). b and x are solver-owned device vectors.
template< typename Real >
static b2s_status
normb_launch( b2s_solver_t* S, const Real* b, const Real* diag )
{
   if( const IluFactors< Real >* ilu = ilu_of< Real >( S ) ) {
      // ||M^-1 b|| with M^-1 b in z (free before the iterations start)
      Real* z = vec_layout< Real >( S ).z;
      B2S_TRY( ilu->apply( b, z, S->cs ) );
      b = z;
   }
   Ctl* ctl = S->ctl_buf.as< Ctl >();
   vec_kernel< Real, NormOp< Real >, NormbFin ><<< wave_grid( vec_kernel< Real, NormOp< Real >, NormbFin >, S->n ), kReduceBlock, 0, S->cs >>>(
      S->n, ctl, NormOp< Real >{ b, diag }, NormbFin{}, S->scr.slot( 0 ) );
   B2S_TRY_CUDA( cudaGetLastError() );
   return B2S_OK;
}

template< typename Real >
static b2s_status cg_iterate( b2s_solver_t* S, const Real* vals, const Real* diag, long long tagbase );

template< typename Real >
static b2s_status
cg_core( b2s_solver_t* S, const Real* vals, const Real* diag, long long tagbase )
{
   const b2s_matrix_t* A = S->A;
   const int64_t n = S->n;
   auto v = vec_layout< Real >( S );
   Ctl* ctl = S->ctl_buf.as< Ctl >();
   B2S_TRY( normb_launch< Real >( S, v.b, diag ) );
   if( const IluFactors< Real >* ilu = ilu_of< Real >( S ) ) {
      // r = b - A x ; z = M^-1 r ; p = z ; s1 = (r, z)
      StoreSink< Real, NoGate > st{ v.r, v.b, NoGate{} };
      B2S_TRY( ( spmv_dispatch< Real, StoreSink< Real, NoGate > >( A, vals, v.x, 0, A->rows, st, RedScratch{}, S->cs ) ) );
      B2S_TRY( ilu->apply( v.r, v.z, S->cs ) );
      vec_kernel< Real, CgPrecInitOp< Real >, CgInitFin ><<< wave_grid( vec_kernel< Real, CgPrecInitOp< Real >, CgInitFin >, n ), kReduceBlock, 0, S->cs >>>(
         n, ctl, CgPrecInitOp< Real >{ v.r, v.z, v.p }, CgInitFin{}, S->scr.slot( 1 ) );
      B2S_TRY_CUDA( cudaGetLastError() );
      return cg_iterate< Real >( S, vals, diag, tagbase );
   }
   {
      CgInitG< Real > sink;
      sink.b = v.b;
      sink.r = v.r;
      sink.z = v.z;
      sink.p = v.p;
      sink.diag = diag;
      sink.ctl = ctl;
      B2S_TRY( ( spmv_dispatch< Real, CgInitG< Real > >( A, vals, v.x, 0, A->rows, sink, S->scr.slot( 1 ), S->cs ) ) );
   }
   return cg_iterate< Real >( S, vals, diag, tagbase );
}

// CG iterations (CG.hpp:60-101) in graph chunks until the device says done
template< typename Real >
static b2s_status
cg_iterate( b2s_solver_t* S, const Real* vals, const Real* diag, long long tagbase )
{
   const b2s_matrix_t* A = S->A;
   const int64_t n = S->n;
   auto v = vec_layout< Real >( S );
   Ctl* ctl = S->ctl_buf.as< Ctl >();
   const IluFactors< Real >* ilu = ilu_of< Real >( S );
   const int chunk = chunk_of( S );
   for( ;; ) {
      B2S_TRY( run_graph( S, tagbase + chunk, [ & ]() -> b2s_status
      {
         for( int k = 0; k < chunk; k++ ) {
            CgApG< Real > ap;
            ap.Ap = v.Ap;
            ap.p = v.p;
            ap.ctl = ctl;
            B2S_TRY( ( spmv_dispatch< Real, CgApG< Real > >( A, vals, v.p, 0, A->rows, ap, S->scr.slot( 2 ), S->cs ) ) );
            if( ilu ) {
               // x, r updates ; z = M^-1 r ; (r, z) -> beta, residue
               CgUpdateOp< Real > up{ v.x, v.r, v.z, v.p, v.Ap, nullptr, Real( 0 ) };
               vec_kernel< Real, CgUpdateOp< Real >, NoFin ><<< wave_grid( vec_kernel< Real, CgUpdateOp< Real >, NoFin >, n ), kReduceBlock, 0, S->cs >>>(
                  n, ctl, up, NoFin{}, S->scr.slot( 3 ) );
               B2S_TRY_CUDA( cudaGetLastError() );
               B2S_TRY( ilu->apply( v.r, v.z, S->cs, DoneGate{ ctl } ) );
               vec_kernel< Real, DotOp< Real >, CgUpdateFin ><<< wave_grid( vec_kernel< Real, DotOp< Real >, CgUpdateFin >, n ), kReduceBlock, 0, S->cs >>>(
                  n, ctl, DotOp< Real >{ v.r, v.z }, CgUpdateFin{}, S->scr.slot( 3 ) );
               B2S_TRY_CUDA( cudaGetLastError() );
            }
            else {
               CgUpdateOp< Real > up{ v.x, v.r, v.z, v.p, v.Ap, diag, Real( 0 ) };
               vec_kernel< Real, CgUpdateOp< Real >, CgUpdateFin ><<< wave_grid( vec_kernel< Real, CgUpdateOp< Real >, CgUpdateFin >, n ), kReduceBlock, 0, S->cs >>>(
                  n, ctl, up, CgUpdateFin{}, S->scr.slot( 3 ) );
               B2S_TRY_CUDA( cudaGetLastError() );
            }
            CgDirOp< Real > dir{ v.p, ( diag || ilu ) ? v.z : v.r, Real( 0 ) };
            vec_kernel< Real, CgDirOp< Real >, NoFin ><<< wave_grid( vec_kernel< Real, CgDirOp< Real >, NoFin >, n ), kReduceBlock, 0, S->cs >>>(
               n, ctl, dir, NoFin{}, S->scr.slot( 4 ) );
            B2S_TRY_CUDA( cudaGetLastError() );
         }
         return B2S_OK;
      } ) );
      int done = 0;
      B2S_TRY( read_done( S, done ) );
      if( done )
         break;
      B2S_TRY( check_wall( S ) );
   }
   return B2S_OK;
}

template< typename Real >
static b2s_status bicgstab_iterate( b2s_solver_t* S, const Real* vals, const Real* diag, long long tagbase );

template< typename Real >
static b2s_status
bicgstab_core( b2s_solver_t* S, const Real* vals, const Real* diag, long long tagbase )
{
   const b2s_matrix_t* A = S->A;
   auto v = vec_layout< Real >( S );
   Ctl* ctl = S->ctl_buf.as< Ctl >();
   const int exact = S->o.bicgstab_exact_residue != 0;
   B2S_TRY( normb_launch< Real >( S, v.b, diag ) );
   auto res_sink = [ & ]( int mode, Real* target ) {
      BiResG< Real > s;
      s.b = v.b;
      s.r = target;
      s.r_ast = v.r_ast;
      s.p = v.p;
      s.s = v.s;
      s.diag = diag;
      s.ctl = ctl;
      s.mode = mode;
      s.exact = exact;
      return s;
   };
   if( const IluFactors< Real >* ilu = ilu_of< Real >( S ) )
      B2S_TRY( prec_spmv< Real >( S, *ilu, vals, v.x, v.b, v.r, res_sink( 0, v.r ), S->scr.slot( 1 ) ) );
   else
      B2S_TRY( ( spmv_dispatch< Real, BiResG< Real > >( A, vals, v.x, 0, A->rows, res_sink( 0, v.r ), S->scr.slot( 1 ),
                                                         S->cs ) ) );
   return bicgstab_iterate< Real >( S, vals, diag, tagbase );
}

// BiCGStab iterations (BICGStab.hpp:58-116) in graph chunks until done
template< typename Real >
static b2s_status
bicgstab_iterate( b2s_solver_t* S, const Real* vals, const Real* diag, long long tagbase )
{
   const b2s_matrix_t* A = S->A;
   const int64_t n = S->n;
   auto v = vec_layout< Real >( S );
   Ctl* ctl = S->ctl_buf.as< Ctl >();
   const IluFactors< Real >* ilu = ilu_of< Real >( S );
   const int exact = S->o.bicgstab_exact_residue != 0;
   const double eps = std::is_same< Real, double >::value ? DBL_EPSILON : (double) FLT_EPSILON;
   auto res_sink = [ & ]( int mode, Real* target ) {
      BiResG< Real > s;
      s.b = v.b;
      s.r = target;
      s.r_ast = v.r_ast;
      s.p = v.p;
      s.s = v.s;
      s.diag = diag;
      s.ctl = ctl;
      s.mode = mode;
      s.exact = exact;
      return s;
   };
   const int chunk = chunk_of( S );
   for( ;; ) {
      B2S_TRY( run_graph( S, tagbase + chunk, [ & ]() -> b2s_status
      {
         for( int k = 0; k < chunk; k++ ) {
            BiMatvecG< Real > m1;
            m1.dst = v.Ap;
            m1.w0 = v.r_ast;
            m1.diag = diag;
            m1.ctl = ctl;
            m1.which = 0;
            if( ilu )
               B2S_TRY( prec_spmv< Real >( S, *ilu, vals, v.p, nullptr, v.Ap, m1, S->scr.slot( 2 ) ) );
            else
               B2S_TRY(
                  ( spmv_dispatch< Real, BiMatvecG< Real > >( A, vals, v.p, 0, A->rows, m1, S->scr.slot( 2 ), S->cs ) ) );
            vec_kernel< Real, BiSOp< Real >, NoFin ><<< wave_grid( vec_kernel< Real, BiSOp< Real >, NoFin >, n ), kReduceBlock, 0, S->cs >>>(
               n, ctl, BiSOp< Real >{ v.s, v.r, v.Ap, Real( 0 ) }, NoFin{}, S->scr.slot( 3 ) );
            B2S_TRY_CUDA( cudaGetLastError() );
            BiMatvecG< Real > m2;
            m2.dst = v.As;
            m2.w0 = v.s;
            m2.diag = diag;
            m2.ctl = ctl;
            m2.which = 1;
            if( ilu )
               B2S_TRY( prec_spmv< Real >( S, *ilu, vals, v.s, nullptr, v.As, m2, S->scr.slot( 4 ) ) );
            else
               B2S_TRY(
                  ( spmv_dispatch< Real, BiMatvecG< Real > >( A, vals, v.s, 0, A->rows, m2, S->scr.slot( 4 ), S->cs ) ) );
            BiXrOp< Real > xr{ v.x, v.r, v.p, v.s, v.As, v.r_ast, Real( 0 ), Real( 0 ) };
            vec_kernel< Real, BiXrOp< Real >, BiXrFin ><<< wave_grid( vec_kernel< Real, BiXrOp< Real >, BiXrFin >, n ), kReduceBlock, 0, S->cs >>>(
               n, ctl, xr, BiXrFin{ eps * eps, exact }, S->scr.slot( 5 ) );
            B2S_TRY_CUDA( cudaGetLastError() );
            // optional restart with a new r0 (runs only when the flag was raised)
            if( ilu ) {
               B2S_TRY( prec_spmv< Real >( S, *ilu, vals, v.x, v.b, v.r, res_sink( 1, v.r ), S->scr.slot( 6 ) ) );
               if( exact )
                  B2S_TRY( prec_spmv< Real >( S, *ilu, vals, v.x, v.b, v.s, res_sink( 2, v.s ), S->scr.slot( 7 ) ) );
            }
            else {
               B2S_TRY( ( spmv_dispatch< Real, BiResG< Real > >( A, vals, v.x, 0, A->rows, res_sink( 1, v.r ),
                                                                  S->scr.slot( 6 ), S->cs ) ) );
               if( exact )
                  B2S_TRY( ( spmv_dispatch< Real, BiResG< Real > >( A, vals, v.x, 0, A->rows, res_sink( 2, v.s ),
                                                                     S->scr.slot( 7 ), S->cs ) ) );
            }
            vec_kernel< Real, BiPOp< Real >, NoFin ><<< wave_grid( vec_kernel< Real, BiPOp< Real >, NoFin >, n ), kReduceBlock, 0, S->cs >>>(
               n, ctl, BiPOp< Real >{ v.p, v.r, v.Ap, Real( 0 ), Real( 0 ) }, NoFin{}, S->scr.slot( 8 ) );
            B2S_TRY_CUDA( cudaGetLastError() );
         }
         return B2S_OK;
      } ) );
      int done = 0;
      B2S_TRY( read_done( S, done ) );
      if( done )
         break;
      B2S_TRY( check_wall( S ) );
   }
   return B2S_OK;
}

// the projections of nk columns with the smallest accumulator bucket that holds them
template< typename Real >
static b2s_status
launch_multidot( int nk, int64_t n, int64_t ld, Ctl* ctl, const Real* V, const Real* w, int k0, GmArrays g, int i, int m,
                 RedScratch md, cudaStream_t s )
{
#define B2S_MD( NKB )                                                                                               \
   gm_multidot_kernel< Real, NKB ><<< wave_grid( gm_multidot_kernel< Real, NKB >, n ), kReduceBlock, 0, s >>>( \
      n, ld, ctl, V, w, k0, nk, g, i, m, md )
   if( nk <= 1 )
      B2S_MD( 1 );
   else if( nk <= 2 )
      B2S_MD( 2 );
   else if( nk <= 4 )
      B2S_MD( 4 );
   else if( nk <= 8 )
      B2S_MD( 8 );
   else
      B2S_MD( 16 );
#undef B2S_MD
   B2S_TRY_CUDA( cudaGetLastError() );
   return B2S_OK;
}

// the fused first-pass update and second-pass projections (columns 0 .. nk-1)
template< typename Real >
static b2s_status
launch_update_dot( int nk, int64_t n, int64_t ld, Ctl* ctl, const Real* V, Real* w, int i, int m, GmArrays g,
                   RedScratch md, cudaStream_t s )
{
#define B2S_UD( NKB )                                                                                          \
   gm_cgs_update_dot_kernel< Real, NKB ><<< wave_grid( gm_cgs_update_dot_kernel< Real, NKB >, n ), kReduceBlock, 0, \
                                            s >>>( n, ld, ctl, V, w, i, nk, m, g, md )
   if( nk <= 1 )
      B2S_UD( 1 );
   else if( nk <= 2 )
      B2S_UD( 2 );
   else if( nk <= 4 )
      B2S_UD( 4 );
   else if( nk <= 8 )
      B2S_UD( 8 );
   else
      B2S_UD( 16 );
#undef B2S_UD
   B2S_TRY_CUDA( cudaGetLastError() );
   return B2S_OK;
}

template< typename Real >
static b2s_status
gmres_cycle( b2s_solver_t* S, const Real* vals, const Real* diag, int m )
{
   const b2s_matrix_t* A = S->A;
   const int64_t n = S->n, ld = S->ld;
   auto v = vec_layout< Real >( S );
   Ctl* ctl = S->ctl_buf.as< Ctl >();
   Real* V = S->V.as< Real >();
   double* gmb = S->gm.as< double >();
   const int M = S->mmax;
   GmArrays g{ gmb, gmb + ( M + 1 ) * M, gmb + ( M + 1 ) * M + ( M + 1 ), gmb + ( M + 1 ) * M + 2 * ( M + 1 ),
               gmb + ( M + 1 ) * M + 3 * ( M + 1 ), gmb + ( M + 1 ) * M + 4 * ( M + 1 ), M + 1 };
   const int variant = S->o.gmres_variant;
   const bool mgs = variant == B2S_GMRES_MGS || variant == B2S_GMRES_MGSR;
   const int reps = ( variant == B2S_GMRES_CGSR || variant == B2S_GMRES_MGSR ) ? 2 : 1;
   RedScratch md{ S->md_partials.as< double >(), S->md_counter.as< unsigned int >() };
   const IluFactors< Real >* ilu = ilu_of< Real >( S );

   gm_start_kernel< Real ><<< wave_grid( gm_start_kernel< Real >, n ), kReduceBlock, 0, S->cs >>>( n, V, v.r, ctl, g, m );
   B2S_TRY_CUDA( cudaGetLastError() );
   for( int i = 0; i < m; i++ ) {
      const Real* vi = V + i * ld;
      if( mgs ) {
         GmWSink< Real, true > ws{ v.w, V, diag, ctl, g, i, m };
         if( ilu )
            B2S_TRY( prec_spmv< Real >( S, *ilu, vals, vi, nullptr, v.w, ws, S->scr.slot( 2 ) ) );
         else
            B2S_TRY(
               ( spmv_dispatch< Real, GmWSink< Real, true > >( A, vals, vi, 0, A->rows, ws, S->scr.slot( 2 ), S->cs ) ) );
         int slot = 3;
         for( int l = 0; l < reps; l++ ) {
            for( int k = ( l == 0 ? 1 : 0 ); k <= i; k++ ) {
               const int kp = ( k == 0 ) ? i : k - 1;
               GmMgsOp< Real > op{ v.w, V + kp * ld, V + k * ld, g.hl + kp, Real( 0 ) };
               arn_kernel< Real, GmMgsOp< Real >, GmMgsFin ><<< wave_grid( arn_kernel< Real, GmMgsOp< Real >, GmMgsFin >, n ), kReduceBlock, 0, S->cs >>>(
                  n, ctl, op, GmMgsFin{ g, k, i, m }, S->scr.slot( slot ) );
               B2S_TRY_CUDA( cudaGetLastError() );
               slot = slot == 3 ? 4 : 3;
            }
         }
         GmMgsLastOp< Real > last{ v.w, vi, g.hl + i, Real( 0 ) };
         arn_kernel< Real, GmMgsLastOp< Real >, GmNormFin ><<< wave_grid( arn_kernel< Real, GmMgsLastOp< Real >, GmNormFin >, n ), kReduceBlock, 0, S->cs >>>(
            n, ctl, last, GmNormFin{ g, i, m }, S->scr.slot( 5 ) );
         B2S_TRY_CUDA( cudaGetLastError() );
      }
      else {
         GmWSink< Real, false > ws{ v.w, V, diag, ctl, g, i, m };
         if( ilu ) {
            // w = M^-1 A v_i (the sink has no reduction of its own)
            StoreSink< Real, GmWSink< Real, false > > st{ v.w, nullptr, ws };
            B2S_TRY( ( spmv_dispatch< Real, StoreSink< Real, GmWSink< Real, false > > >( A, vals, vi, 0, A->rows, st,
                                                                                        RedScratch{}, S->cs ) ) );
            B2S_TRY( ilu->apply( v.w, v.w, S->cs, ws ) );
         }
         else
            B2S_TRY(
               ( spmv_dispatch< Real, GmWSink< Real, false > >( A, vals, vi, 0, A->rows, ws, RedScratch{}, S->cs ) ) );
         // projections on every column (pass 0)
         for( int k0 = 0; k0 <= i; k0 += kMd )
            B2S_TRY( launch_multidot< Real >( std::min( kMd, i + 1 - k0 ), n, ld, ctl, V, v.w, k0, g, i, m, md, S->cs ) );
         if( reps == 2 ) {
            // CGSR: update fused with the second projections on the first
            // columns, the rest projected on their own
            B2S_TRY( launch_update_dot< Real >( std::min( kMd, i + 1 ), n, ld, ctl, V, v.w, i, m, g, md, S->cs ) );
            for( int k0 = kMd; k0 <= i; k0 += kMd )
               B2S_TRY(
                  launch_multidot< Real >( std::min( kMd, i + 1 - k0 ), n, ld, ctl, V, v.w, k0, g, i, m, md, S->cs ) );
         }
         gm_cgs_update_kernel< Real, true ><<< wave_grid( gm_cgs_update_kernel< Real, true >, n ), kReduceBlock, 0,
                                                S->cs >>>( n, ld, ctl, V, v.w, i, m, g, S->scr.slot( 5 ) );
         B2S_TRY_CUDA( cudaGetLastError() );
      }
      gm_normalize_kernel< Real ><<< wave_grid( gm_normalize_kernel< Real >, n ), kReduceBlock, 0, S->cs >>>( n, ctl, V + ( i + 1 ) * ld, v.w );
      B2S_TRY_CUDA( cudaGetLastError() );
   }
   gm_backsolve_kernel<<< 1, 32, 0, S->cs >>>( ctl, g );
   B2S_TRY_CUDA( cudaGetLastError() );
   gm_xupdate_kernel< Real ><<< wave_grid( gm_xupdate_kernel< Real >, n ), kReduceBlock, 0, S->cs >>>( n, ld, ctl, V, v.x, g );
   B2S_TRY_CUDA( cudaGetLastError() );
   GmResSink< Real > rs{ v.b, v.r, diag, ctl, 1 };
   if( ilu )
      B2S_TRY( prec_spmv< Real >( S, *ilu, vals, v.x, v.b, v.r, rs, S->scr.slot( 6 ) ) );
   else
      B2S_TRY( ( spmv_dispatch< Real, GmResSink< Real > >( A, vals, v.x, 0, A->rows, rs, S->scr.slot( 6 ), S->cs ) ) );
   return B2S_OK;
}


// An SpMV M^-1 A src through `sink` (Jacobi inside the sink, ILU(0) between
// the product and the sink's pass), or M^-1 (b - A src) when b != NULL.
template< typename Real, class Sink >
static b2s_status
pspmv( b2s_solver_t* S, const Real* vals, const Real* src, const Real* b, Real* out, Sink sink, RedScratch rs )
{
   if( const IluFactors< Real >* ilu = ilu_of< Real >( S ) )
      return prec_spmv< Real >( S, *ilu, vals, src, b, out, sink, rs );
   return spmv_dispatch< Real, Sink >( S->A, vals, src, 0, S->A->rows, sink, rs, S->cs );
}

// ---------------------------------------------------------------------------
// GMRES with Householder reflections in compact WY form (GMRES.hpp:348-640,
// update :670-715). The reflectors y_0..y_m are the columns of V (as TNL's Y);
// the Arnoldi vectors are not stored. The small matrices (H, s, the Givens
// rotations, T and the top (m+1) x (m+1) block of Y) live on the host, as in
// TNL, so this variant reads a few scalars per step from the device; its
// vector work runs in the kernels below.

// out = M^-1 (b - A x) (b != NULL) or M^-1 A x ; *sq = (out, out)
template< typename Real >
struct CwySink
{
   static constexpr int NR = 1;
   Real* out;
   const Real* b;
   const Real* diag;
   double* sq;
   int pre = 0;
   __device__ bool skip() const { return false; }
   __device__ __forceinline__ void
   put( int row, Real sv, double* acc ) const
   {
      Real r = pre ? sv : ( b ? b[ row ] - sv : sv );
      if( diag && ! pre )
         r = r / diag[ row ];
      out[ row ] = r;
      acc[ 0 ] += (double) r * (double) r;
   }
   __device__ void finish( const double* t ) const { *sq = t[ 0 ]; }
};

// y = z with its first i entries zeroed ; acc (y, y)
template< typename Real >
struct CwyTruncOp
{
   static constexpr int NR = 1;
   Real* y;
   const Real* z;
   int64_t i;
   __device__ __forceinline__ void load( const Ctl& ) {}
   __device__ __forceinline__ void
   operator()( int64_t j, double* acc ) const
   {
      const Real v = j < i ? Real( 0 ) : z[ j ];
      y[ j ] = v;
      acc[ 0 ] += (double) v * (double) v;
   }
};

struct StoreFin
{
   static constexpr bool active = true;
   double* out;
   __device__ void operator()( Ctl&, const double* t ) const { *out = t[ 0 ]; }
};

// y = alpha * Y[:, 0..ncols) coef + beta * y, the column sum first (MatrixOperations gemv)
template< typename Real >
__global__ void __launch_bounds__( kReduceBlock )
cwy_gemv_kernel( int64_t n, int64_t ld, const Real* __restrict__ Y, int ncols, const double* __restrict__ coef,
                 double alpha, double beta, Real* __restrict__ y )
{
   __shared__ Real ax[ 256 ];
   for( int k = threadIdx.x; k < ncols; k += blockDim.x )
      ax[ k ] = (Real) alpha * (Real) coef[ k ];
   __syncthreads();
   for( int64_t j = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; j < n; j += (int64_t) gridDim.x * blockDim.x ) {
      Real aux = 0;
      for( int k = 0; k < ncols; k++ )
         aux += Y[ j + k * ld ] * ax[ k ];
      y[ j ] = beta != 0.0 ? aux + (Real) beta * y[ j ] : aux;
   }
}

template< typename Real >
static b2s_status
gmres_cwy_core( b2s_solver_t* S, const Real* vals, const Real* diag )
{
   const int64_t n = S->n, ld = S->ld;
   const int M = S->mmax;
   auto v = vec_layout< Real >( S );
   Ctl* ctl = S->ctl_buf.as< Ctl >();
   Real* Y = S->V.as< Real >();
   Real *z = v.z, *w = v.w, *vi = v.s, *r = v.r;
   // device scalars: [0] a squared norm, [1 .. M+1] dot products, [M+2 ..] gemv coefficients
   double* dsc = S->gm.as< double >();
   double* ddot = dsc + 1;
   double* dcoef = dsc + 2 + M;
   cudaStream_t cs = S->cs;
   auto sync = [ & ]() -> b2s_status
   {
      B2S_TRY_CUDA( cudaStreamSynchronize( cs ) );
      return B2S_OK;
   };
   auto pmatvec = [ & ]( const Real* src, const Real* b, Real* out ) -> b2s_status
   {
      return pspmv< Real >( S, vals, src, b, out, CwySink< Real >{ out, b, diag, dsc }, S->scr.slot( 1 ) );
   };
   // aux[k] = (Y_k, a) for k < ncols
   auto multidot = [ & ]( const Real* a, int ncols, double* aux ) -> b2s_status
   {
      for( int k = 0; k < ncols; k++ ) {
         vec_kernel< Real, DotOp< Real >, StoreFin ><<< wave_grid( vec_kernel< Real, DotOp< Real >, StoreFin >, n ), kReduceBlock, 0, cs >>>(
            n, ctl, DotOp< Real >{ Y + k * ld, a }, StoreFin{ ddot + k }, S->scr.slot( 3 ) );
         B2S_TRY_CUDA( cudaGetLastError() );
      }
      B2S_TRY_CUDA( cudaMemcpyAsync( aux, ddot, ncols * sizeof( double ), cudaMemcpyDeviceToHost, cs ) );
      return sync();
   };
   auto gemv = [ & ]( int ncols, const double* coef, double alpha, double beta, Real* y ) -> b2s_status
   {
      B2S_TRY_CUDA( cudaMemcpyAsync( dcoef, coef, ncols * sizeof( double ), cudaMemcpyHostToDevice, cs ) );
      cwy_gemv_kernel< Real ><<< wave_grid( cwy_gemv_kernel< Real >, n ), kReduceBlock, 0, cs >>>( n, ld, Y, ncols, dcoef, alpha, beta, y );
      B2S_TRY_CUDA( cudaGetLastError() );
      return B2S_OK;
   };
   auto get = [ & ]( const Real* p, int64_t k, Real& out ) -> b2s_status
   {
      B2S_TRY_CUDA( cudaMemcpyAsync( &out, p + k, sizeof( Real ), cudaMemcpyDeviceToHost, cs ) );
      return sync();
   };
   auto set = [ & ]( Real* p, int64_t k, Real val ) -> b2s_status
   {
      B2S_TRY_CUDA( cudaMemcpyAsync( p + k, &val, sizeof( Real ), cudaMemcpyHostToDevice, cs ) );
      return sync();
   };
   // IterativeSolver control on the host
   Ctl& c = *S->h_ctl;
   B2S_TRY( read_ctl( S ) );
   const double tol = c.tol, divtol = c.div_tol;
   const long long maxit = c.maxit, minit = c.minit;
   long long it = 0;
   double residue = 0;
   auto check_next_h = [ & ]()
   {
      return ! ( std::isnan( residue ) || it > maxit || ( residue > divtol && it >= minit ) ||
                 ( residue < tol && it >= minit ) );
   };
   auto next_iteration_h = [ & ]()
   {
      const bool go = check_next_h();
      it++;
      return go;
   };
   // ||M^-1 b||
   B2S_TRY( normb_launch< Real >( S, v.b, diag ) );
   B2S_TRY( read_ctl( S ) );
   const double normb = c.normb;
   if( n == 0 ) {
      c.it = 0;
      c.residue = 0;
      B2S_TRY_CUDA( cudaMemcpyAsync( S->ctl_buf.p, S->h_ctl, sizeof( Ctl ), cudaMemcpyHostToDevice, cs ) );
      return sync();
   }
   const int W = M + 1;
   std::vector< double > H( (size_t) W * M ), s( W ), csv( W ), snv( W ), T( (size_t) W * W ), YL( (size_t) W * W ),
      aux( W ), yv( W );
   double beta = 0;
   B2S_TRY( pmatvec( v.x, v.b, r ) );
   B2S_TRY_CUDA( cudaMemcpyAsync( &beta, dsc, sizeof( double ), cudaMemcpyDeviceToHost, cs ) );
   B2S_TRY( sync() );
   beta = std::sqrt( beta );
   residue = beta / normb;
   double beta_ratio = 1;
   int restart_cycles = 0, m = M;
   const int rmin = S->o.gmres_restarting_min, rmax = S->o.gmres_restarting_max;
   const int dmin = S->o.gmres_restarting_step_min, dmax = S->o.gmres_restarting_step_max;
   // the solution update of steps 0..k (GMRES.hpp:641-715)
   auto update = [ & ]( int k ) -> b2s_status
   {
      for( int i = 0; i <= m; i++ )
         yv[ i ] = s[ i ];
      for( int i = k; i >= 0; i-- ) {
         if( H[ i + i * W ] == 0 ) {
            set_error( "GMRES (CWY): zero on the diagonal of the Hessenberg matrix" );
            return B2S_BREAKDOWN;
         }
         yv[ i ] /= H[ i + i * W ];
         for( int j = i - 1; j >= 0; j-- )
            yv[ j ] -= H[ j + i * W ] * yv[ i ];
      }
      // x += sum_j y_j e_j - Y_k T_k sum_j y_j Y_j^T e_j
      for( int j = 0; j <= k; j++ )
         aux[ j ] = 0;
      for( int j = 0; j <= k; j++ )
         for( int i = 0; i <= j; i++ )
            aux[ i ] += yv[ j ] * YL[ j + i * W ];
      for( int i = 0; i <= k; i++ ) {
         double a2 = 0;
         for( int j = i; j <= k; j++ )
            a2 += T[ i + j * W ] * aux[ j ];
         aux[ i ] = a2;
      }
      B2S_TRY( gemv( k + 1, aux.data(), -1.0, 1.0, v.x ) );
      std::vector< Real > xh( k + 1 );
      B2S_TRY_CUDA( cudaMemcpyAsync( xh.data(), v.x, ( k + 1 ) * sizeof( Real ), cudaMemcpyDeviceToHost, cs ) );
      B2S_TRY( sync() );
      for( int j = 0; j <= k; j++ )
         xh[ j ] = xh[ j ] + (Real) yv[ j ];
      B2S_TRY_CUDA( cudaMemcpyAsync( v.x, xh.data(), ( k + 1 ) * sizeof( Real ), cudaMemcpyHostToDevice, cs ) );
      return sync();
   };
   bool early = false;
   while( check_next_h() ) {
      B2S_TRY( check_wall( S ) );
      // Baker-Jessup-Kolev adaptivity of the restart length (GMRES.hpp:118-137)
      if( rmax > rmin && restart_cycles > 0 ) {
         if( beta_ratio > 0.99 )
            m = rmax;
         else if( beta_ratio >= 0.175 ) {
            const int step = dmin + (int) ( (float) ( dmax - dmin ) / ( rmax - rmin ) * ( m - rmin ) );
            if( m - step >= rmin )
               m -= step;
            else
               m = rmax;
         }
      }
      // orthogonalize_CWY (GMRES.hpp:348-425)
      B2S_TRY_CUDA( cudaMemcpyAsync( z, r, n * sizeof( Real ), cudaMemcpyDeviceToDevice, cs ) );
      std::fill( H.begin(), H.end(), 0.0 );
      std::fill( s.begin(), s.end(), 0.0 );
      std::fill( T.begin(), T.end(), 0.0 );
      int o_steps = m;
      for( int i = 0; i <= m && next_iteration_h(); i++ ) {
         Real* yi = Y + i * ld;
         // hauseholder_generate: y_i = z truncated, ||y_i||, y_ii += sign * norm, t_i, T column
         vec_kernel< Real, CwyTruncOp< Real >, StoreFin ><<< wave_grid( vec_kernel< Real, CwyTruncOp< Real >, StoreFin >, n ), kReduceBlock, 0, cs >>>(
            n, ctl, CwyTruncOp< Real >{ yi, z, i }, StoreFin{ dsc }, S->scr.slot( 4 ) );
         B2S_TRY_CUDA( cudaGetLastError() );
         double nz2 = 0;
         B2S_TRY_CUDA( cudaMemcpyAsync( &nz2, dsc, sizeof( double ), cudaMemcpyDeviceToHost, cs ) );
         Real y_ii = 0;  // entries past the system's size are zero (GMRES with m >= n)
         B2S_TRY( sync() );
         if( i < n )
            B2S_TRY( get( yi, i, y_ii ) );
         const Real normz = (Real) std::sqrt( nz2 );
         if( i < n )
            B2S_TRY( set( yi, i, y_ii > 0 ? y_ii + normz : y_ii - normz ) );
         const double norm_yi_squared = 2 * ( (double) normz * normz + std::fabs( (double) y_ii ) * normz );
         const double t_i = 2.0 / norm_yi_squared;
         T[ i + i * W ] = t_i;
         if( i > 0 ) {
            B2S_TRY( multidot( yi, i, aux.data() ) );
            for( int k = 0; k < i; k++ ) {
               T[ k + i * W ] = 0.0;
               for( int j = k; j < i; j++ )
                  T[ k + i * W ] -= T[ k + j * W ] * ( t_i * aux[ j ] );
            }
         }
         // hauseholder_apply_trunc: the top of y_i to YL ; out = z - y_i (first i + 1 entries)
         std::vector< Real > top( W ), ztop( i + 1 );
         B2S_TRY_CUDA( cudaMemcpyAsync( top.data(), yi, std::min< int64_t >( W, n ) * sizeof( Real ),
                                        cudaMemcpyDeviceToHost, cs ) );
         B2S_TRY_CUDA( cudaMemcpyAsync( ztop.data(), z, std::min< int64_t >( i + 1, n ) * sizeof( Real ),
                                        cudaMemcpyDeviceToHost, cs ) );
         B2S_TRY( sync() );
         for( int k = 0; k < W; k++ )
            YL[ k + i * W ] = k < n ? (double) top[ k ] : 0.0;
         double* out = i == 0 ? s.data() : &H[ ( i - 1 ) * W ];
         for( int k = 0; k <= i && k < n; k++ )
            out[ k ] = (double) ztop[ k ] - YL[ k + i * W ];
         // hauseholder_cwy: v_i = (I - Y_i T_i Y_i^T) e_i
         for( int k = 0; k <= i; k++ )
            aux[ k ] = YL[ i + k * W ];
         for( int k = 0; k <= i; k++ ) {
            double a2 = 0;
            for( int j = k; j <= i; j++ )
               a2 += T[ k + j * W ] * aux[ j ];
            aux[ k ] = a2;
         }
         B2S_TRY( gemv( i + 1, aux.data(), -1.0, 0.0, vi ) );
         if( i < n ) {
            Real vii;
            B2S_TRY( get( vi, i, vii ) );
            B2S_TRY( set( vi, i, (Real) 1.0 + vii ) );
         }
         if( i < m ) {
            // w = M^-1 A v_i ; z = (I - Y_i T_i^T Y_i^T) w
            B2S_TRY( pmatvec( vi, nullptr, w ) );
            B2S_TRY( multidot( w, i + 1, aux.data() ) );
            for( int k = i; k >= 0; k-- ) {
               double a2 = 0;
               for( int j = 0; j <= k; j++ )
                  a2 += T[ j + k * W ] * aux[ j ];
               aux[ k ] = a2;
            }
            B2S_TRY_CUDA( cudaMemcpyAsync( z, w, n * sizeof( Real ), cudaMemcpyDeviceToDevice, cs ) );
            B2S_TRY( gemv( i + 1, aux.data(), -1.0, 1.0, z ) );
         }
         // Givens rotations G_0 .. G_{i-1} (GMRES.hpp:751-763)
         if( i > 0 ) {
            const int q = i - 1;
            for( int k = 0; k < q; k++ )
               apply_plane_rotation( H[ k + q * W ], H[ k + 1 + q * W ], csv[ k ], snv[ k ] );
            if( H[ q + 1 + q * W ] != 0.0 ) {
               gen_plane_rotation( H[ q + q * W ], H[ q + 1 + q * W ], csv[ q ], snv[ q ] );
               apply_plane_rotation( H[ q + q * W ], H[ q + 1 + q * W ], csv[ q ], snv[ q ] );
               apply_plane_rotation( s[ q ], s[ q + 1 ], csv[ q ], snv[ q ] );
            }
         }
         residue = std::fabs( s[ i ] ) / normb;
         if( i > 0 && ! check_next_h() ) {
            o_steps = i - 1;
            break;
         }
      }
      if( o_steps < m ) {
         B2S_TRY( update( o_steps ) );
         early = true;
         break;
      }
      B2S_TRY( update( m - 1 ) );
      B2S_TRY( pmatvec( v.x, v.b, r ) );
      double b2 = 0;
      B2S_TRY_CUDA( cudaMemcpyAsync( &b2, dsc, sizeof( double ), cudaMemcpyDeviceToHost, cs ) );
      B2S_TRY( sync() );
      const double beta_old = beta;
      beta = std::sqrt( b2 );
      residue = beta / normb;
      ++restart_cycles;
      beta_ratio = beta / beta_old;
   }
   (void) early;
   c.it = it;
   c.residue = residue;
   c.done = 1;
   B2S_TRY_CUDA( cudaMemcpyAsync( S->ctl_buf.p, S->h_ctl, sizeof( Ctl ), cudaMemcpyHostToDevice, cs ) );
   return sync();
}

template< typename Real >
static b2s_status
gmres_core( b2s_solver_t* S, const Real* vals, const Real* diag, long long tagbase )
{
   if( S->o.gmres_variant == B2S_GMRES_CWY )
      return gmres_cwy_core< Real >( S, vals, diag );
   const b2s_matrix_t* A = S->A;
   auto v = vec_layout< Real >( S );
   Ctl* ctl = S->ctl_buf.as< Ctl >();
   const int rmin = S->o.gmres_restarting_min, rmax = S->o.gmres_restarting_max;
   const int dmin = S->o.gmres_restarting_step_min, dmax = S->o.gmres_restarting_step_max;
   B2S_TRY( normb_launch< Real >( S, v.b, diag ) );
   GmResSink< Real > rs0{ v.b, v.r, diag, ctl, 0 };
   if( const IluFactors< Real >* ilu = ilu_of< Real >( S ) )
      B2S_TRY( prec_spmv< Real >( S, *ilu, vals, v.x, v.b, v.r, rs0, S->scr.slot( 1 ) ) );
   else
      B2S_TRY( ( spmv_dispatch< Real, GmResSink< Real > >( A, vals, v.x, 0, A->rows, rs0, S->scr.slot( 1 ), S->cs ) ) );
   B2S_TRY( read_ctl( S ) );
   double beta_ratio = 1.0;
   int restart_cycles = 0, m = rmax;
   while( host_check_next( *S->h_ctl ) ) {
      // Baker-Jessup-Kolev adaptivity of the restart length (GMRES.hpp:118-137)
      if( rmax > rmin && restart_cycles > 0 ) {
         if( beta_ratio > 0.99 )
            m = rmax;
         else if( beta_ratio >= 0.175 ) {
            const int step = dmin + (int) ( (float) ( dmax - dmin ) / ( rmax - rmin ) * ( m - rmin ) );
            if( m - step >= rmin )
               m -= step;
            else
               m = rmax;
         }
      }
      B2S_TRY( run_graph( S, tagbase + m, [ & ]() { return gmres_cycle< Real >( S, vals, diag, m ); } ) );
      B2S_TRY( read_ctl( S ) );
      B2S_TRY( check_wall( S ) );
      const Ctl& c = *S->h_ctl;
      if( c.reason == 3 || c.o_steps < m )
         break;
      ++restart_cycles;
      beta_ratio = c.gm_beta / c.beta_old;
   }
   return B2S_OK;
}

// TFQMR (TFQMR.hpp:18-114): iterations in graph chunks of pairs (odd, even),
// then the last iteration's x update
template< typename Real >
static b2s_status
tfqmr_core( b2s_solver_t* S, const Real* vals, const Real* diag, long long tagbase )
{
   const int64_t n = S->n;
   auto v = vec_layout< Real >( S );
   Ctl* ctl = S->ctl_buf.as< Ctl >();
   // r, w, u, v, Au, d, r_ast
   Real *r = v.r, *w = v.w, *u = v.p, *vv = v.As, *Au = v.Ap, *d = v.s, *r_ast = v.r_ast;
   B2S_TRY( normb_launch< Real >( S, v.b, diag ) );
   B2S_TRY( pspmv< Real >( S, vals, v.x, v.b, r, TfInitSink< Real >{ v.b, r, w, u, r_ast, d, diag, ctl },
                           S->scr.slot( 1 ) ) );
   B2S_TRY( pspmv< Real >( S, vals, u, nullptr, Au, TfAuSink< Real, 0 >{ Au, vv, r_ast, diag, ctl },
                           S->scr.slot( 2 ) ) );
   const int pairs = std::max( 1, chunk_of( S ) / 2 );
   for( ;; ) {
      B2S_TRY( run_graph( S, tagbase + pairs, [ & ]() -> b2s_status
      {
         for( int k = 0; k < pairs; k++ ) {
            // odd iteration: alpha is known
            vec_kernel< Real, TfStepOp< Real, false >, TfStepFin< false > ><<< wave_grid( vec_kernel< Real, TfStepOp< Real, false >, TfStepFin< false > >, n ), kReduceBlock, 0, S->cs >>>(
               n, ctl, TfStepOp< Real, false >{ v.x, w, d, u, Au, r_ast, 0, 0, 0 }, TfStepFin< false >{}, S->scr.slot( 3 ) );
            vec_kernel< Real, TfUOp< Real >, NoFin ><<< wave_grid( vec_kernel< Real, TfUOp< Real >, NoFin >, n ), kReduceBlock, 0, S->cs >>>(
               n, ctl, TfUOp< Real >{ u, vv, 0 }, NoFin{}, S->scr.slot( 4 ) );
            B2S_TRY_CUDA( cudaGetLastError() );
            // even iteration
            B2S_TRY( pspmv< Real >( S, vals, u, nullptr, Au, TfAuSink< Real, 1 >{ Au, vv, r_ast, diag, ctl },
                                    RedScratch{} ) );
            vec_kernel< Real, TfStepOp< Real, true >, TfStepFin< true > ><<< wave_grid( vec_kernel< Real, TfStepOp< Real, true >, TfStepFin< true > >, n ), kReduceBlock, 0, S->cs >>>(
               n, ctl, TfStepOp< Real, true >{ v.x, w, d, u, Au, r_ast, 0, 0, 0 }, TfStepFin< true >{}, S->scr.slot( 5 ) );
            vec_kernel< Real, TfDirOp< Real >, NoFin ><<< wave_grid( vec_kernel< Real, TfDirOp< Real >, NoFin >, n ), kReduceBlock, 0, S->cs >>>(
               n, ctl, TfDirOp< Real >{ u, vv, w, Au, 0, 0 }, NoFin{}, S->scr.slot( 6 ) );
            B2S_TRY_CUDA( cudaGetLastError() );
            B2S_TRY( pspmv< Real >( S, vals, u, nullptr, Au, TfAuSink< Real, 2 >{ Au, vv, r_ast, diag, ctl },
                                    S->scr.slot( 7 ) ) );
         }
         return B2S_OK;
      } ) );
      int done = 0;
      B2S_TRY( read_done( S, done ) );
      if( done )
         break;
      B2S_TRY( check_wall( S ) );
   }
   if( n > 0 ) {
      tf_flush_kernel< Real ><<< wave_grid( tf_flush_kernel< Real >, n ), kReduceBlock, 0, S->cs >>>( n, ctl, v.x, d );
      B2S_TRY_CUDA( cudaGetLastError() );
   }
   return B2S_OK;
}

// BiCGStab(ell) (BICGStabL.hpp:42-250): ||M^-1 b||, r_0 = M^-1 (b - A x), the
// shadow residual and the first outer test
template< typename Real >
static b2s_status
bicgstabl_init( b2s_solver_t* S, const Real* vals, const Real* diag )
{
   const int64_t n = S->n, ld = S->ld;
   const int ell = S->o.bicgstab_ell;
   auto v = vec_layout< Real >( S );
   Ctl* ctl = S->ctl_buf.as< Ctl >();
   Real* R = S->V.as< Real >();
   Real* U = R + ( ell + 1 ) * ld;
   B2S_TRY( normb_launch< Real >( S, v.b, diag ) );
   B2S_TRY( pspmv< Real >( S, vals, v.x, v.b, R, BlResSink< Real, 0 >{ v.b, R, diag, ctl }, S->scr.slot( 1 ) ) );
   vec_kernel< Real, BlInitOp< Real >, BlInitFin ><<< wave_grid( vec_kernel< Real, BlInitOp< Real >, BlInitFin >, n ), kReduceBlock, 0, S->cs >>>(
      n, ctl, BlInitOp< Real >{ R, v.r_ast, U, 0 }, BlInitFin{}, S->scr.slot( 2 ) );
   B2S_TRY_CUDA( cudaGetLastError() );
   return B2S_OK;
}

// outer iterations (ell Bi-CG steps, the MGS part and the final updates) in
// graph chunks until the device says done
template< typename Real >
static b2s_status
bicgstabl_iterate( b2s_solver_t* S, const Real* vals, const Real* diag, long long tagbase )
{
   const int64_t n = S->n, ld = S->ld;
   const int ell = S->o.bicgstab_ell;
   auto v = vec_layout< Real >( S );
   Ctl* ctl = S->ctl_buf.as< Ctl >();
   Real* R = S->V.as< Real >();
   Real* U = R + ( ell + 1 ) * ld;
   Real *r_ast = v.r_ast, *tmp = v.s;
   double* gb = S->gm.as< double >();
   const BlArrays g{ gb, gb + ell * ell, gb + ell * ell + ( ell + 1 ), gb + ell * ell + 2 * ( ell + 1 ),
                     gb + ell * ell + 3 * ( ell + 1 ), ell };
   const int exact = S->o.bicgstab_exact_residue != 0;
   const int outer = std::max( 1, chunk_of( S ) / ell );
   for( ;; ) {
      B2S_TRY( run_graph( S, tagbase + outer, [ & ]() -> b2s_status
      {
         for( int k = 0; k < outer; k++ ) {
            for( int j = 0; j < ell; j++ ) {
               vec_kernel< Real, BlGeamUOp< Real >, NoFin ><<< wave_grid( vec_kernel< Real, BlGeamUOp< Real >, NoFin >, n ), kReduceBlock, 0, S->cs >>>(
                  n, ctl, BlGeamUOp< Real >{ R, U, ld, j, 0 }, NoFin{}, S->scr.slot( 3 ) );
               B2S_TRY_CUDA( cudaGetLastError() );
               B2S_TRY( pspmv< Real >( S, vals, U + j * ld, nullptr, U + ( j + 1 ) * ld,
                                       BlMatvecSink< Real, false >{ U + ( j + 1 ) * ld, r_ast, diag, ctl, 0 },
                                       S->scr.slot( 4 ) ) );
               vec_kernel< Real, BlRUpdateOp< Real >, NoFin ><<< wave_grid( vec_kernel< Real, BlRUpdateOp< Real >, NoFin >, n ), kReduceBlock, 0, S->cs >>>(
                  n, ctl, BlRUpdateOp< Real >{ R, U, v.x, ld, j, 0 }, NoFin{}, S->scr.slot( 5 ) );
               B2S_TRY_CUDA( cudaGetLastError() );
               B2S_TRY( pspmv< Real >( S, vals, R + j * ld, nullptr, R + ( j + 1 ) * ld,
                                       BlMatvecSink< Real, true >{ R + ( j + 1 ) * ld, r_ast, diag, ctl, j + 1 == ell },
                                       S->scr.slot( 6 ) ) );
            }
            for( int j = 1; j <= ell; j++ )
               for( int kk = 1; kk <= j; kk++ ) {
                  vec_kernel< Real, BlMgsOp< Real >, BlMgsFin ><<< wave_grid( vec_kernel< Real, BlMgsOp< Real >, BlMgsFin >, n ), kReduceBlock, 0, S->cs >>>(
                     n, ctl, BlMgsOp< Real >{ R, ld, j, kk, g, 0 }, BlMgsFin{ g, j, kk }, S->scr.slot( 7 ) );
                  B2S_TRY_CUDA( cudaGetLastError() );
               }
            vec_kernel< Real, BlFinalOp< Real >, BlFinalFin ><<< wave_grid( vec_kernel< Real, BlFinalOp< Real >, BlFinalFin >, n ), kReduceBlock, 0, S->cs >>>(
               n, ctl, BlFinalOp< Real >{ v.x, R, U, r_ast, ld, g, {}, {}, {} }, BlFinalFin{ exact }, S->scr.slot( 8 ) );
            B2S_TRY_CUDA( cudaGetLastError() );
            if( exact )
               B2S_TRY( pspmv< Real >( S, vals, v.x, v.b, tmp, BlResSink< Real, 1 >{ v.b, tmp, diag, ctl },
                                       S->scr.slot( 9 ) ) );
         }
         return B2S_OK;
      } ) );
      int done = 0;
      B2S_TRY( read_done( S, done ) );
      if( done )
         break;
      B2S_TRY( check_wall( S ) );
   }
   return B2S_OK;
}

template< typename Real >
static b2s_status
bicgstabl_core( b2s_solver_t* S, const Real* vals, const Real* diag, long long tagbase )
{
   B2S_TRY( bicgstabl_init< Real >( S, vals, diag ) );
   return bicgstabl_iterate< Real >( S, vals, diag, tagbase );
}

// ---------------------------------------------------------------------------
// Jacobi and SOR (stationary.cuh). `adiag` is A's diagonal (the sweeps divide
// by it whatever the preconditioner setting: TNL's stationary solvers fetch
// the diagonal themselves and use no preconditioner).
template< typename Real >
static b2s_status
stat_begin( b2s_solver_t* S, const Real* b )
{
   // resetIterations; residue = tol + 1; bNorm = ||b|| (Jacobi.hpp:84-95, SOR.hpp:83-93)
   S->h_ctl->residue = S->h_ctl->tol + 1.0;
   B2S_TRY_CUDA( cudaMemcpyAsync( S->ctl_buf.p, S->h_ctl, sizeof( Ctl ), cudaMemcpyHostToDevice, S->cs ) );
   Ctl* ctl = S->ctl_buf.as< Ctl >();
   vec_kernel< Real, NormOp< Real >, StatNormbFin ><<< wave_grid( vec_kernel< Real, NormOp< Real >, StatNormbFin >, S->n ), kReduceBlock, 0, S->cs >>>(
      S->n, ctl, NormOp< Real >{ b, nullptr }, StatNormbFin{}, S->scr.slot( 0 ) );
   B2S_TRY_CUDA( cudaGetLastError() );
   return B2S_OK;
}

template< typename Real >
static b2s_status
stat_residue( b2s_solver_t* S, const Real* vals, const Real* b, const Real* x, int always )
{
   StatResG< Real > r{ b, S->ctl_buf.as< Ctl >(), (long long) S->o.residue_period, always };
   return spmv_dispatch< Real, StatResG< Real > >( S->A, vals, x, 0, S->A->rows, r, S->scr.slot( 5 ), S->cs );
}

// Jacobi.hpp:67-110: per loop pass nextIteration, x -> aux, [residue of x],
// the iteration count, aux -> x, [residue of x]; then the final residue
template< typename Real >
static b2s_status
jacobi_core( b2s_solver_t* S, const Real* vals, const Real* adiag, long long tagbase )
{
   auto v = vec_layout< Real >( S );
   Ctl* ctl = S->ctl_buf.as< Ctl >();
   B2S_TRY( stat_begin< Real >( S, v.b ) );
   const Real omega = (Real) S->o.omega;
   const int pairs = std::max( 1, chunk_of( S ) / 2 );
   for( ;; ) {
      B2S_TRY( run_graph( S, tagbase + pairs, [ & ]() -> b2s_status
      {
         for( int k = 0; k < pairs; k++ ) {
            stat_ctl_kernel<<< 1, 1, 0, S->cs >>>( ctl, 0 );
            B2S_TRY_CUDA( cudaGetLastError() );
            JacobiG< Real > s1{ v.x, v.z, v.b, adiag, omega, ctl };
            B2S_TRY( ( spmv_dispatch< Real, JacobiG< Real > >( S->A, vals, v.x, 0, S->A->rows, s1, RedScratch{}, S->cs ) ) );
            B2S_TRY( stat_residue< Real >( S, vals, v.b, v.x, 0 ) );
            stat_ctl_kernel<<< 1, 1, 0, S->cs >>>( ctl, 1 );
            B2S_TRY_CUDA( cudaGetLastError() );
            JacobiG< Real > s2{ v.z, v.x, v.b, adiag, omega, ctl };
            B2S_TRY( ( spmv_dispatch< Real, JacobiG< Real > >( S->A, vals, v.z, 0, S->A->rows, s2, RedScratch{}, S->cs ) ) );
            B2S_TRY( stat_residue< Real >( S, vals, v.b, v.x, 0 ) );
         }
         return B2S_OK;
      } ) );
      int done = 0;
      B2S_TRY( read_done( S, done ) );
      if( done )
         break;
      B2S_TRY( check_wall( S ) );
   }
   return stat_residue< Real >( S, vals, v.b, v.x, 1 );
}

// SOR.hpp:66-99: per iteration nextIteration, one sweep, [residue]; the
// sweeps alternate between x and aux, the last result is moved to x
template< typename Real >
static b2s_status
sor_core( b2s_solver_t* S, const SorPlan< Real >& P, const Real* vals, const Real* adiag, long long tagbase )
{
   auto v = vec_layout< Real >( S );
   Ctl* ctl = S->ctl_buf.as< Ctl >();
   B2S_TRY( stat_begin< Real >( S, v.b ) );
   const Real omega = (Real) S->o.omega;
   const int sweeps = std::max( 2, chunk_of( S ) / 2 * 2 );
   Real* buf[ 2 ] = { v.x, v.z };
   for( ;; ) {
      B2S_TRY( run_graph( S, tagbase + sweeps, [ & ]() -> b2s_status
      {
         for( int k = 0; k < sweeps; k++ ) {
            stat_ctl_kernel<<< 1, 1, 0, S->cs >>>( ctl, 0 );
            B2S_TRY_CUDA( cudaGetLastError() );
            B2S_TRY( P.sweep( v.b, adiag, buf[ k & 1 ], buf[ ( k + 1 ) & 1 ], omega, ctl, S->cs ) );
            B2S_TRY( stat_residue< Real >( S, vals, v.b, buf[ ( k + 1 ) & 1 ], 0 ) );
         }
         return B2S_OK;
      } ) );
      int done = 0;
      B2S_TRY( read_done( S, done ) );
      if( done )
         break;
      B2S_TRY( check_wall( S ) );
   }
   B2S_TRY( P.check( S->cs ) );
   // the failed check counted one iteration more than the sweeps made
   B2S_TRY( read_ctl( S ) );
   const long long made = S->h_ctl->it - 1;
   if( made > 0 && ( made & 1 ) && S->n > 0 )
      B2S_TRY_CUDA( cudaMemcpyAsync( v.x, v.z, (size_t) S->n * sizeof( Real ), cudaMemcpyDeviceToDevice, S->cs ) );
   return stat_residue< Real >( S, vals, v.b, v.x, 1 );
}

template< typename Real >
static const SorPlan< Real >&
sor_of( const b2s_solver_t* S )
{
   if constexpr( std::is_same< Real, double >::value )
      return S->sor64;
   else
      return S->sor32;
}

template< typename Real >
static b2s_status
run_core( b2s_solver_t* S, const Real* vals, const Real* diag, double tol, long long maxit, Ctl& out )
{
   B2S_TRY( init_ctl( S, tol, maxit ) );
   const long long tag = ( (long long) ( std::is_same< Real, double >::value ? 1 : 2 ) << 40 ) + ( (long long) S->o.solver << 32 );
   switch( S->o.solver ) {
      case B2S_CG:
         B2S_TRY( cg_core< Real >( S, vals, diag, tag ) );
         break;
      case B2S_BICGSTAB:
         B2S_TRY( bicgstab_core< Real >( S, vals, diag, tag ) );
         break;
      case B2S_GMRES:
         B2S_TRY( gmres_core< Real >( S, vals, diag, tag ) );
         break;
      case B2S_TFQMR:
         B2S_TRY( tfqmr_core< Real >( S, vals, diag, tag ) );
         break;
      case B2S_BICGSTABL:
         B2S_TRY( bicgstabl_core< Real >( S, vals, diag, tag ) );
         break;
      case B2S_JACOBI:
         B2S_TRY( jacobi_core< Real >( S, vals, S->A->diagonal.as< Real >(), tag ) );
         break;
      case B2S_SOR:
         B2S_TRY( sor_core< Real >( S, sor_of< Real >( S ), vals, S->A->diagonal.as< Real >(), tag ) );
         break;
      default:
         set_error( "unknown solver %d", S->o.solver );
         return B2S_INVALID_ARG;
   }
   B2S_TRY( read_ctl( S ) );
   out = *S->h_ctl;
   return B2S_OK;
}

// ---------------------------------------------------------------------------
// Mixed precision: FP64 iterative refinement around FP32 inner solves.
//   r = b - A x (FP64) ; stop when ||r|| / ||b|| <= tol
//   solve A d = r in FP32 (inner tolerance) ; x += d (FP64)
template< typename Real >
struct RefineResSink
{
   static constexpr int NR = 1;
   const double* b;
   float* r32;
   Ctl* ctl;
   __device__ bool skip() const { return false; }
   __device__ __forceinline__ void
   put( int row, double s, double* acc ) const
   {
      const double rr = b[ row ] - s;
      r32[ row ] = (float) rr;
      acc[ 0 ] += rr * rr;
   }
   __device__ void finish( const double* t ) const { ctl->outer_res = sqrt( t[ 0 ] ); }
};

__global__ void
refine_update_kernel( int64_t n, double* __restrict__ x, const float* __restrict__ d, float* __restrict__ dzero )
{
   for( int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x ) {
      x[ i ] += (double) d[ i ];
      dzero[ i ] = 0.0f;
   }
}

// ||b - A x|| / ||b|| in FP64 for any matrix type (the report's true residual)
template< typename Real >
struct TrueResSink
{
   static constexpr int NR = 2;
   const Real* b;
   double* out;  // out[0] = ||r||, out[1] = ||b||
   __device__ bool skip() const { return false; }
   __device__ __forceinline__ void
   put( int row, Real s, double* acc ) const
   {
      const double bb = (double) b[ row ];
      const double rr = bb - (double) s;
      acc[ 0 ] += rr * rr;
      acc[ 1 ] += bb * bb;
   }
   __device__ void
   finish( const double* t ) const
   {
      out[ 0 ] = sqrt( t[ 0 ] );
      out[ 1 ] = sqrt( t[ 1 ] );
   }
};

template< typename Real >
static b2s_status
true_residual( b2s_solver_t* S, const Real* vals, const Real* b, const Real* x, double& res )
{
   double* d_out = &S->ctl_buf.as< Ctl >()->outer_norm;  // reuse two doubles of the control block
   TrueResSink< Real > sink{ b, d_out };
   B2S_TRY( ( spmv_dispatch< Real, TrueResSink< Real > >( S->A, vals, x, 0, S->A->rows, sink, S->scr.slot( 9 ), S->cs ) ) );
   double h[ 2 ];
   B2S_TRY_CUDA( cudaMemcpyAsync( h, d_out, 2 * sizeof( double ), cudaMemcpyDeviceToHost, S->cs ) );
   B2S_TRY_CUDA( cudaStreamSynchronize( S->cs ) );
   res = h[ 1 ] > 0 ? h[ 0 ] / h[ 1 ] : h[ 0 ];
   return B2S_OK;
}

static b2s_status
solve_plain( b2s_solver_t* S, b2s_solve_report& rep )
{
   Ctl c{};
   if( S->A->dtype == B2S_F64 ) {
      auto v = vec_layout< double >( S );
      const double* diag = S->o.preconditioner == B2S_PRECOND_JACOBI ? S->A->diagonal.as< double >() : nullptr;
      B2S_TRY( run_core< double >( S, S->A->values.as< double >(), diag, S->o.convergence_residue, S->o.max_iterations, c ) );
      if( ilu_of< double >( S ) )
         B2S_TRY( S->ilu64.check( S->cs ) );
      B2S_TRY( true_residual< double >( S, S->A->values.as< double >(), v.b, v.x, rep.true_residual ) );
   }
   else {
      auto v = vec_layout< float >( S );
      const float* diag = S->o.preconditioner == B2S_PRECOND_JACOBI ? S->A->diagonal.as< float >() : nullptr;
      B2S_TRY( run_core< float >( S, S->A->values.as< float >(), diag, S->o.convergence_residue, S->o.max_iterations, c ) );
      if( ilu_of< float >( S ) )
         B2S_TRY( S->ilu32.check( S->cs ) );
      B2S_TRY( true_residual< float >( S, S->A->values.as< float >(), v.b, v.x, rep.true_residual ) );
   }
   rep.iterations = c.it;
   rep.residue = c.residue;
   rep.refinements = 0;
   rep.status = convergence_status( c );
   rep.converged = rep.status == B2S_OK;
   return B2S_OK;
}

// the tightest relative residual an FP32 inner solve is asked to reach
constexpr double kInnerFloor = 1e-6;

static b2s_status
mixed_refine( b2s_solver_t* S, b2s_solve_report& rep )
{
   const int64_t n = S->n;
   const int64_t ln = ( n + 63 ) / 64 * 64;
   double* b64 = S->outer.as< double >();
   double* x64 = b64 + ln;
   auto v = vec_layout< float >( S );
   const float* vals32 = S->A->values32.as< float >();
   const float* diag32 = S->o.preconditioner ? S->diag32.as< float >() : nullptr;
   Ctl* ctl = S->ctl_buf.as< Ctl >();
   // ||b||
   double normb = 0;
   {
      B2S_TRY( init_ctl( S, 0, 0 ) );  // clears `done` before the reduction reads it
      vec_kernel< double, NormOp< double >, NormbFin ><<< wave_grid( vec_kernel< double, NormOp< double >, NormbFin >, n ), kReduceBlock, 0, S->cs >>>(
         n, ctl, NormOp< double >{ b64, nullptr }, NormbFin{}, S->scr.slot( 0 ) );
      B2S_TRY_CUDA( cudaGetLastError() );
      B2S_TRY( read_ctl( S ) );
      normb = S->h_ctl->normb;
   }
   B2S_TRY_CUDA( cudaMemsetAsync( v.x, 0, n * sizeof( float ), S->cs ) );
   long long total_it = 0;
   double res = 0, last_inner = 0;
   int refinements = 0;
   b2s_status inner_status = B2S_OK;
   const double tol = S->o.convergence_residue;
   int max_ref = S->o.max_refinements > 0 ? S->o.max_refinements : 20;
   if( S->o.solver == B2S_GMRES )  // one refinement per restart cycle
      max_ref = (int) std::max< long long >(
         max_ref, std::min< long long >( 1000000, S->o.max_iterations / std::max( 1, S->o.gmres_restarting_max ) + 1 ) );
   double prev_res = INFINITY;
   for( ;; ) {
      // r = b - A x in FP64, stored as the FP32 right-hand side of the inner solve
      B2S_TRY( init_ctl( S, 0, 0 ) );
      RefineResSink< double > rsink{ b64, v.b, ctl };
      B2S_TRY( ( spmv_dispatch< double, RefineResSink< double > >( S->A, S->A->values.as< double >(), x64, 0, S->A->rows,
                                                                    rsink, S->scr.slot( 1 ), S->cs ) ) );
      B2S_TRY( read_ctl( S ) );
      res = S->h_ctl->outer_res / normb;
      if( ! ( res > tol ) || std::isnan( res ) )
         break;
      if( refinements >= max_ref || total_it >= S->o.max_iterations || ! ( res < prev_res ) ) {
         inner_status = B2S_NOT_CONVERGED;
         break;
      }
      prev_res = res;
      // inner FP32 solve from d = 0 to a relative tolerance; the last steps ask
      // only for what is left to reach tol
      // — never below 1e-6: an FP32 recurrence asked for more may never report it
      // (TFQMR on the 128^3 conv-diff matrix asked for 3e-7 iterated until the
      // wall-clock bound)
      const double inner_tol = std::max( { S->o.inner_tolerance, 0.5 * tol / res, kInnerFloor } );
      // GMRES: one restart cycle per refinement, so the FP64 correction lands
      // exactly where a plain restarted GMRES would restart anyway
      long long inner_max = S->o.max_iterations - total_it;
      if( S->o.solver == B2S_GMRES )
         inner_max = std::min< long long >( inner_max, S->o.gmres_restarting_max );
      Ctl c{};
      B2S_TRY( run_core< float >( S, vals32, diag32,
                                  S->o.solver == B2S_GMRES ? std::max( 0.5 * tol / res, 1e-7 ) : inner_tol, inner_max, c ) );
      total_it += c.it;
      last_inner = c.residue;
      refinements++;
      if( std::isnan( c.residue ) ) {
         inner_status = B2S_NAN;
         break;
      }
      refine_update_kernel<<< wave_grid( refine_update_kernel, n ), 256, 0, S->cs >>>( n, x64, v.x, v.x );
      B2S_TRY_CUDA( cudaGetLastError() );
   }
   (void) last_inner;
   rep.iterations = total_it;
   rep.residue = res;
   rep.true_residual = res;
   rep.refinements = refinements;
   if( std::isnan( res ) )
      rep.status = B2S_NAN;
   else if( res <= tol )
      rep.status = B2S_OK;
   else
      rep.status = inner_status != B2S_OK ? inner_status : B2S_NOT_CONVERGED;
   rep.converged = rep.status == B2S_OK;
   return B2S_OK;
}

// ---------------------------------------------------------------------------
// Mixed precision with reliable updates (CG, BiCGStab, BiCGStab(ell)): the
// FP32 recurrence is not restarted at a refinement; its residual is replaced
// by the FP64 one.
struct Reliable
{
   double normb = 0, res = 0;  // ||b|| and the last true relative residual
};

#ifndef B2S_RELIABLE_DELTA
#define B2S_RELIABLE_DELTA 0.1
#endif
static constexpr double kReliableDelta = B2S_RELIABLE_DELTA;  // residue reduction per phase

// x64 += d ; d = 0 ; b32 (or r32) = b64 - A64 x64 ; res = ||b64 - A64 x64|| / ||b64||
static b2s_status
reliable_residual( b2s_solver_t* S, float* r32_out, Reliable& R )
{
   const int64_t n = S->n, ln = ( n + 63 ) / 64 * 64;
   double* b64 = S->outer.as< double >();
   double* x64 = b64 + ln;
   auto v = vec_layout< float >( S );
   Ctl* ctl = S->ctl_buf.as< Ctl >();
   refine_update_kernel<<< wave_grid( refine_update_kernel, n ), 256, 0, S->cs >>>( n, x64, v.x, v.x );
   B2S_TRY_CUDA( cudaGetLastError() );
   RefineResSink< double > rsink{ b64, r32_out, ctl };
   B2S_TRY( ( spmv_dispatch< double, RefineResSink< double > >( S->A, S->A->values.as< double >(), x64, 0, S->A->rows,
                                                                rsink, S->scr.slot( 1 ), S->cs ) ) );
   B2S_TRY( read_ctl( S ) );
   R.res = S->h_ctl->outer_res / R.normb;
   return B2S_OK;
}

// host edits of the control block between phases (the stream is idle)
static b2s_status
write_ctl( b2s_solver_t* S )
{
   B2S_TRY_CUDA( cudaMemcpyAsync( S->ctl_buf.p, S->h_ctl, sizeof( Ctl ), cudaMemcpyHostToDevice, S->cs ) );
   return B2S_OK;
}

static b2s_status
mixed_reliable( b2s_solver_t* S, b2s_solve_report& rep )
{
   const int64_t n = S->n;
   const int64_t ln = ( n + 63 ) / 64 * 64;
   double* b64 = S->outer.as< double >();
   auto v = vec_layout< float >( S );
   const float* vals32 = S->A->values32.as< float >();
   const float* diag32 = S->o.preconditioner ? S->diag32.as< float >() : nullptr;
   Ctl* ctl = S->ctl_buf.as< Ctl >();
   const double tol = S->o.convergence_residue;
   const bool cg = S->o.solver == B2S_CG;
   const bool bl = S->o.solver == B2S_BICGSTABL;
   const long long tag = ( 3LL << 40 ) + ( (long long) S->o.solver << 32 );
   (void) ln;
   Reliable R;
   // ||b||
   B2S_TRY( init_ctl( S, 0, 0 ) );
   vec_kernel< double, NormOp< double >, NormbFin ><<< wave_grid( vec_kernel< double, NormOp< double >, NormbFin >, n ), kReduceBlock, 0, S->cs >>>(
      n, ctl, NormOp< double >{ b64, nullptr }, NormbFin{}, S->scr.slot( 0 ) );
   B2S_TRY_CUDA( cudaGetLastError() );
   B2S_TRY( read_ctl( S ) );
   R.normb = S->h_ctl->normb;
   // first residual (d = 0): r32 = b64 - A64 x64
   B2S_TRY_CUDA( cudaMemsetAsync( v.x, 0, n * sizeof( float ), S->cs ) );
   B2S_TRY( reliable_residual( S, cg ? v.r : v.b, R ) );
   long long updates = 0, it_carry = 0;
   int stalls = 0;
   double best = R.res;
   b2s_status st = B2S_OK;
   bool first = true;
   while( R.res > tol && ! std::isnan( R.res ) ) {
      // the phase's target: a kReliableDelta reduction, or what is left to tol
      const double factor = std::max( kReliableDelta, 0.5 * tol / R.res );
      if( ! first ) {
         // the last phase ended with `done` set; the replacement kernels run
         // only on a live control block
         S->h_ctl->done = 0;
         S->h_ctl->reason = 0;
         B2S_TRY( write_ctl( S ) );
      }
      if( cg ) {
         // z = M^-1 r ; p = z (first phase) ; s1 = (r, z) ; beta against s1_prev
         const int restart = first || stalls > 0 ? 1 : 0;
         if( first ) {
            Ctl c{};
            c.div_tol = S->o.divergence_residue;
            c.maxit = S->o.max_iterations;
            c.minit = S->o.min_iterations;
            c.normb = 1.0;
            *S->h_ctl = c;
            B2S_TRY( write_ctl( S ) );
         }
         vec_kernel< float, CgReplaceOp< float >, CgReplaceFin ><<< wave_grid( vec_kernel< float, CgReplaceOp< float >, CgReplaceFin >, n ), kReduceBlock, 0, S->cs >>>(
            n, ctl, CgReplaceOp< float >{ v.r, v.z, v.p, diag32, restart }, CgReplaceFin{ restart }, S->scr.slot( 2 ) );
         B2S_TRY_CUDA( cudaGetLastError() );
         if( ! restart ) {
            CgDirOp< float > dir{ v.p, diag32 ? v.z : v.r, 0.0f };
            vec_kernel< float, CgDirOp< float >, NoFin ><<< wave_grid( vec_kernel< float, CgDirOp< float >, NoFin >, n ), kReduceBlock, 0, S->cs >>>(
               n, ctl, dir, NoFin{}, S->scr.slot( 4 ) );
            B2S_TRY_CUDA( cudaGetLastError() );
         }
         B2S_TRY( read_ctl( S ) );
         if( first )
            S->h_ctl->it = 0;
         S->h_ctl->tol = S->h_ctl->residue * factor;
         if( first ) {
            // IterativeSolver::nextIteration before the first iteration
            if( S->h_ctl->residue < S->h_ctl->tol || S->h_ctl->it > S->h_ctl->maxit )
               S->h_ctl->done = 1;
            S->h_ctl->it++;
         }
         B2S_TRY( write_ctl( S ) );
         B2S_TRY( cg_iterate< float >( S, vals32, diag32, tag ) );
      }
      else if( bl ) {
         // BiCGStab(ell): phase 0 initialises from r_0 = M^-1 b32 (x = d = 0);
         // later phases replace r_0 and keep U_0, r_ast and the scalars
         if( first ) {
            if( updates > 0 ) {
               B2S_TRY( read_ctl( S ) );
               it_carry += S->h_ctl->it;
            }
            Ctl c{};
            c.div_tol = S->o.divergence_residue;
            c.maxit = std::max< long long >( 1, S->o.max_iterations - it_carry );
            c.minit = S->o.min_iterations;
            *S->h_ctl = c;
            B2S_TRY( write_ctl( S ) );
            B2S_TRY( bicgstabl_init< float >( S, vals32, diag32 ) );
         }
         else {
            vec_kernel< float, BlReplaceOp< float >, BlReplaceFin ><<< wave_grid( vec_kernel< float, BlReplaceOp< float >, BlReplaceFin >, n ), kReduceBlock, 0, S->cs >>>(
               n, ctl, BlReplaceOp< float >{ v.b, S->V.as< float >(), v.r_ast, diag32 }, BlReplaceFin{},
               S->scr.slot( 2 ) );
            B2S_TRY_CUDA( cudaGetLastError() );
         }
         B2S_TRY( read_ctl( S ) );
         S->h_ctl->tol = S->h_ctl->residue * factor;
         B2S_TRY( write_ctl( S ) );
         if( ! first ) {
            bl_resume_kernel<<< 1, 1, 0, S->cs >>>( ctl );
            B2S_TRY_CUDA( cudaGetLastError() );
         }
         B2S_TRY( bicgstabl_iterate< float >( S, vals32, diag32, tag ) );
      }
      else {
         // BiCGStab: phase 0 initialises from r = M^-1 b32 (x = d = 0);
         // later phases replace r and keep p, r_ast
         if( first ) {
            if( updates > 0 ) {
               B2S_TRY( read_ctl( S ) );
               it_carry += S->h_ctl->it;
            }
            Ctl c{};
            c.div_tol = S->o.divergence_residue;
            c.maxit = std::max< long long >( 1, S->o.max_iterations - it_carry );
            c.minit = S->o.min_iterations;
            *S->h_ctl = c;
            B2S_TRY( write_ctl( S ) );
            vec_kernel< float, NormOp< float >, NormbFin ><<< wave_grid( vec_kernel< float, NormOp< float >, NormbFin >, n ), kReduceBlock, 0, S->cs >>>(
               n, ctl, NormOp< float >{ v.b, diag32 }, NormbFin{}, S->scr.slot( 0 ) );
            B2S_TRY_CUDA( cudaGetLastError() );
            BiResG< float > rs;
            rs.b = v.b;
            rs.r = v.r;
            rs.r_ast = v.r_ast;
            rs.p = v.p;
            rs.s = v.s;
            rs.diag = diag32;
            rs.ctl = ctl;
            rs.mode = 0;
            rs.exact = 0;
            B2S_TRY( ( spmv_dispatch< float, BiResG< float > >( S->A, vals32, v.x, 0, S->A->rows, rs, S->scr.slot( 1 ),
                                                                S->cs ) ) );
         }
         else {
            vec_kernel< float, BiReplaceOp< float >, BiReplaceFin ><<< wave_grid( vec_kernel< float, BiReplaceOp< float >, BiReplaceFin >, n ), kReduceBlock, 0, S->cs >>>(
               n, ctl, BiReplaceOp< float >{ v.b, v.r, v.r_ast, diag32 }, BiReplaceFin{}, S->scr.slot( 2 ) );
            B2S_TRY_CUDA( cudaGetLastError() );
            vec_kernel< float, BiPOp< float >, NoFin ><<< wave_grid( vec_kernel< float, BiPOp< float >, NoFin >, n ), kReduceBlock, 0, S->cs >>>(
               n, ctl, BiPOp< float >{ v.p, v.r, v.Ap, 0.0f, 0.0f }, NoFin{}, S->scr.slot( 8 ) );
            B2S_TRY_CUDA( cudaGetLastError() );
         }
         B2S_TRY( read_ctl( S ) );
         S->h_ctl->tol = S->h_ctl->residue * factor;
         B2S_TRY( write_ctl( S ) );
         B2S_TRY( bicgstab_iterate< float >( S, vals32, diag32, tag ) );
      }
      first = false;
      B2S_TRY( read_ctl( S ) );
      const Ctl c = *S->h_ctl;
      // x64 += d ; residual replaced from FP64
      B2S_TRY( reliable_residual( S, cg ? v.r : v.b, R ) );
      updates++;
      if( std::isnan( R.res ) || std::isnan( c.residue ) ) {
         st = B2S_NAN;
         break;
      }
      if( R.res <= tol )
         break;
      if( c.it >= c.maxit ) {
         st = B2S_NOT_CONVERGED;
         break;
      }
      // no progress: restart the recurrence from the true residual; give up
      // after three phases without progress
      if( R.res < best * 0.9 ) {
         best = R.res;
         stalls = 0;
      }
      else if( ++stalls >= 3 ) {
         st = B2S_NOT_CONVERGED;
         break;
      }
#ifndef B2S_RELIABLE_NO_RESTART
      if( ! cg && stalls > 0 )
         first = true;  // BiCGStab restart: new shadow residual from the true one
#endif
   }
   B2S_TRY( read_ctl( S ) );
   rep.iterations = it_carry + S->h_ctl->it;
   rep.residue = R.res;
   rep.true_residual = R.res;
   rep.refinements = updates;
   rep.status = std::isnan( R.res ) ? B2S_NAN : ( R.res <= tol ? B2S_OK : ( st != B2S_OK ? st : B2S_NOT_CONVERGED ) );
   rep.converged = rep.status == B2S_OK;
   return B2S_OK;
}

static b2s_status
solve_mixed( b2s_solver_t* S, b2s_solve_report& rep )
{
   if( S->o.solver == B2S_CG || S->o.solver == B2S_BICGSTAB || S->o.solver == B2S_BICGSTABL )
      return mixed_reliable( S, rep );
   return mixed_refine( S, rep );
}

template< typename Real >
__global__ void
cast_vec_kernel( const Real* __restrict__ in, float* __restrict__ out, int64_t n )
{
   for( int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x )
      out[ i ] = (float) in[ i ];
}

}  // namespace b2s

extern "C" {

void
b2s_solve_opts_default( b2s_solve_opts* o )
{
   if( ! o )
      return;
   std::memset( o, 0, sizeof( *o ) );
   o->solver = B2S_CG;
   o->preconditioner = B2S_PRECOND_NONE;
   o->convergence_residue = 1e-6;
   o->divergence_residue = DBL_MAX;
   o->max_iterations = 1000000000;
   o->min_iterations = 0;
   o->gmres_variant = B2S_GMRES_MGSR;
   o->gmres_restarting_min = 10;
   o->gmres_restarting_max = 10;
   o->gmres_restarting_step_min = 3;
   o->gmres_restarting_step_max = 3;
   o->bicgstab_exact_residue = 0;
   o->bicgstab_ell = 1;
   o->precision = B2S_PRECISION_PLAIN;
   o->inner_tolerance = 1e-4;
   o->max_refinements = 20;
   o->check_interval = 0;
   o->omega = 1.0;
   o->residue_period = 4;
   o->ilut_p = 0;
   o->ilut_threshold = 1e-4;
}

b2s_status
b2s_solver_create( b2s_matrix A, const b2s_solve_opts* opts, b2s_solver* out )
{
   clear_error();
   B2S_NO_BINARY( A, "a solver" );
   B2S_CHECK_ARG( A && out, "NULL argument" );
   *out = nullptr;
   B2S_CHECK_ARG( A->rows == A->cols, "the matrix must be square" );
   b2s_solve_opts o;
   b2s_solve_opts_default( &o );
   if( opts )
      o = *opts;
   B2S_CHECK_ARG( o.solver >= B2S_CG && o.solver <= B2S_SOR, "solver" );
   if( o.solver == B2S_JACOBI || o.solver == B2S_SOR ) {
      // TNL's stationary solvers take no preconditioner (setPreconditioner is
      // accepted and unused) and have no mixed-precision form here
      B2S_CHECK_ARG( o.residue_period > 0, "residue_period > 0" );
      if( o.precision == B2S_PRECISION_MIXED ) {
         set_error( "Jacobi and SOR run in the matrix value type only" );
         return B2S_UNSUPPORTED;
      }
      o.preconditioner = B2S_PRECOND_NONE;
   }
   if( o.solver == B2S_BICGSTABL ) {
      if( o.bicgstab_ell == 0 )
         o.bicgstab_ell = 1;  // TNL's default for "bicgstab-ell"
      B2S_CHECK_ARG( o.bicgstab_ell >= 1 && o.bicgstab_ell <= kMaxEll, "bicgstab_ell in [1, 16]" );
   }
   B2S_CHECK_ARG( o.preconditioner >= B2S_PRECOND_NONE && o.preconditioner <= B2S_PRECOND_ILUT, "preconditioner" );
   if( ( o.preconditioner == B2S_PRECOND_ILU0 || o.preconditioner == B2S_PRECOND_ILUT )
       && o.precision == B2S_PRECISION_MIXED ) {
      set_error( "ILU(0) and ILUT are provided for the plain (single-precision-type) solves" );
      return B2S_UNSUPPORTED;
   }
   if( o.preconditioner == B2S_PRECOND_ILUT )
      B2S_CHECK_ARG( o.ilut_p >= 0, "ilut_p >= 0" );
   B2S_CHECK_ARG( o.precision == 0 || o.precision == 1, "precision" );
   if( o.solver == B2S_GMRES ) {
      // GMRES.hpp:78-90
      if( o.gmres_restarting_min <= 0 || o.gmres_restarting_max <= 0 || o.gmres_restarting_min > o.gmres_restarting_max ) {
         set_error( "wrong GMRES restarting parameters: r_min = %d, r_max = %d", o.gmres_restarting_min,
                    o.gmres_restarting_max );
         return B2S_INVALID_ARG;
      }
      if( o.gmres_restarting_step_min < 0 || o.gmres_restarting_step_max < 0
          || o.gmres_restarting_step_min > o.gmres_restarting_step_max ) {
         set_error( "wrong GMRES restarting adjustment parameters" );
         return B2S_INVALID_ARG;
      }
      B2S_CHECK_ARG( o.gmres_variant >= B2S_GMRES_CGS && o.gmres_variant <= B2S_GMRES_CWY, "gmres_variant" );
      B2S_CHECK_ARG( o.gmres_restarting_max <= 255, "gmres_restarting_max <= 255" );
   }
   if( o.precision == B2S_PRECISION_MIXED && A->dtype != B2S_F64 ) {
      set_error( "mixed precision needs an FP64 matrix (the FP32 copy is made by the solver)" );
      return B2S_INVALID_ARG;
   }
   std::unique_ptr< b2s_solver_t > S( new b2s_solver_t() );
   S->A = A;
   if( A->symmetric ) {
      // the solvers fuse their dot products into the product's row pass, which
      // needs whole rows: they run on the general form L + L^T - D
      B2S_TRY( expand_symmetric( A, nullptr, &S->expanded ) );
      B2S_TRY_CUDA( cudaStreamSynchronize( nullptr ) );  // the solver's own stream does not wait on stream 0
      S->A = A = S->expanded;
   }
   S->o = o;
   S->mixed = o.precision == B2S_PRECISION_MIXED;
   S->n = A->rows;
   const AllocCtx* actx = thread_alloc_ctx();
   if( actx && actx->solver_stream ) {
      S->cs = actx->solver_stream;
      S->ev0 = actx->ev0;
      S->ev1 = actx->ev1;
      S->owns_stream = false;
   }
   else
      B2S_TRY_CUDA( cudaStreamCreateWithFlags( &S->cs, cudaStreamNonBlocking ) );
   if( thread_alloc_ctx() ) {
      // server workers: pageable mirror (cudaFreeHost would wait for the
      // other requests' kernels)
      S->h_ctl = new Ctl();
   }
   else {
      B2S_TRY_CUDA( cudaMallocHost( &S->h_ctl, sizeof( Ctl ) ) );
      S->h_ctl_pinned = true;
   }
   if( S->owns_stream ) {
      B2S_TRY_CUDA( cudaEventCreate( &S->ev0 ) );
      B2S_TRY_CUDA( cudaEventCreate( &S->ev1 ) );
   }
   B2S_TRY( S->ctl_buf.alloc( sizeof( Ctl ) ) );
   B2S_TRY( S->scr.init( 10, S->cs ) );
   B2S_TRY( S->md_partials.alloc( (size_t) kMd * kMaxReduceGrid * sizeof( double ) ) );
   B2S_TRY( S->md_counter.alloc( 64 ) );
   B2S_TRY_CUDA( cudaMemsetAsync( S->md_counter.p, 0, 64, S->cs ) );
   const size_t es = ( S->mixed || A->dtype == B2S_F32 ) ? 4 : 8;
   const int64_t ln = ( (int64_t) S->n + 63 ) / 64 * 64;
   B2S_TRY( S->vecs.alloc( (size_t) 10 * ln * es ) );
   B2S_TRY_CUDA( cudaMemsetAsync( S->vecs.p, 0, (size_t) 10 * ln * es, S->cs ) );
   if( S->mixed ) {
      cudaStream_t s0 = S->cs;
      B2S_TRY( ensure_fp32_copy( A, s0 ) );
      B2S_TRY( S->outer.alloc( (size_t) 2 * ln * sizeof( double ) ) );
      if( o.preconditioner ) {
         B2S_TRY( S->diag32.alloc( (size_t) std::max( S->n, 1 ) * sizeof( float ) ) );
         if( S->n > 0 ) {
            cast_vec_kernel< double ><<< wave_grid( cast_vec_kernel< double >, S->n ), 256, 0, s0 >>>( A->diagonal.as< double >(), S->diag32.as< float >(),
                                                                       S->n );
            B2S_TRY_CUDA( cudaGetLastError() );
         }
      }
   }
   if( o.preconditioner == B2S_PRECOND_ILU0 ) {
      // Preconditioner::update( matrix ): the factorization, once per solver
      if( A->dtype == B2S_F64 )
         B2S_TRY( ilu_factorize< double >( A, A->values.as< double >(), S->ilu64, S->cs ) );
      else
         B2S_TRY( ilu_factorize< float >( A, A->values.as< float >(), S->ilu32, S->cs ) );
   }
   if( o.preconditioner == B2S_PRECOND_ILUT ) {
      if( A->dtype == B2S_F64 )
         B2S_TRY( ilut_factorize< double >( A, o.ilut_p, o.ilut_threshold, S->ilu64, S->cs ) );
      else
         B2S_TRY( ilut_factorize< float >( A, o.ilut_p, o.ilut_threshold, S->ilu32, S->cs ) );
   }
   if( o.solver == B2S_GMRES ) {
      const int M = o.gmres_restarting_max;
      S->mmax = M;
      S->ld = ( (int64_t) S->n + 31 ) / 32 * 32;  // columns aligned to 256 B (GMRES.hpp:765-772)
      B2S_TRY( S->V.alloc( (size_t) ( M + 1 ) * S->ld * es ) );
      B2S_TRY( S->gm.alloc( (size_t) ( ( M + 1 ) * M + 5 * ( M + 1 ) ) * sizeof( double ) ) );
   }
   if( o.solver == B2S_SOR ) {
      // the sweep's level order, once per solver
      if( A->dtype == B2S_F64 )
         B2S_TRY( S->sor64.build( A, S->cs ) );
      else
         B2S_TRY( S->sor32.build( A, S->cs ) );
   }
   if( o.solver == B2S_BICGSTABL ) {
      // R and U, ell + 1 columns each (BICGStabL.hpp:280-285), and T, sigma, g_0..g_2
      const int ell = o.bicgstab_ell;
      S->ld = ( (int64_t) S->n + 31 ) / 32 * 32;
      const size_t bytes = (size_t) 2 * ( ell + 1 ) * S->ld * es;
      B2S_TRY( S->V.alloc( std::max< size_t >( bytes, 64 ) ) );
      B2S_TRY_CUDA( cudaMemsetAsync( S->V.p, 0, std::max< size_t >( bytes, 64 ), S->cs ) );
      const size_t gbytes = (size_t) ( ell * ell + 4 * ( ell + 1 ) ) * sizeof( double );
      B2S_TRY( S->gm.alloc( gbytes ) );
      B2S_TRY_CUDA( cudaMemsetAsync( S->gm.p, 0, gbytes, S->cs ) );
   }
   B2S_TRY_CUDA( cudaStreamSynchronize( S->cs ) );
   *out = S.release();
   return B2S_OK;
}

b2s_status
b2s_solver_destroy( b2s_solver s )
{
   clear_error();
   if( s )
      cudaStreamSynchronize( s->cs );
   delete s;
   return B2S_OK;
}

b2s_status
b2s_solve( b2s_solver S, const void* b, void* x, b2s_memory where, b2s_stream stream, b2s_solve_report* report )
{
   clear_error();
   B2S_CHECK_ARG( S && ( b || S->n == 0 ) && ( x || S->n == 0 ), "NULL argument" );
   B2S_CHECK_ARG( where == B2S_HOST || where == B2S_DEVICE, "where" );
   b2s_solve_report rep{};
   const int64_t n = S->n;
   cudaStream_t us = as_stream( stream );
   S->t_start = std::chrono::steady_clock::now();
   // order the solver's private stream after the caller's stream
   B2S_TRY_CUDA( cudaEventRecord( S->ev0, us ) );
   B2S_TRY_CUDA( cudaStreamWaitEvent( S->cs, S->ev0, 0 ) );
   const size_t ues = S->A->dtype == B2S_F64 ? 8 : 4;  // user-facing value size (FP64 for mixed)
   const cudaMemcpyKind k_in = where == B2S_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
   const cudaMemcpyKind k_out = where == B2S_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
   void *db, *dx;
   if( S->mixed ) {
      const int64_t ln = ( n + 63 ) / 64 * 64;
      db = S->outer.as< double >();
      dx = S->outer.as< double >() + ln;
   }
   else if( S->A->dtype == B2S_F64 ) {
      auto v = vec_layout< double >( S );
      db = v.b;
      dx = v.x;
   }
   else {
      auto v = vec_layout< float >( S );
      db = v.b;
      dx = v.x;
   }
   if( n > 0 ) {
      B2S_TRY_CUDA( cudaMemcpyAsync( db, b, n * ues, k_in, S->cs ) );
      B2S_TRY_CUDA( cudaMemcpyAsync( dx, x, n * ues, k_in, S->cs ) );
   }
   B2S_TRY_CUDA( cudaEventRecord( S->ev0, S->cs ) );
   b2s_status st = S->mixed ? solve_mixed( S, rep ) : solve_plain( S, rep );
   if( st != B2S_OK )
      return st;
   B2S_TRY_CUDA( cudaEventRecord( S->ev1, S->cs ) );
   if( n > 0 )
      B2S_TRY_CUDA( cudaMemcpyAsync( x, dx, n * ues, k_out, S->cs ) );
   B2S_TRY_CUDA( cudaStreamSynchronize( S->cs ) );
   float ms = 0;
   cudaEventElapsedTime( &ms, S->ev0, S->ev1 );
   rep.device_ms = ms;
   // the caller's stream sees the result
   B2S_TRY_CUDA( cudaEventRecord( S->ev1, S->cs ) );
   B2S_TRY_CUDA( cudaStreamWaitEvent( us, S->ev1, 0 ) );
   if( report )
      *report = rep;
   return (b2s_status) rep.status;
}

}  // extern "C"
