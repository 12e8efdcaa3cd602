// Device side of TFQMR (Solvers/Linear/TFQMR.hpp:18-114) and BiCGStab(ell)
// (Solvers/Linear/BICGStabL.hpp:42-250): SpMV sinks and fused vector passes
// whose last block ("finisher") advances the scalar recurrences in the
// control block, as for CG / BiCGStab.
#pragma once

#include "krylov_kernels.cuh"

namespace b2s {

// ---------------------------------------------------------------------------
// TFQMR. Vectors: r, w, u, v, Au, d, r_ast. TNL's iteration m (counted from 1)
// computes alpha = rho / (v, r_ast) when m is odd, Au = M^-1 A u when m is
// even, then w -= alpha Au, d = u + (theta^2 eta / alpha) d, the QMR scalars,
// x += eta d, and either u -= alpha v (odd) or rho, beta, u = w + beta u,
// v = beta Au + beta^2 v, Au = M^-1 A u, v += Au (even). Here the x update of
// iteration m runs inside iteration m+1's first pass (before d changes), and
// once more after the loop for the last iteration (tf_flush_kernel).

// r = M^-1 (b - A x) ; w = u = r_ast = r ; d = 0 ; acc (r, r) -> tau, rho
template< typename Real >
struct TfInitSink
{
   static constexpr int NR = 1;
   const Real* b;
   Real *r, *w, *u, *r_ast, *d;
   const Real* diag;
   Ctl* ctl;
   int pre = 0;  // 1: sv is already M^-1 (b - A x)
   __device__ bool skip() const { return false; }
   __device__ __forceinline__ void
   put( int row, Real sv, double* acc ) const
   {
      Real rr = pre ? sv : b[ row ] - sv;
      if( diag && ! pre )
         rr = rr / diag[ row ];
      r[ row ] = rr;
      w[ row ] = rr;
      u[ row ] = rr;
      r_ast[ row ] = rr;
      d[ row ] = 0;
      acc[ 0 ] += (double) rr * (double) rr;
   }
   __device__ void
   finish( const double* t ) const
   {
      Ctl& c = *ctl;
      c.tf_tau = sqrt( t[ 0 ] );
      c.tf_rho = t[ 0 ];  // (r_ast, r) with r_ast = r
      c.tf_theta = c.tf_eta = c.tf_alpha = 0.0;
   }
};

// Au = M^-1 A u. MODE 0 (start): v = Au, acc (v, r_ast) -> residue, first
// nextIteration, alpha of iteration 1. MODE 1 (even iteration, first
// product): Au only. MODE 2 (even iteration, second product): v += Au,
// acc (v, r_ast) -> alpha of the next (odd) iteration, nextIteration.
template< typename Real, int MODE >
struct TfAuSink
{
   static constexpr int NR = MODE == 1 ? 0 : 1;
   Real *Au, *v;
   const Real *r_ast, *diag;
   Ctl* ctl;
   int pre = 0;
   __device__ bool skip() const { return MODE != 0 && ctl->done != 0; }
   __device__ __forceinline__ void
   put( int row, Real sv, double* acc ) const
   {
      if( diag && ! pre )
         sv = sv / diag[ row ];
      Au[ row ] = sv;
      if constexpr( MODE == 0 ) {
         v[ row ] = sv;
         acc[ 0 ] += (double) sv * (double) r_ast[ row ];
      }
      if constexpr( MODE == 2 ) {
         const Real vv = v[ row ] + sv;
         v[ row ] = vv;
         acc[ 0 ] += (double) vv * (double) r_ast[ row ];
      }
   }
   __device__ void
   finish( const double* t ) const
   {
      Ctl& c = *ctl;
      if constexpr( MODE == 0 ) {
         c.it = 0;
         c.residue = c.tf_tau / c.normb;
      }
      c.tf_alpha = c.tf_rho / t[ 0 ];
      next_iteration( c );
   }
};

// x += eta d (the previous iteration's) ; w -= alpha Au ; d = u + (theta^2 eta / alpha) d ;
// acc (w, w) [, (w, r_ast) in even iterations]
template< typename Real, bool EVEN >
struct TfStepOp
{
   static constexpr int NR = EVEN ? 2 : 1;
   Real *x, *w, *d;
   const Real *u, *Au, *r_ast;
   Real eta, alpha, coef;
   __device__ __forceinline__ void
   load( const Ctl& c )
   {
      eta = (Real) c.tf_eta;
      alpha = (Real) c.tf_alpha;
      coef = (Real) ( c.tf_theta * c.tf_theta * c.tf_eta / c.tf_alpha );
   }
   __device__ __forceinline__ void
   operator()( int64_t i, double* acc ) const
   {
      const Real dd = d[ i ];
      x[ i ] += eta * dd;
      const Real ww = w[ i ] - alpha * Au[ i ];
      w[ i ] = ww;
      d[ i ] = u[ i ] + coef * dd;
      acc[ 0 ] += (double) ww * (double) ww;
      if constexpr( EVEN )
         acc[ 1 ] += (double) ww * (double) r_ast[ i ];
   }
   __device__ __forceinline__ void
   apply4( int64_t i, double* acc ) const
   {
      V4< Real > X = ld4( x + i ), W = ld4( w + i ), D = ld4( d + i );
      const V4< Real > U = ld4( u + i ), AU = ld4( Au + i );
      V4< Real > RA;
      if constexpr( EVEN )
         RA = ld4( r_ast + i );
#pragma unroll
      for( int k = 0; k < 4; k++ ) {
         const Real dd = D.v[ k ];
         X.v[ k ] += eta * dd;
         const Real ww = W.v[ k ] - alpha * AU.v[ k ];
         W.v[ k ] = ww;
         D.v[ k ] = U.v[ k ] + coef * dd;
         acc[ 0 ] += (double) ww * (double) ww;
         if constexpr( EVEN )
            acc[ 1 ] += (double) ww * (double) RA.v[ k ];
      }
      st4( x + i, X );
      st4( w + i, W );
      st4( d + i, D );
   }
};

// theta, c, tau, eta, residue = tau sqrt(m + 1) / ||M^-1 b|| and the
// convergence break (TFQMR.hpp:79-89); even iterations: rho, beta
// (:91-94); odd iterations end here (nextIteration of the next one)
template< bool EVEN >
struct TfStepFin
{
   static constexpr bool active = true;
   __device__ void
   operator()( Ctl& c, const double* t ) const
   {
      const double w_norm = sqrt( t[ 0 ] );
      c.tf_theta = w_norm / c.tf_tau;
      const double cc = 1.0 / sqrt( 1.0 + c.tf_theta * c.tf_theta );
      c.tf_tau = c.tf_tau * c.tf_theta * cc;
      c.tf_eta = cc * cc * c.tf_alpha;
      c.residue = c.tf_tau * sqrt( (double) ( c.it + 1 ) ) / c.normb;
      if( c.it > c.minit && c.residue < c.tol ) {
         c.done = 1;
         c.reason = 1;
         return;
      }
      if constexpr( EVEN ) {
         const double rho_new = t[ 1 ];
         c.tf_beta = rho_new / c.tf_rho;
         c.tf_rho = rho_new;
      }
      else
         next_iteration( c );
   }
};

// odd iterations: u -= alpha v
template< typename Real >
struct TfUOp
{
   static constexpr int NR = 1;
   Real* u;
   const Real* v;
   Real alpha;
   __device__ __forceinline__ void load( const Ctl& c ) { alpha = (Real) c.tf_alpha; }
   __device__ __forceinline__ void operator()( int64_t i, double* ) const { u[ i ] = u[ i ] - alpha * v[ i ]; }
   __device__ __forceinline__ void
   apply4( int64_t i, double* ) const
   {
      V4< Real > U = ld4( u + i );
      const V4< Real > V = ld4( v + i );
#pragma unroll
      for( int k = 0; k < 4; k++ )
         U.v[ k ] = U.v[ k ] - alpha * V.v[ k ];
      st4( u + i, U );
   }
};

// even iterations: u = w + beta u ; v = beta Au + beta^2 v
template< typename Real >
struct TfDirOp
{
   static constexpr int NR = 1;
   Real *u, *v;
   const Real *w, *Au;
   Real beta, beta2;
   __device__ __forceinline__ void
   load( const Ctl& c )
   {
      beta = (Real) c.tf_beta;
      beta2 = beta * beta;
   }
   __device__ __forceinline__ void
   operator()( int64_t i, double* ) const
   {
      u[ i ] = w[ i ] + beta * u[ i ];
      v[ i ] = beta * Au[ i ] + beta2 * v[ i ];
   }
   __device__ __forceinline__ void
   apply4( int64_t i, double* ) const
   {
      V4< Real > U = ld4( u + i ), V = ld4( v + i );
      const V4< Real > W = ld4( w + i ), AU = ld4( Au + i );
#pragma unroll
      for( int k = 0; k < 4; k++ ) {
         U.v[ k ] = W.v[ k ] + beta * U.v[ k ];
         V.v[ k ] = beta * AU.v[ k ] + beta2 * V.v[ k ];
      }
      st4( u + i, U );
      st4( v + i, V );
   }
};

// x += eta d of the last iteration (runs once, after the loop has ended)
template< typename Real >
__global__ void __launch_bounds__( kReduceBlock )
tf_flush_kernel( int64_t n, const Ctl* ctl, Real* __restrict__ x, const Real* __restrict__ d )
{
   const Real eta = (Real) ctl->tf_eta;
   for( int64_t i = blockIdx.x * (int64_t) kReduceBlock + threadIdx.x; i < n; i += (int64_t) gridDim.x * kReduceBlock )
      x[ i ] += eta * d[ i ];
}

// ---------------------------------------------------------------------------
// BiCGStab(ell). R_0..R_ell and U_0..U_ell are columns of two column-major
// arrays with leading dimension ld; r_0 = R_0, u_0 = U_0. The small arrays
// (T, sigma_1..ell, g_0, g_1, g_2) live in device memory.
constexpr int kMaxEll = 16;

struct BlArrays
{
   double *T, *sigma, *g0, *g1, *g2;  // T: ell x ell (T[(i-1) + (j-1) ell]); the rest ell + 1
   int ell;
};

// the start of step j of the Bi-CG part: nextIteration, rho_1 = (r_ast, r_j),
// beta = alpha rho_1 / rho_0, rho_0 = rho_1 (BICGStabL.hpp:85-93)
__device__ __forceinline__ void
bl_step( Ctl& c, double rho1 )
{
   c.it++;
   c.bl_beta = c.bl_alpha * rho1 / c.bl_rho0;
   c.bl_rho0 = rho1;
}

// the outer loop's test (checkNextIteration, no count) and rho_0 = -omega rho_0,
// then step 0 with rho_1 = (r_ast, r_0) taken from the last pass over r_0
__device__ __forceinline__ void
bl_outer( Ctl& c )
{
   if( ! check_next( c ) ) {
      c.done = 1;
      c.reason = 1;
      return;
   }
   c.bl_rho0 = -c.bl_omega * c.bl_rho0;
   bl_step( c, c.bl_rho1 );
}

// r = M^-1 (b - A x) ; acc (r, r). MODE 0: r_0 at the start (sigma_0);
// MODE 1: the exact residue (bicgstab-exact-residue) -> residue, outer test.
template< typename Real, int MODE >
struct BlResSink
{
   static constexpr int NR = 1;
   const Real* b;
   Real* r;
   const Real* diag;
   Ctl* ctl;
   int pre = 0;
   __device__ bool skip() const { return MODE != 0 && ctl->done != 0; }
   __device__ __forceinline__ void
   put( int row, Real sv, double* acc ) const
   {
      Real rr = pre ? sv : b[ row ] - sv;
      if( diag && ! pre )
         rr = rr / diag[ row ];
      r[ row ] = rr;
      acc[ 0 ] += (double) rr * (double) rr;
   }
   __device__ void
   finish( const double* t ) const
   {
      Ctl& c = *ctl;
      if constexpr( MODE == 0 ) {
         c.bl_sigma0 = sqrt( t[ 0 ] );
         if( isnan( c.bl_sigma0 ) ) {
            // TNL throws "initial residue is NAN" (BICGStabL.hpp:63-64)
            c.residue = c.bl_sigma0;
            c.done = 1;
            c.reason = 1;
         }
      }
      else {
         c.residue = sqrt( t[ 0 ] ) / c.normb;
         bl_outer( c );
      }
   }
};

// r_ast = r_0 / sigma_0 ; u_0 = 0 ; acc (r_ast, r_0) (BICGStabL.hpp:66-73)
template< typename Real >
struct BlInitOp
{
   static constexpr int NR = 1;
   const Real* r0;
   Real *r_ast, *u0;
   Real sigma0;
   __device__ __forceinline__ void load( const Ctl& c ) { sigma0 = (Real) c.bl_sigma0; }
   __device__ __forceinline__ void
   operator()( int64_t i, double* acc ) const
   {
      const Real r = r0[ i ];
      const Real ra = r / sigma0;
      r_ast[ i ] = ra;
      u0[ i ] = 0;
      acc[ 0 ] += (double) ra * (double) r;
   }
};
struct BlInitFin
{
   static constexpr bool active = true;
   __device__ void
   operator()( Ctl& c, const double* t ) const
   {
      c.bl_rho0 = 1.0;
      c.bl_alpha = 0.0;
      c.bl_omega = 1.0;
      c.it = 0;
      c.residue = c.bl_sigma0 / c.normb;
      c.bl_rho1 = t[ 0 ];
      bl_outer( c );
   }
};

// U_c = R_c - beta U_c for c = 0..j (geam, BICGStabL.hpp:95-101)
template< typename Real >
struct BlGeamUOp
{
   static constexpr int NR = 1;
   const Real* R;
   Real* U;
   int64_t ld;
   int j;
   Real beta;
   __device__ __forceinline__ void load( const Ctl& c ) { beta = (Real) c.bl_beta; }
   __device__ __forceinline__ void
   operator()( int64_t i, double* ) const
   {
      for( int c = 0; c <= j; c++ )
         U[ c * ld + i ] = R[ c * ld + i ] - beta * U[ c * ld + i ];
   }
};

// dst = M^-1 A src ; acc (r_ast, dst). LAST_R = false: dst = u_{j+1}, gamma ->
// alpha = rho_0 / gamma (BICGStabL.hpp:103-113). LAST_R = true: dst = r_{j+1};
// unless j + 1 = ell, the finisher starts step j + 1.
template< typename Real, bool R_STEP >
struct BlMatvecSink
{
   static constexpr int NR = 1;
   Real* dst;
   const Real *r_ast, *diag;
   Ctl* ctl;
   int last;  // R_STEP: j + 1 == ell
   int pre = 0;
   __device__ bool skip() const { return ctl->done != 0; }
   __device__ __forceinline__ void
   put( int row, Real sv, double* acc ) const
   {
      if( diag && ! pre )
         sv = sv / diag[ row ];
      dst[ row ] = sv;
      acc[ 0 ] += (double) r_ast[ row ] * (double) sv;
   }
   __device__ void
   finish( const double* t ) const
   {
      Ctl& c = *ctl;
      if constexpr( ! R_STEP )
         c.bl_alpha = c.bl_rho0 / t[ 0 ];
      else if( ! last )
         bl_step( c, t[ 0 ] );
   }
};

// R_c -= alpha U_{c+1} for c = 0..j ; x += alpha u_0 (BICGStabL.hpp:115-146)
template< typename Real >
struct BlRUpdateOp
{
   static constexpr int NR = 1;
   Real* R;
   const Real* U;
   Real* x;
   int64_t ld;
   int j;
   Real alpha;
   __device__ __forceinline__ void load( const Ctl& c ) { alpha = (Real) c.bl_alpha; }
   __device__ __forceinline__ void
   operator()( int64_t i, double* ) const
   {
      for( int c = 0; c <= j; c++ )
         R[ c * ld + i ] = R[ c * ld + i ] - alpha * U[ ( c + 1 ) * ld + i ];
      x[ i ] += alpha * U[ i ];
   }
};

// MGS of column j, pass k = 1..j (BICGStabL.hpp:152-166): first r_j -= T_{k-1,j} r_{k-1}
// (k > 1); then acc (r_k, r_j) for T_{k,j} (k < j), or (r_j, r_j) and (r_0, r_j) for
// sigma_j and g_1[j] (k = j)
template< typename Real >
struct BlMgsOp
{
   static constexpr int NR = 2;
   Real* R;
   int64_t ld;
   int j, k;
   BlArrays g;
   Real t_prev;
   __device__ __forceinline__ void
   load( const Ctl& )
   {
      t_prev = k > 1 ? (Real) __ldcg( g.T + ( k - 2 ) + ( j - 1 ) * g.ell ) : Real( 0 );
   }
   __device__ __forceinline__ void
   operator()( int64_t i, double* acc ) const
   {
      Real rj = R[ j * ld + i ];
      if( k > 1 ) {
         rj = rj - t_prev * R[ ( k - 1 ) * ld + i ];
         R[ j * ld + i ] = rj;
      }
      if( k < j )
         acc[ 0 ] += (double) R[ k * ld + i ] * (double) rj;
      else {
         acc[ 0 ] += (double) rj * (double) rj;
         acc[ 1 ] += (double) R[ i ] * (double) rj;
      }
   }
};

// T_{k,j} = (r_k, r_j) / sigma_k, or sigma_j and g_1[j] = (r_0, r_j) / sigma_j;
// after the last column: omega, g_0 = T^-1 g_1, g_2 = T S g_0 (BICGStabL.hpp:168-193)
struct BlMgsFin
{
   static constexpr bool active = true;
   BlArrays g;
   int j, k;
   __device__ void
   operator()( Ctl& c, const double* t ) const
   {
      const int ell = g.ell;
      double* T = g.T;
      if( k < j ) {
         T[ ( k - 1 ) + ( j - 1 ) * ell ] = t[ 0 ] / g.sigma[ k ];
         return;
      }
      g.sigma[ j ] = t[ 0 ];
      g.g1[ j ] = t[ 1 ] / g.sigma[ j ];
      if( j < ell )
         return;
      c.bl_omega = g.g1[ ell ];
      for( int jj = ell; jj >= 1; jj-- ) {
         double s = g.g1[ jj ];
         for( int i = jj + 1; i <= ell; i++ )
            s -= T[ ( jj - 1 ) + ( i - 1 ) * ell ] * g.g0[ i ];
         g.g0[ jj ] = s;
      }
      for( int jj = 1; jj < ell; jj++ ) {
         double s = g.g0[ jj + 1 ];
         for( int i = jj + 1; i < ell; i++ )
            s += T[ ( jj - 1 ) + ( i - 1 ) * ell ] * g.g0[ i + 1 ];
         g.g2[ jj ] = s;
      }
      g.g2[ 0 ] = g.g0[ 1 ];
   }
};

// x += R_[0:ell-1] g_2 ; r_0 -= R_[1:ell] g_1[1:ell] ; u_0 -= U_[1:ell] g_0[1:ell]
// (gemv: the column sum first, then added to y; BICGStabL.hpp:196-231) ;
// acc (r_0, r_0), (r_ast, r_0)
template< typename Real >
struct BlFinalOp
{
   static constexpr int NR = 2;
   Real *x, *R, *U;
   const Real* r_ast;
   int64_t ld;
   BlArrays g;
   Real c2[ kMaxEll ], c1[ kMaxEll ], c0[ kMaxEll ];
   __device__ __forceinline__ void
   load( const Ctl& )
   {
      for( int k = 0; k < g.ell; k++ ) {
         c2[ k ] = (Real) __ldcg( g.g2 + k );
         c1[ k ] = -(Real) __ldcg( g.g1 + k + 1 );
         c0[ k ] = -(Real) __ldcg( g.g0 + k + 1 );
      }
   }
   __device__ __forceinline__ void
   operator()( int64_t i, double* acc ) const
   {
      const int ell = g.ell;
      Real ax = 0, ar = 0, au = 0;
      for( int k = 0; k < ell; k++ ) {
         ax += R[ k * ld + i ] * c2[ k ];
         ar += R[ ( k + 1 ) * ld + i ] * c1[ k ];
         au += U[ ( k + 1 ) * ld + i ] * c0[ k ];
      }
      x[ i ] = ax + x[ i ];
      const Real r0 = ar + R[ i ];
      R[ i ] = r0;
      U[ i ] = au + U[ i ];
      acc[ 0 ] += (double) r0 * (double) r0;
      acc[ 1 ] += (double) r_ast[ i ] * (double) r0;
   }
};

// Mixed precision, residual replacement (reliable updates: Sleijpen & van
// der Vorst, "Reliable updated residuals in hybrid Bi-CG methods", Computing
// 56, 1996): r_0 = M^-1 b with b the FP64 residual stored in FP32 (the FP32
// correction starts again from 0); acc (r_0, r_0), (r_ast, r_0). U_0 and the
// recurrence scalars are kept.
template< typename Real >
struct BlReplaceOp
{
   static constexpr int NR = 2;
   const Real* b;
   Real* r0;
   const Real *r_ast, *diag;
   __device__ __forceinline__ void load( const Ctl& ) {}
   __device__ __forceinline__ void
   operator()( int64_t i, double* acc ) const
   {
      Real rr = b[ i ];
      if( diag )
         rr = rr / diag[ i ];
      r0[ i ] = rr;
      acc[ 0 ] += (double) rr * (double) rr;
      acc[ 1 ] += (double) r_ast[ i ] * (double) rr;
   }
};

// the replaced r_0's norm and (r_ast, r_0); the outer test waits for the new
// phase's tolerance (bl_resume_kernel)
struct BlReplaceFin
{
   static constexpr bool active = true;
   __device__ void
   operator()( Ctl& c, const double* t ) const
   {
      c.bl_sigma0 = sqrt( t[ 0 ] );
      c.residue = c.bl_sigma0 / c.normb;
      c.bl_rho1 = t[ 1 ];
   }
};

// the outer loop's continuation after a replacement: test, rho_0, step 0
__global__ void
bl_resume_kernel( Ctl* ctl )
{
   Ctl& c = *ctl;
   if( c.done )
      return;
   bl_outer( c );
}

// sigma_0 = ||r_0||, residue (unless exact), outer test, next step's rho
struct BlFinalFin
{
   static constexpr bool active = true;
   int exact;
   __device__ void
   operator()( Ctl& c, const double* t ) const
   {
      c.bl_rho1 = t[ 1 ];
      if( exact )
         return;
      c.residue = sqrt( t[ 0 ] ) / c.normb;
      bl_outer( c );
   }
};

}  // namespace b2s
