// Batched solves in one persistent launch: many independent SPD systems,
// each with 1..8 right-hand sides, solved by TNL's CG recurrence
// (Solvers/Linear/CG.hpp:17-104) with the Jacobi preconditioner
// (Preconditioners/Diagonal.hpp:13-47), one thread-block cluster per system.
//
// The kernel is persistent: clusters take systems from a device work queue
// (largest first, so the long ones do not end up in the tail) until it is
// empty. A cluster of C CTAs (one per SM) splits a system's rows; its
// reductions go through distributed shared memory and every CTA sums the C
// partials in rank order, so all of them take the same decisions and the
// result does not depend on timing. Between the three phases of an iteration
// the cluster synchronizes with barrier.cluster (no global memory flags, no
// spin waits). With C SMs per system only 148/C systems are active at a
// time, which keeps their matrices and Krylov vectors resident in the 126 MB
// L2; C is chosen by the autotuner from timed samples of the batch.
//
// Right-hand sides of one system are interleaved (element (i, j) at
// i*k + j), so one pass over a matrix row serves all k of them.
//
// TNL solves one system per call (and one right-hand side per solve); this
// batched form has no counterpart there.
#include "b2s_internal.cuh"

#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <numeric>
#include <vector>

namespace cg = cooperative_groups;

namespace b2s {

constexpr int kBatchBlock = 1024;
constexpr int kBatchMaxRhs = 8;
constexpr int kBatchWarps = kBatchBlock / 32;

struct BatchArgs
{
   const int32_t* off;
   const int32_t* col;
   const double* val;
   const double* diag;     // Jacobi diagonal; nullptr: no preconditioner
   const int64_t* row_ptr;  // nsys + 1
   const int32_t* nrhs;     // nsys
   const int64_t* vec_off;  // nsys: first element of the system's interleaved vectors
   const int64_t* rhs_off;  // nsys: first right-hand side of the system (report slots)
   const int32_t* order;    // work queue: systems, largest first
   int32_t nsys;
   const double* B;
   double* X;
   double *R, *P, *AP;
   int64_t* it_out;
   double* res_out;
   int32_t* status_out;
   unsigned int* counter;
   double tol, div_tol;
   int64_t maxit, minit;
   int64_t* t_sys;  // optional (autotuner): global-timer ns at start and end of each system
};

__device__ __forceinline__ int64_t
global_ns()
{
   int64_t t;
   asm volatile( "mov.u64 %0, %%globaltimer;" : "=l"( t ) );
   return t;
}

// Per-CTA shared state of the system being solved.
template< int K >
struct SysState
{
   double part[ 2 ][ 2 * K ];  // this CTA's partial sums (double buffered)
   double red[ kBatchWarps ][ 2 * K ];
   double normb[ K ], s1[ K ], alpha[ K ], beta[ K ], residue[ K ];
   long long it[ K ];
   int done[ K ], reason[ K ];
};

// Sum of NR values over the CTA (fixed order); the CTA's total lands in
// part[0..NR). `red` holds kBatchWarps rows of `ld` doubles.
template< int NR >
__device__ __forceinline__ void
cta_partial( double ( &v )[ NR ], double* red, int ld, double* part )
{
   const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
   for( int k = 0; k < NR; k++ ) {
      double s = v[ k ];
#pragma unroll
      for( int o = 16; o > 0; o >>= 1 )
         s += __shfl_xor_sync( 0xffffffffu, s, o );
      if( lane == 0 )
         red[ warp * ld + k ] = s;
   }
   __syncthreads();
   if( threadIdx.x < NR ) {
      double s = 0;
      for( int w = 0; w < kBatchWarps; w++ )
         s += red[ w * ld + threadIdx.x ];
      part[ threadIdx.x ] = s;
   }
}

// Cluster-wide totals of NR values: every CTA sums the C partials in rank order.
template< int NR >
__device__ __forceinline__ void
cluster_total( cg::cluster_group& cl, double* part, double ( &tot )[ NR ] )
{
   cl.sync();
   const int C = (int) cl.num_blocks();
#pragma unroll
   for( int k = 0; k < NR; k++ )
      tot[ k ] = 0.0;
   for( int q = 0; q < C; q++ ) {
      const double* pq = cl.map_shared_rank( part, q );
#pragma unroll
      for( int k = 0; k < NR; k++ )
         tot[ k ] += pq[ k ];
   }
}

// IterativeSolver::checkNextIteration / nextIteration for one right-hand side
__device__ __forceinline__ void
next_iteration_rhs( double residue, long long& it, int& done, int& reason, const BatchArgs& a )
{
   const bool go = ! ( isnan( residue ) || it > a.maxit || ( residue > a.div_tol && it >= a.minit )
                       || ( residue < a.tol && it >= a.minit ) );
   it++;
   if( ! go ) {
      done = 1;
      reason = 1;
   }
}

// y(rows) = A p over the CTA's rows of the system, K columns at once;
// `fn( i_local, acc )` receives each row's K sums.
template< int K, class F >
__device__ __forceinline__ void
spmm_rows( const BatchArgs& a, int64_t row0, int64_t r_begin, int64_t r_end, const double* p, F&& fn )
{
   for( int64_t i = r_begin + threadIdx.x; i < r_end; i += kBatchBlock ) {
      const int64_t gr = row0 + i;
      const int b = __ldg( a.off + gr ), e = __ldg( a.off + gr + 1 );
      double acc[ K ];
#pragma unroll
      for( int j = 0; j < K; j++ )
         acc[ j ] = 0.0;
      // the row's columns and values four at a time, then their gathers, so a
      // stencil row costs two round trips instead of one per nonzero
      for( int t0 = b; t0 < e; t0 += 4 ) {
         int lc[ 4 ];
         double v[ 4 ];
#pragma unroll
         for( int u = 0; u < 4; u++ ) {
            lc[ u ] = t0 + u < e ? __ldg( a.col + t0 + u ) - (int) row0 : 0;
            v[ u ] = t0 + u < e ? __ldg( a.val + t0 + u ) : 0.0;
         }
#pragma unroll
         for( int u = 0; u < 4; u++ ) {
            if( t0 + u < e ) {
               const double* pc = p + (int64_t) lc[ u ] * K;
#pragma unroll
               for( int j = 0; j < K; j++ )
                  acc[ j ] += v[ u ] * __ldcg( pc + j );  // written by other CTAs: read through L2
            }
         }
      }
      fn( i, acc );
   }
}

template< int K >
__device__ void
solve_system( const BatchArgs& a, int sys, cg::cluster_group& cl, SysState< K >& st )
{
   const int C = (int) cl.num_blocks(), q = (int) cl.block_rank();
   const int64_t row0 = a.row_ptr[ sys ], n = a.row_ptr[ sys + 1 ] - row0;
   const int64_t r_begin = n * q / C, r_end = n * ( q + 1 ) / C;
   const int64_t vo = a.vec_off[ sys ];
   const double* B = a.B + vo;
   double* X = a.X + vo;
   double* R = a.R + vo;
   double* P = a.P + vo;
   double* AP = a.AP + vo;
   const double* dg = a.diag ? a.diag + row0 : nullptr;
   int buf = 0;

   // ||M^-1 b|| per right-hand side (CG.hpp:24-32)
   {
      double v[ K ];
#pragma unroll
      for( int j = 0; j < K; j++ )
         v[ j ] = 0.0;
      for( int64_t i = r_begin + threadIdx.x; i < r_end; i += kBatchBlock ) {
         const double d = dg ? dg[ i ] : 1.0;
#pragma unroll
         for( int j = 0; j < K; j++ ) {
            const double t = dg ? B[ i * K + j ] / d : B[ i * K + j ];
            v[ j ] += t * t;
         }
      }
      cta_partial< K >( v, &st.red[ 0 ][ 0 ], 2 * K, st.part[ buf ] );
      double tot[ K ];
      cluster_total< K >( cl, st.part[ buf ], tot );
      buf ^= 1;
      if( threadIdx.x == 0 )
         for( int j = 0; j < K; j++ ) {
            st.normb[ j ] = sqrt( tot[ j ] );
            if( st.normb[ j ] == 0.0 )
               st.normb[ j ] = 1.0;
         }
   }
   // r = b - A x ; z = M^-1 r ; p = z ; s1 = (r, z) (CG.hpp:37-58)
   {
      double v[ K ];
#pragma unroll
      for( int j = 0; j < K; j++ )
         v[ j ] = 0.0;
      spmm_rows< K >( a, row0, r_begin, r_end, X, [ & ]( int64_t i, const double( &acc )[ K ] ) {
         const double d = dg ? dg[ i ] : 1.0;
#pragma unroll
         for( int j = 0; j < K; j++ ) {
            const double r = B[ i * K + j ] - acc[ j ];
            const double z = dg ? r / d : r;
            R[ i * K + j ] = r;
            P[ i * K + j ] = z;
            v[ j ] += r * z;
         }
      } );
      cta_partial< K >( v, &st.red[ 0 ][ 0 ], 2 * K, st.part[ buf ] );
      double tot[ K ];
      cluster_total< K >( cl, st.part[ buf ], tot );
      buf ^= 1;
      if( threadIdx.x == 0 )
         for( int j = 0; j < K; j++ ) {
            st.s1[ j ] = tot[ j ];
            st.it[ j ] = 0;
            st.done[ j ] = 0;
            st.reason[ j ] = 0;
            st.residue[ j ] = sqrt( tot[ j ] ) / st.normb[ j ];
            next_iteration_rhs( st.residue[ j ], st.it[ j ], st.done[ j ], st.reason[ j ], a );
         }
      __syncthreads();
   }
   for( ;; ) {
      bool any = false;
#pragma unroll
      for( int j = 0; j < K; j++ )
         any |= ! st.done[ j ];
      if( ! any )
         break;
      // P of every row is complete before anyone gathers it
      cl.sync();
      // s2 = (A p, p)
      {
         double v[ K ];
#pragma unroll
         for( int j = 0; j < K; j++ )
            v[ j ] = 0.0;
         spmm_rows< K >( a, row0, r_begin, r_end, P, [ & ]( int64_t i, const double( &acc )[ K ] ) {
#pragma unroll
            for( int j = 0; j < K; j++ ) {
               AP[ i * K + j ] = acc[ j ];
               v[ j ] += acc[ j ] * P[ i * K + j ];
            }
         } );
         cta_partial< K >( v, &st.red[ 0 ][ 0 ], 2 * K, st.part[ buf ] );
         double tot[ K ];
         cluster_total< K >( cl, st.part[ buf ], tot );
         buf ^= 1;
         if( threadIdx.x == 0 )
            for( int j = 0; j < K; j++ ) {
               if( st.done[ j ] )
                  continue;
               if( tot[ j ] == 0.0 ) {
                  // p = 0 => r = 0: solved (CG.hpp:64-67)
                  st.residue[ j ] = 0.0;
                  st.done[ j ] = 1;
                  st.reason[ j ] = 2;
                  st.alpha[ j ] = 0.0;
               }
               else
                  st.alpha[ j ] = st.s1[ j ] / tot[ j ];
            }
         __syncthreads();
      }
      // x += alpha p ; r -= alpha Ap ; z = M^-1 r ; s1 = (r, z)
      {
         double al[ K ], v[ K ];
         bool act[ K ];
#pragma unroll
         for( int j = 0; j < K; j++ ) {
            al[ j ] = st.alpha[ j ];
            act[ j ] = ! st.done[ j ];
            v[ j ] = 0.0;
         }
         for( int64_t i = r_begin + threadIdx.x; i < r_end; i += kBatchBlock ) {
            const double d = dg ? dg[ i ] : 1.0;
#pragma unroll
            for( int j = 0; j < K; j++ ) {
               if( ! act[ j ] )
                  continue;
               const int64_t e = i * K + j;
               X[ e ] += al[ j ] * P[ e ];
               const double r = R[ e ] - al[ j ] * AP[ e ];
               R[ e ] = r;
               v[ j ] += dg ? r * ( r / d ) : r * r;
            }
         }
         cta_partial< K >( v, &st.red[ 0 ][ 0 ], 2 * K, st.part[ buf ] );
         double tot[ K ];
         cluster_total< K >( cl, st.part[ buf ], tot );
         buf ^= 1;
         if( threadIdx.x == 0 )
            for( int j = 0; j < K; j++ ) {
               if( st.done[ j ] )
                  continue;
               const double s2 = st.s1[ j ];
               st.s1[ j ] = tot[ j ];
               st.beta[ j ] = s2 == 0.0 ? 0.0 : tot[ j ] / s2;
               st.residue[ j ] = sqrt( tot[ j ] ) / st.normb[ j ];
               next_iteration_rhs( st.residue[ j ], st.it[ j ], st.done[ j ], st.reason[ j ], a );
            }
         __syncthreads();
      }
      // p = z + beta p
      {
         double be[ K ];
         bool act[ K ];
#pragma unroll
         for( int j = 0; j < K; j++ ) {
            be[ j ] = st.beta[ j ];
            act[ j ] = ! st.done[ j ];
         }
         for( int64_t i = r_begin + threadIdx.x; i < r_end; i += kBatchBlock ) {
            const double d = dg ? dg[ i ] : 1.0;
#pragma unroll
            for( int j = 0; j < K; j++ ) {
               if( ! act[ j ] )
                  continue;
               const int64_t e = i * K + j;
               const double z = dg ? R[ e ] / d : R[ e ];
               P[ e ] = z + be[ j ] * P[ e ];
            }
         }
      }
   }
   // report (rank 0)
   if( q == 0 && threadIdx.x < K ) {
      const int j = threadIdx.x;
      const int64_t slot = a.rhs_off[ sys ] + j;
      a.it_out[ slot ] = st.it[ j ];
      a.res_out[ slot ] = st.residue[ j ];
      const double r = st.residue[ j ];
      int s = B2S_OK;
      if( isnan( r ) )
         s = B2S_NAN;
      else if( r > a.div_tol && st.it[ j ] > a.minit )
         s = B2S_DIVERGED;
      else if( st.it[ j ] >= a.maxit || r > a.tol )
         s = st.reason[ j ] == 2 ? B2S_OK : B2S_NOT_CONVERGED;
      a.status_out[ slot ] = s;
   }
}

__global__ void __launch_bounds__( kBatchBlock, 1 )
batch_cg_kernel( BatchArgs a )
{
   cg::cluster_group cl = cg::this_cluster();
   __shared__ __align__( 16 ) unsigned char smem_raw[ sizeof( SysState< kBatchMaxRhs > ) ];
   __shared__ int next_sys;
   for( ;; ) {
      if( cl.block_rank() == 0 && threadIdx.x == 0 )
         next_sys = (int) atomicAdd( a.counter, 1u );
      cl.sync();
      const int idx = *cl.map_shared_rank( &next_sys, 0 );
      // every CTA has read rank 0's ticket before it can be overwritten
      cl.sync();
      if( idx >= a.nsys )
         break;
      const int sys = a.order[ idx ];
      const bool stamp = a.t_sys && cl.block_rank() == 0 && threadIdx.x == 0;
      if( stamp )
         a.t_sys[ 2 * sys ] = global_ns();
      switch( a.nrhs[ sys ] ) {
#define B2S_BATCH_K( KK )                                                                            \
   case KK:                                                                                          \
      solve_system< KK >( a, sys, cl, *reinterpret_cast< SysState< KK >* >( smem_raw ) );          \
      break;
         B2S_BATCH_K( 1 )
         B2S_BATCH_K( 2 )
         B2S_BATCH_K( 3 )
         B2S_BATCH_K( 4 )
         B2S_BATCH_K( 5 )
         B2S_BATCH_K( 6 )
         B2S_BATCH_K( 7 )
         B2S_BATCH_K( 8 )
#undef B2S_BATCH_K
         default:
            break;
      }
      // the shared state of this system is dead before the next one starts
      cl.sync();
      if( stamp )
         a.t_sys[ 2 * sys + 1 ] = global_ns();
   }
}

__global__ void
batch_diag_kernel( int64_t rows, const int32_t* __restrict__ off, const int32_t* __restrict__ col,
                   const double* __restrict__ val, double* diag )
{
   for( int64_t r = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; r < rows; r += (int64_t) gridDim.x * blockDim.x ) {
      double d = 0.0;
      for( int t = off[ r ]; t < off[ r + 1 ]; t++ )
         if( col[ t ] == r ) {
            d = val[ t ];
            break;
         }
      diag[ r ] = d;  // Diagonal::update takes A_ii (Diagonal.hpp:24-36); solve divides by it
   }
}

}  // namespace b2s

using namespace b2s;

struct b2s_batch_t
{
   int32_t nsys = 0;
   int64_t rows = 0, nnz = 0, nvec = 0, nslots = 0;
   std::vector< int64_t > row_ptr_h, vec_off_h, rhs_off_h;
   std::vector< int32_t > nrhs_h;
   DevBuf off, col, val, diag, row_ptr, nrhs, vec_off, rhs_off, order;
   DevBuf R, P, AP, counter, it_out, res_out, status_out;
   b2s_batch_opts o{};
   int cluster = 0;  // chosen cluster size
};

namespace b2s {

static b2s_status
launch_batch( b2s_batch_t* bt, const double* B, double* X, int cluster, int nsys_limit, int64_t maxit,
              cudaStream_t s, const int32_t* order = nullptr, int64_t* t_sys = nullptr, int* clusters_out = nullptr )
{
   BatchArgs a{};
   a.off = bt->off.as< int32_t >();
   a.col = bt->col.as< int32_t >();
   a.val = bt->val.as< double >();
   a.diag = bt->o.preconditioner ? bt->diag.as< double >() : nullptr;
   a.row_ptr = bt->row_ptr.as< int64_t >();
   a.nrhs = bt->nrhs.as< int32_t >();
   a.vec_off = bt->vec_off.as< int64_t >();
   a.rhs_off = bt->rhs_off.as< int64_t >();
   a.order = order ? order : bt->order.as< int32_t >();
   a.nsys = nsys_limit;
   a.B = B;
   a.X = X;
   a.R = bt->R.as< double >();
   a.P = bt->P.as< double >();
   a.AP = bt->AP.as< double >();
   a.it_out = bt->it_out.as< int64_t >();
   a.res_out = bt->res_out.as< double >();
   a.status_out = bt->status_out.as< int32_t >();
   a.counter = bt->counter.as< unsigned int >();
   a.tol = bt->o.convergence_residue;
   a.div_tol = bt->o.divergence_residue;
   a.maxit = maxit;
   a.minit = bt->o.min_iterations;
   a.t_sys = t_sys;
   B2S_TRY_CUDA( cudaMemsetAsync( bt->counter.p, 0, sizeof( unsigned int ), s ) );
   cudaLaunchConfig_t cfg{};
   cudaLaunchAttribute attr[ 1 ];
   attr[ 0 ].id = cudaLaunchAttributeClusterDimension;
   attr[ 0 ].val.clusterDim.x = cluster;
   attr[ 0 ].val.clusterDim.y = 1;
   attr[ 0 ].val.clusterDim.z = 1;
   cfg.blockDim = dim3( kBatchBlock );
   cfg.dynamicSmemBytes = 0;
   cfg.stream = s;
   cfg.attrs = attr;
   cfg.numAttrs = 1;
   cfg.gridDim = dim3( cluster );
   int nclusters = 0;
   B2S_TRY_CUDA( cudaOccupancyMaxActiveClusters( &nclusters, batch_cg_kernel, &cfg ) );
   if( nclusters < 1 ) {
      set_error( "batched solver: a cluster of %d CTAs does not fit on the device", cluster );
      return B2S_UNSUPPORTED;
   }
   if( clusters_out )
      *clusters_out = nclusters;
   nclusters = std::min( nclusters, std::max( 1, nsys_limit ) );
   cfg.gridDim = dim3( nclusters * cluster );
   B2S_TRY_CUDA( cudaLaunchKernelEx( &cfg, batch_cg_kernel, a ) );
   return B2S_OK;
}

// Autotuner of the cluster size. A sample of systems (even strides through
// the size-sorted queue) is solved to convergence under every candidate C
// while the kernel stamps each system's start and end. For C the full batch
// is predicted as
//     max( sum over the batch of (duration x C) / (resident clusters x C),
//          longest single system )
// — the SM time the systems need spread over the device, or the tail of the
// slowest one, whichever is longer — scaling the sample's SM time by
// nsys / sample. The C with the smallest prediction wins.
static b2s_status
autotune_cluster( b2s_batch_t* bt, const double* B, double* X, cudaStream_t s, int& best )
{
   best = 1;
   const int cands[] = { 1, 2, 4, 8 };
   const int sms = num_sms();
   const int sample = std::min( bt->nsys, 2 * sms );
   std::vector< int32_t > order_h( bt->nsys );
   B2S_TRY( copy_d2h( order_h.data(), bt->order.p, bt->nsys * sizeof( int32_t ), s ) );
   std::vector< int32_t > pick( sample );
   for( int k = 0; k < sample; k++ )
      pick[ k ] = order_h[ (int64_t) k * bt->nsys / sample ];
   DevBuf sample_order, stamps;
   B2S_TRY( sample_order.alloc( sample * sizeof( int32_t ) ) );
   B2S_TRY( copy_h2d( sample_order.p, pick.data(), sample * sizeof( int32_t ), s ) );
   B2S_TRY( stamps.alloc( (size_t) 2 * bt->nsys * sizeof( int64_t ) ) );
   std::vector< int64_t > t( 2 * bt->nsys );
   double best_est = 1e300;
   for( int c : cands ) {
      int nclusters = 0;
      b2s_status st = launch_batch( bt, B, X, c, sample, bt->o.max_iterations, s, sample_order.as< int32_t >(),
                                    stamps.as< int64_t >(), &nclusters );
      if( st != B2S_OK ) {
         cudaGetLastError();
         clear_error();
         continue;
      }
      B2S_TRY( copy_d2h( t.data(), stamps.p, t.size() * sizeof( int64_t ), s ) );
      double sm_ns = 0, longest = 0;
      for( int k = 0; k < sample; k++ ) {
         const int sys = pick[ k ];
         const double d = (double) ( t[ 2 * sys + 1 ] - t[ 2 * sys ] );
         sm_ns += d * c;
         longest = std::max( longest, d );
      }
      const double total_sm_ns = sm_ns * ( (double) bt->nsys / sample );
      const double est = std::max( total_sm_ns / ( (double) std::max( nclusters, 1 ) * c ), longest );
      if( est < best_est ) {
         best_est = est;
         best = c;
      }
   }
   return B2S_OK;
}

}  // namespace b2s

extern "C" {

void
b2s_batch_opts_default( b2s_batch_opts* o )
{
   if( ! o )
      return;
   std::memset( o, 0, sizeof( *o ) );
   o->preconditioner = B2S_PRECOND_JACOBI;
   o->convergence_residue = 1e-8;
   o->divergence_residue = 1e300;
   o->max_iterations = 1000000;
   o->min_iterations = 0;
   o->cluster_size = 0;
}

b2s_status
b2s_batch_create( int32_t nsys, const int64_t* row_ptr, const int32_t* nrhs, const int32_t* offsets,
                  const int32_t* columns, const double* values, b2s_memory where, const b2s_batch_opts* opts,
                  b2s_stream stream, b2s_batch* out )
{
   clear_error();
   B2S_CHECK_ARG( out && row_ptr && nrhs && offsets && nsys >= 0, "NULL argument" );
   *out = nullptr;
   B2S_CHECK_ARG( where == B2S_HOST || where == B2S_DEVICE, "where" );
   cudaStream_t s = as_stream( stream );
   std::unique_ptr< b2s_batch_t > bt( new b2s_batch_t() );
   b2s_batch_opts_default( &bt->o );
   if( opts )
      bt->o = *opts;
   B2S_CHECK_ARG( bt->o.preconditioner == B2S_PRECOND_NONE || bt->o.preconditioner == B2S_PRECOND_JACOBI,
                  "batched solves take no preconditioner or Jacobi" );
   B2S_CHECK_ARG( bt->o.cluster_size == 0 || bt->o.cluster_size == 1 || bt->o.cluster_size == 2
                     || bt->o.cluster_size == 4 || bt->o.cluster_size == 8,
                  "cluster_size in {0 (autotune), 1, 2, 4, 8}" );
   bt->nsys = nsys;
   bt->row_ptr_h.assign( row_ptr, row_ptr + nsys + 1 );
   bt->nrhs_h.assign( nrhs, nrhs + nsys );
   B2S_CHECK_ARG( bt->row_ptr_h[ 0 ] == 0, "row_ptr[0] must be 0" );
   for( int i = 0; i < nsys; i++ ) {
      B2S_CHECK_ARG( bt->row_ptr_h[ i + 1 ] >= bt->row_ptr_h[ i ], "row_ptr must be non-decreasing" );
      B2S_CHECK_ARG( bt->nrhs_h[ i ] >= 1 && bt->nrhs_h[ i ] <= kBatchMaxRhs, "right-hand sides per system in [1, 8]" );
   }
   bt->rows = bt->row_ptr_h[ nsys ];
   B2S_CHECK_ARG( bt->rows < INT32_MAX, "total rows must fit in int32" );
   int32_t nnz32 = 0;
   if( where == B2S_HOST )
      nnz32 = offsets[ bt->rows ];
   else
      B2S_TRY( copy_d2h( &nnz32, offsets + bt->rows, sizeof( int32_t ), s ) );
   bt->nnz = nnz32;
   B2S_CHECK_ARG( bt->nnz >= 0 && ( bt->nnz == 0 || ( columns && values ) ), "columns / values" );
   bt->vec_off_h.resize( nsys );
   bt->rhs_off_h.resize( nsys );
   int64_t v = 0, k = 0;
   for( int i = 0; i < nsys; i++ ) {
      bt->vec_off_h[ i ] = v;
      bt->rhs_off_h[ i ] = k;
      v += ( bt->row_ptr_h[ i + 1 ] - bt->row_ptr_h[ i ] ) * bt->nrhs_h[ i ];
      k += bt->nrhs_h[ i ];
   }
   bt->nvec = v;
   bt->nslots = k;
   // work queue: largest systems first (rows x right-hand sides)
   std::vector< int32_t > order( nsys );
   std::iota( order.begin(), order.end(), 0 );
   std::stable_sort( order.begin(), order.end(), [ & ]( int a, int b ) {
      const int64_t wa = ( bt->row_ptr_h[ a + 1 ] - bt->row_ptr_h[ a ] ) * ( 4 + bt->nrhs_h[ a ] );
      const int64_t wb = ( bt->row_ptr_h[ b + 1 ] - bt->row_ptr_h[ b ] ) * ( 4 + bt->nrhs_h[ b ] );
      return wa > wb;
   } );
   const cudaMemcpyKind kin = where == B2S_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
   B2S_TRY( bt->off.alloc( ( bt->rows + 1 ) * sizeof( int32_t ) ) );
   B2S_TRY( bt->col.alloc( std::max< int64_t >( bt->nnz, 1 ) * sizeof( int32_t ) ) );
   B2S_TRY( bt->val.alloc( std::max< int64_t >( bt->nnz, 1 ) * sizeof( double ) ) );
   B2S_TRY_CUDA( cudaMemcpyAsync( bt->off.p, offsets, ( bt->rows + 1 ) * sizeof( int32_t ), kin, s ) );
   if( bt->nnz > 0 ) {
      B2S_TRY_CUDA( cudaMemcpyAsync( bt->col.p, columns, bt->nnz * sizeof( int32_t ), kin, s ) );
      B2S_TRY_CUDA( cudaMemcpyAsync( bt->val.p, values, bt->nnz * sizeof( double ), kin, s ) );
   }
   B2S_TRY( bt->diag.alloc( std::max< int64_t >( bt->rows, 1 ) * sizeof( double ) ) );
   if( bt->rows > 0 ) {
      batch_diag_kernel<<< (int) std::min< int64_t >( ( bt->rows + 255 ) / 256, (int64_t) num_sms() * 16 ), 256, 0,
                              s >>>( bt->rows, bt->off.as< int32_t >(), bt->col.as< int32_t >(), bt->val.as< double >(),
                                     bt->diag.as< double >() );
      B2S_TRY_CUDA( cudaGetLastError() );
   }
   B2S_TRY( bt->row_ptr.alloc( ( nsys + 1 ) * sizeof( int64_t ) ) );
   B2S_TRY( bt->nrhs.alloc( std::max( nsys, 1 ) * sizeof( int32_t ) ) );
   B2S_TRY( bt->vec_off.alloc( std::max( nsys, 1 ) * sizeof( int64_t ) ) );
   B2S_TRY( bt->rhs_off.alloc( std::max( nsys, 1 ) * sizeof( int64_t ) ) );
   B2S_TRY( bt->order.alloc( std::max( nsys, 1 ) * sizeof( int32_t ) ) );
   B2S_TRY( copy_h2d( bt->row_ptr.p, bt->row_ptr_h.data(), ( nsys + 1 ) * sizeof( int64_t ), s ) );
   if( nsys > 0 ) {
      B2S_TRY( copy_h2d( bt->nrhs.p, bt->nrhs_h.data(), nsys * sizeof( int32_t ), s ) );
      B2S_TRY( copy_h2d( bt->vec_off.p, bt->vec_off_h.data(), nsys * sizeof( int64_t ), s ) );
      B2S_TRY( copy_h2d( bt->rhs_off.p, bt->rhs_off_h.data(), nsys * sizeof( int64_t ), s ) );
      B2S_TRY( copy_h2d( bt->order.p, order.data(), nsys * sizeof( int32_t ), s ) );
   }
   const size_t vb = (size_t) std::max< int64_t >( bt->nvec, 1 ) * sizeof( double );
   B2S_TRY( bt->R.alloc( vb ) );
   B2S_TRY( bt->P.alloc( vb ) );
   B2S_TRY( bt->AP.alloc( vb ) );
   B2S_TRY( bt->counter.alloc( 64 ) );
   B2S_TRY( bt->it_out.alloc( std::max< int64_t >( bt->nslots, 1 ) * sizeof( int64_t ) ) );
   B2S_TRY( bt->res_out.alloc( std::max< int64_t >( bt->nslots, 1 ) * sizeof( double ) ) );
   B2S_TRY( bt->status_out.alloc( std::max< int64_t >( bt->nslots, 1 ) * sizeof( int32_t ) ) );
   B2S_TRY_CUDA( cudaStreamSynchronize( s ) );
   bt->cluster = bt->o.cluster_size;
   *out = bt.release();
   return B2S_OK;
}

b2s_status
b2s_batch_destroy( b2s_batch b )
{
   clear_error();
   delete b;
   return B2S_OK;
}

b2s_status
b2s_batch_solve( b2s_batch bt, const double* B, double* X, b2s_stream stream, b2s_batch_report* report )
{
   clear_error();
   B2S_CHECK_ARG( bt && ( bt->nvec == 0 || ( B && X ) ), "NULL argument" );
   cudaStream_t s = as_stream( stream );
   b2s_batch_report rep{};
   if( bt->nsys == 0 ) {
      if( report )
         *report = rep;
      return B2S_OK;
   }
   if( bt->cluster == 0 ) {
      // autotune on a copy of the initial guess so X is untouched
      DevBuf xs;
      B2S_TRY( xs.alloc( bt->nvec * sizeof( double ) ) );
      B2S_TRY_CUDA( cudaMemcpyAsync( xs.p, X, bt->nvec * sizeof( double ), cudaMemcpyDeviceToDevice, s ) );
      int best = 1;
      B2S_TRY( autotune_cluster( bt, B, xs.as< double >(), s, best ) );
      B2S_TRY_CUDA( cudaStreamSynchronize( s ) );
      bt->cluster = best;
   }
   cudaEvent_t e0, e1;
   B2S_TRY_CUDA( cudaEventCreate( &e0 ) );
   B2S_TRY_CUDA( cudaEventCreate( &e1 ) );
   cudaEventRecord( e0, s );
   b2s_status st = launch_batch( bt, B, X, bt->cluster, bt->nsys, bt->o.max_iterations, s );
   cudaEventRecord( e1, s );
   if( st == B2S_OK ) {
      cudaError_t e = cudaEventSynchronize( e1 );
      if( e != cudaSuccess ) {
         set_error( "batched solve: %s", cudaGetErrorString( e ) );
         st = B2S_CUDA_ERROR;
      }
   }
   float ms = 0;
   if( st == B2S_OK )
      cudaEventElapsedTime( &ms, e0, e1 );
   cudaEventDestroy( e0 );
   cudaEventDestroy( e1 );
   if( st != B2S_OK )
      return st;
   std::vector< int64_t > its( bt->nslots );
   std::vector< double > res( bt->nslots );
   std::vector< int32_t > sts( bt->nslots );
   B2S_TRY( copy_d2h( its.data(), bt->it_out.p, bt->nslots * sizeof( int64_t ), s ) );
   B2S_TRY( copy_d2h( res.data(), bt->res_out.p, bt->nslots * sizeof( double ), s ) );
   B2S_TRY( copy_d2h( sts.data(), bt->status_out.p, bt->nslots * sizeof( int32_t ), s ) );
   rep.device_ms = ms;
   rep.cluster_size = bt->cluster;
   rep.solves = bt->nslots;
   for( int64_t i = 0; i < bt->nslots; i++ ) {
      rep.total_iterations += its[ i ];
      rep.max_iterations = std::max< int64_t >( rep.max_iterations, its[ i ] );
      rep.max_residue = std::max( rep.max_residue, res[ i ] );
      if( sts[ i ] == B2S_OK )
         rep.converged++;
   }
   if( report )
      *report = rep;
   return rep.converged == bt->nslots ? B2S_OK : B2S_NOT_CONVERGED;
}

b2s_status
b2s_batch_results( b2s_batch bt, int64_t* iterations, double* residues, int32_t* statuses )
{
   clear_error();
   B2S_CHECK_ARG( bt, "NULL batch" );
   if( iterations )
      B2S_TRY( copy_d2h( iterations, bt->it_out.p, bt->nslots * sizeof( int64_t ), nullptr ) );
   if( residues )
      B2S_TRY( copy_d2h( residues, bt->res_out.p, bt->nslots * sizeof( double ), nullptr ) );
   if( statuses )
      B2S_TRY( copy_d2h( statuses, bt->status_out.p, bt->nslots * sizeof( int32_t ), nullptr ) );
   return B2S_OK;
}

}  // extern "C"
