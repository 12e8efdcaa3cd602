// ILU(0) factorization set-up and the stand-alone preconditioner handle
// (Preconditioners::Diagonal / ILU0 update + solve, Solvers/Linear/Preconditioners/).
#include "ilu.cuh"

#include <algorithm>
#include <memory>
#include <vector>

namespace b2s {

// diag[i] = position of A_ii; *unsorted = the first row whose columns are not
// strictly increasing, *missing = the first row without a stored diagonal
__global__ void
ilu_prepare_kernel( int32_t n, const int32_t* __restrict__ off, const int32_t* __restrict__ col,
                    int32_t* __restrict__ diag, int* unsorted, int* missing )
{
   for( int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x ) {
      const int b = off[ i ], e = off[ i + 1 ];
      int d = -1;
      for( int k = b; k < e; k++ ) {
         if( k > b && col[ k ] <= col[ k - 1 ] )
            atomicMin( unsorted, (int) i );
         if( col[ k ] == (int) i )
            d = k;
      }
      diag[ i ] = d;
      if( d < 0 )
         atomicMin( missing, (int) i );
   }
}

template< typename Tin, typename Tout >
__global__ void
ilu_cast_kernel( const Tin* __restrict__ in, Tout* __restrict__ out, int64_t n )
{
   for( int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x )
      out[ i ] = (Tout) in[ i ];
}

static int
grid_n( int64_t n )
{
   return (int) std::max< int64_t >( 1, std::min< int64_t >( ( n + 255 ) / 256, (int64_t) num_sms() * 32 ) );
}

template< typename Real >
b2s_status
ilu_levels( IluFactors< Real >& F, const std::vector< int32_t >& hoff, const std::vector< int32_t >& hcol,
            const std::vector< int32_t >& hdiag, cudaStream_t s )
{
   const int32_t n = F.n;
   std::vector< int32_t > lev( (size_t) std::max( n, 1 ) ), ord;
   auto order = [ & ]( int depth, DevBuf& out, int32_t& len ) -> b2s_status
   {
      // counting sort of the rows by level, rows in increasing order within a
      // level, every level padded (-1) to a multiple of the rows per ticket
      std::vector< int64_t > count( (size_t) depth, 0 ), start( (size_t) depth + 1, 0 );
      for( int32_t i = 0; i < n; i++ )
         count[ lev[ i ] ]++;
      for( int l = 0; l < depth; l++ )
         start[ l + 1 ] = start[ l ] + ( count[ l ] + kIluRows - 1 ) / kIluRows * kIluRows;
      if( start[ depth ] > INT32_MAX - 32 ) {
         set_error( "ILU: too many rows" );
         return B2S_INDEX_OVERFLOW;
      }
      len = (int32_t) start[ depth ];
      ord.assign( (size_t) len + 32, -1 );
      for( int32_t i = 0; i < n; i++ )
         ord[ start[ lev[ i ] ]++ ] = i;
      B2S_TRY( out.alloc( ord.size() * sizeof( int32_t ) ) );
      return copy_h2d( out.p, ord.data(), ord.size() * sizeof( int32_t ), s );
   };
   int depth = 0;
   for( int32_t i = 0; i < n; i++ ) {
      int l = 0;
      for( int32_t k = hoff[ i ]; k < hdiag[ i ]; k++ )
         l = std::max( l, lev[ hcol[ k ] ] + 1 );
      lev[ i ] = l;
      depth = std::max( depth, l + 1 );
   }
   F.levels_l = depth;
   B2S_TRY( order( depth, F.ord_l, F.n_ord_l ) );
   depth = 0;
   for( int32_t i = n - 1; i >= 0; i-- ) {
      int l = 0;
      for( int32_t k = hdiag[ i ] + 1; k < hoff[ i + 1 ]; k++ )
         l = std::max( l, lev[ hcol[ k ] ] + 1 );
      lev[ i ] = l;
      depth = std::max( depth, l + 1 );
   }
   F.levels_u = depth;
   B2S_TRY( order( depth, F.ord_u, F.n_ord_u ) );
   // resident warps only: every SM full of 256-thread blocks
   F.grid = num_sms() * ( 2048 / kIluBlock );
   return B2S_OK;
}

template b2s_status ilu_levels< double >( IluFactors< double >&, const std::vector< int32_t >&,
                                          const std::vector< int32_t >&, const std::vector< int32_t >&, cudaStream_t );
template b2s_status ilu_levels< float >( IluFactors< float >&, const std::vector< int32_t >&,
                                         const std::vector< int32_t >&, const std::vector< int32_t >&, cudaStream_t );

template< typename Real >
b2s_status
ilu_factorize( const b2s_matrix_t* A, const Real* values, IluFactors< Real >& F, cudaStream_t s )
{
   if( A->rows != A->cols ) {
      set_error( "ILU(0) needs a square matrix" );
      return B2S_INVALID_ARG;
   }
   F.n = A->rows;
   int64_t nnz = A->nnz;
   const Real* vals = values;
   DevBuf own_vals;
   if( A->format == B2S_CSR ) {
      F.off = A->offsets.as< int32_t >();
      F.col = A->columns.as< int32_t >();
   }
   else {
      // the rows of a padded layout in storage order (TNL's row views), zeros kept
      DevBuf v;
      B2S_TRY( layout_to_csr( A, false, F.off_own, F.col_own, v, nnz, s ) );
      F.off = F.off_own.template as< int32_t >();
      F.col = F.col_own.template as< int32_t >();
      if( ( A->dtype == B2S_F64 ) == std::is_same< Real, double >::value )
         own_vals = std::move( v );
      else {
         B2S_TRY( own_vals.alloc( (size_t) std::max< int64_t >( nnz, 1 ) * sizeof( Real ) ) );
         if( nnz > 0 ) {
            if( A->dtype == B2S_F64 )
               ilu_cast_kernel< double, Real ><<< grid_n( nnz ), 256, 0, s >>>( v.as< double >(), own_vals.as< Real >(), nnz );
            else
               ilu_cast_kernel< float, Real ><<< grid_n( nnz ), 256, 0, s >>>( v.as< float >(), own_vals.as< Real >(), nnz );
            B2S_TRY_CUDA( cudaGetLastError() );
         }
      }
      vals = own_vals.as< Real >();
   }
   const int32_t n = F.n;
   B2S_TRY( F.lu.alloc( (size_t) std::max< int64_t >( nnz, 1 ) * sizeof( Real ) ) );
   B2S_TRY( F.diag.alloc( (size_t) std::max( n, 1 ) * sizeof( int32_t ) ) );
   B2S_TRY( F.flags.alloc( (size_t) std::max( n, 1 ) * sizeof( int32_t ) ) );
   B2S_TRY( F.state.alloc( sizeof( IluState ) ) );
   B2S_TRY_CUDA( cudaMemsetAsync( F.flags.p, 0, (size_t) std::max( n, 1 ) * sizeof( int32_t ), s ) );
   B2S_TRY_CUDA( cudaMemsetAsync( F.state.p, 0, sizeof( IluState ), s ) );
   if( nnz > 0 )
      B2S_TRY_CUDA( cudaMemcpyAsync( F.lu.p, vals, (size_t) nnz * sizeof( Real ), cudaMemcpyDeviceToDevice, s ) );
   if( n == 0 )
      return B2S_OK;
   DevBuf bad;
   B2S_TRY( bad.alloc( 2 * sizeof( int ) ) );
   const int init[ 2 ] = { INT32_MAX, INT32_MAX };
   B2S_TRY( copy_h2d( bad.p, init, sizeof( init ), s ) );
   ilu_prepare_kernel<<< grid_n( n ), 256, 0, s >>>( n, F.off, F.col, F.diag.template as< int32_t >(), bad.as< int >(),
                                                     bad.as< int >() + 1 );
   B2S_TRY_CUDA( cudaGetLastError() );
   int h[ 2 ];
   B2S_TRY( copy_d2h( h, bad.p, sizeof( h ), s ) );
   if( h[ 0 ] != INT32_MAX ) {
      set_error( "ILU(0) needs the columns of every row sorted (row %d is not)", h[ 0 ] );
      return B2S_INVALID_ARG;
   }
   if( h[ 1 ] != INT32_MAX ) {
      set_error( "A(%d, %d) is missing.", h[ 1 ], h[ 1 ] );
      return B2S_INVALID_ARG;
   }
   // levels of the dependency DAGs of L (rows below) and U (rows above), on
   // the host in one pass each; rows are then handed out level by level
   {
      std::vector< int32_t > hoff( (size_t) n + 1 ), hcol( (size_t) std::max< int64_t >( nnz, 1 ) ), hdiag( (size_t) n );
      B2S_TRY( copy_d2h( hoff.data(), F.off, hoff.size() * sizeof( int32_t ), s ) );
      if( nnz > 0 )
         B2S_TRY( copy_d2h( hcol.data(), F.col, (size_t) nnz * sizeof( int32_t ), s ) );
      B2S_TRY( copy_d2h( hdiag.data(), F.diag.template as< int32_t >(), hdiag.size() * sizeof( int32_t ), s ) );
      B2S_TRY( ilu_levels( F, hoff, hcol, hdiag, s ) );
   }
   const IluView< Real > v = F.view();
   ilu_begin_kernel< NoGate ><<< 1, 1, 0, s >>>( v.st, NoGate{} );
   ilu_factor_kernel< Real ><<< F.grid, kIluBlock, 0, s >>>( v );
   B2S_TRY_CUDA( cudaGetLastError() );
   B2S_TRY_CUDA( cudaStreamSynchronize( s ) );
   return F.check( s );
}

template b2s_status ilu_factorize< double >( const b2s_matrix_t*, const double*, IluFactors< double >&, cudaStream_t );
template b2s_status ilu_factorize< float >( const b2s_matrix_t*, const float*, IluFactors< float >&, cudaStream_t );

// x = b / diag (Preconditioners::Diagonal::solve, Diagonal.hpp:38-47)
template< typename Real >
__global__ void
jacobi_apply_kernel( int64_t n, const Real* __restrict__ diag, const Real* b, Real* x )
{
   for( int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x )
      x[ i ] = b[ i ] / diag[ i ];
}

}  // namespace b2s

using namespace b2s;

struct b2s_precond_t
{
   int32_t kind = 0;
   int32_t dtype = 0;
   int32_t n = 0;
   const b2s_matrix_t* A = nullptr;
   IluFactors< double > f64;
   IluFactors< float > f32;
   DevBuf stage_b, stage_x;
   b2s_matrix_t* expanded = nullptr;  // L + L^T - D of a SymmetricMatrix (the factors refer to it)
   ~b2s_precond_t() { delete expanded; }
};

extern "C" {

static b2s_status
precond_create( b2s_matrix A, int32_t kind, int32_t ilut_p, double ilut_tau, b2s_stream stream, b2s_precond* out )
{
   clear_error();
   B2S_NO_BINARY( A, "a preconditioner" );
   B2S_CHECK_ARG( A && out, "NULL argument" );
   *out = nullptr;
   B2S_CHECK_ARG( kind == B2S_PRECOND_JACOBI || kind == B2S_PRECOND_ILU0 || kind == B2S_PRECOND_ILUT,
                  "preconditioner kind" );
   B2S_CHECK_ARG( A->rows == A->cols, "the matrix must be square" );
   cudaStream_t s = as_stream( stream );
   std::unique_ptr< b2s_precond_t > M( new b2s_precond_t() );
   M->kind = kind;
   M->dtype = A->dtype;
   M->n = A->rows;
   M->A = A;
   if( kind == B2S_PRECOND_ILU0 || kind == B2S_PRECOND_ILUT ) {
      if( A->symmetric ) {
         B2S_TRY( expand_symmetric( A, s, &M->expanded ) );
         A = M->expanded;
      }
      if( kind == B2S_PRECOND_ILUT ) {
         if( A->dtype == B2S_F64 )
            B2S_TRY( ilut_factorize< double >( A, ilut_p, ilut_tau, M->f64, s ) );
         else
            B2S_TRY( ilut_factorize< float >( A, ilut_p, ilut_tau, M->f32, s ) );
      }
      else if( A->dtype == B2S_F64 )
         B2S_TRY( ilu_factorize< double >( A, A->values.as< double >(), M->f64, s ) );
      else
         B2S_TRY( ilu_factorize< float >( A, A->values.as< float >(), M->f32, s ) );
   }
   *out = M.release();
   return B2S_OK;
}

b2s_status
b2s_precond_create( b2s_matrix A, int32_t kind, b2s_stream stream, b2s_precond* out )
{
   // ILUT with TNL's defaults (ILUT.h:79-82)
   return precond_create( A, kind, 0, 1e-4, stream, out );
}

b2s_status
b2s_precond_create_ilut( b2s_matrix A, int32_t p, double threshold, b2s_stream stream, b2s_precond* out )
{
   return precond_create( A, B2S_PRECOND_ILUT, p, threshold, stream, out );
}

b2s_status
b2s_precond_solve( b2s_precond M, const void* b, void* x, b2s_memory where, b2s_stream stream )
{
   clear_error();
   B2S_CHECK_ARG( M, "NULL preconditioner" );
   B2S_CHECK_ARG( where == B2S_HOST || where == B2S_DEVICE, "where" );
   B2S_CHECK_ARG( M->n == 0 || ( b && x ), "NULL vector" );
   if( M->n == 0 )
      return B2S_OK;
   cudaStream_t s = as_stream( stream );
   const size_t es = M->dtype == B2S_F64 ? 8 : 4, bytes = (size_t) M->n * es;
   const void* db = b;
   void* dx = x;
   if( where == B2S_HOST ) {
      if( M->stage_b.bytes < bytes )
         B2S_TRY( M->stage_b.alloc( bytes ) );
      if( M->stage_x.bytes < bytes )
         B2S_TRY( M->stage_x.alloc( bytes ) );
      B2S_TRY_CUDA( cudaMemcpyAsync( M->stage_b.p, b, bytes, cudaMemcpyHostToDevice, s ) );
      db = M->stage_b.p;
      dx = M->stage_x.p;
   }
   if( M->kind == B2S_PRECOND_JACOBI ) {
      if( M->dtype == B2S_F64 )
         jacobi_apply_kernel< double ><<< grid_n( M->n ), 256, 0, s >>>( M->n, M->A->diagonal.as< double >(),
                                                                       (const double*) db, (double*) dx );
      else
         jacobi_apply_kernel< float ><<< grid_n( M->n ), 256, 0, s >>>( M->n, M->A->diagonal.as< float >(),
                                                                      (const float*) db, (float*) dx );
      B2S_TRY_CUDA( cudaGetLastError() );
   }
   else if( M->dtype == B2S_F64 )
      B2S_TRY( M->f64.apply( (const double*) db, (double*) dx, s ) );
   else
      B2S_TRY( M->f32.apply( (const float*) db, (float*) dx, s ) );
   if( where == B2S_HOST )
      B2S_TRY_CUDA( cudaMemcpyAsync( x, dx, bytes, cudaMemcpyDeviceToHost, s ) );
   B2S_TRY_CUDA( cudaStreamSynchronize( s ) );
   if( M->kind == B2S_PRECOND_ILU0 || M->kind == B2S_PRECOND_ILUT )
      return M->dtype == B2S_F64 ? M->f64.check( s ) : M->f32.check( s );
   return B2S_OK;
}

b2s_status
b2s_precond_destroy( b2s_precond M )
{
   clear_error();
   delete M;
   return B2S_OK;
}

}  // extern "C"
