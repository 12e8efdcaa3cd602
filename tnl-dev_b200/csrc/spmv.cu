// Public SpMV entry point: SparseMatrix::vectorProduct (Matrices/SparseMatrix.h:1078-1085,
// SparseMatrixView.hpp:390-490).
#include "spmv_kernels.cuh"

namespace b2s {

template< typename Real >
b2s_status
spmv_plain( const SpmvArgs< Real >& a, Real* y, Real alpha, Real beta, cudaStream_t s )
{
   YSink< Real > sink{ y, alpha, beta, keeper_mode( alpha, beta ) };
   return spmv_dispatch< Real, YSink< Real > >( a.A, a.values, a.x, a.row_begin, a.row_end, sink, RedScratch{}, s );
}

template b2s_status spmv_plain< double >( const SpmvArgs< double >&, double*, double, double, cudaStream_t );
template b2s_status spmv_plain< float >( const SpmvArgs< float >&, float*, float, float, cudaStream_t );

b2s_status
device_status( b2s_matrix_t* A, cudaStream_t s )
{
   int flag = 0;
   B2S_TRY( copy_d2h( &flag, A->status.p, sizeof( int ), s ) );
   if( flag ) {
      B2S_TRY_CUDA( cudaMemsetAsync( A->status.p, 0, sizeof( int ), s ) );
      set_error( "a bounded wait inside an SpMV kernel gave up (bulk copy did not complete)" );
      return B2S_TIMEOUT;
   }
   return B2S_OK;
}

template< typename Real >
static b2s_status
spmv_public( b2s_matrix A, const void* x, void* y, double alpha, double beta, int32_t rb, int32_t re, b2s_memory where,
             cudaStream_t s )
{
   const Real* dx = static_cast< const Real* >( x );
   Real* dy = static_cast< Real* >( y );
   if( where == B2S_HOST ) {
      // host vectors: stage through the handle's device buffers on the caller's stream
      const size_t bx = (size_t) std::max( A->cols, 1 ) * sizeof( Real );
      const size_t by = (size_t) std::max( A->rows, 1 ) * sizeof( Real );
      if( A->stage_x.bytes < bx )
         B2S_TRY( A->stage_x.alloc( bx ) );
      if( A->stage_y.bytes < by )
         B2S_TRY( A->stage_y.alloc( by ) );
      B2S_TRY_CUDA( cudaMemcpyAsync( A->stage_x.p, x, (size_t) A->cols * sizeof( Real ), cudaMemcpyHostToDevice, s ) );
      if( beta != 0.0 || rb != 0 || re != A->rows )
         B2S_TRY_CUDA( cudaMemcpyAsync( A->stage_y.p, y, (size_t) A->rows * sizeof( Real ), cudaMemcpyHostToDevice, s ) );
      dx = A->stage_x.as< Real >();
      dy = A->stage_y.as< Real >();
   }
   SpmvArgs< Real > a{ A, A->values.as< Real >(), dx, rb, re };
   B2S_TRY( spmv_plain< Real >( a, dy, (Real) alpha, (Real) beta, s ) );
   if( where == B2S_HOST ) {
      B2S_TRY_CUDA( cudaMemcpyAsync( y, dy, (size_t) A->rows * sizeof( Real ), cudaMemcpyDeviceToHost, s ) );
      B2S_TRY_CUDA( cudaStreamSynchronize( s ) );
      return device_status( A, s );
   }
   return B2S_OK;
}

}  // namespace b2s

using namespace b2s;

extern "C" b2s_status
b2s_matrix_device_status( b2s_matrix A, b2s_stream stream )
{
   clear_error();
   B2S_CHECK_ARG( A, "matrix handle is NULL" );
   B2S_TRY_CUDA( cudaStreamSynchronize( as_stream( stream ) ) );
   return device_status( A, as_stream( stream ) );
}

extern "C" b2s_status
b2s_spmv( b2s_matrix A, const void* x, void* y, double alpha, double beta, int32_t row_begin, int32_t row_end,
          b2s_memory where, b2s_stream stream )
{
   clear_error();
   B2S_CHECK_ARG( A, "matrix handle is NULL" );
   B2S_CHECK_ARG( where == B2S_HOST || where == B2S_DEVICE, "where" );
   if( row_end == 0 )
      row_end = A->rows;
   B2S_CHECK_ARG( row_begin >= 0 && row_begin <= row_end && row_end <= A->rows, "row range" );
   B2S_CHECK_ARG( ( x || A->cols == 0 ) && ( y || A->rows == 0 ), "x/y NULL" );
   if( A->dtype == B2S_F64 )
      return spmv_public< double >( A, x, y, alpha, beta, row_begin, row_end, where, as_stream( stream ) );
   return spmv_public< float >( A, x, y, alpha, beta, row_begin, row_end, where, as_stream( stream ) );
}
