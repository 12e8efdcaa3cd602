// Row and column permutations of sparse matrices and arrays on the device:
//   permuteMatrixRows    (Matrices/MatrixPermutationApplier.h:17-62), CSR
//   permuteMatrixColumns (Matrices/MatrixPermutationApplier.h:64-90), any layout
//   reorderSparseMatrix  (Matrices/SparseOperations_impl.h:253-312), CSR -> CSR
//   reorderArray         (Matrices/SparseOperations_impl.h:314-338)
// TNL runs reorderSparseMatrix on the host only; here all four are kernels.
// Every permutation index is range-checked on the device (a bad index fails
// the call with B2S_INVALID_ARG before anything is written back).
#include "b2s_internal.cuh"

#include <algorithm>
#include <memory>

namespace b2s {

// flag[0] |= 1 when some index is outside [0, bound)
__global__ void
perm_check_kernel( const int32_t* __restrict__ p, int64_t n, int32_t bound, int* flag )
{
   for( int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x )
      if( p[ i ] < 0 || p[ i ] >= bound )
         atomicOr( flag, 1 );
}

// len[i] = length of row perm[i]
__global__ void
perm_lengths_kernel( const int32_t* __restrict__ off, const int32_t* __restrict__ perm, int32_t rows, int64_t* len )
{
   for( int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i <= rows; i += (int64_t) gridDim.x * blockDim.x )
      len[ i ] = i < rows ? (int64_t) off[ perm[ i ] + 1 ] - off[ perm[ i ] ] : 0;
}

__global__ void
i64_to_i32_kernel( const int64_t* __restrict__ a, int32_t* b, int64_t n )
{
   for( int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x )
      b[ i ] = (int32_t) a[ i ];
}

// row i of the result = row perm[i]; columns mapped by iperm (when given) and,
// with SORT, sorted ascending (insertion sort of the row, one warp lane per row)
template< typename Real, bool SORT >
__global__ void
perm_rows_copy_kernel( const int32_t* __restrict__ off, const int32_t* __restrict__ col, const Real* __restrict__ val,
                       const int32_t* __restrict__ perm, const int32_t* __restrict__ iperm, int32_t rows,
                       const int32_t* __restrict__ noff, int32_t* ncol, Real* nval )
{
   for( int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < rows; i += (int64_t) gridDim.x * blockDim.x ) {
      const int b = off[ perm[ i ] ], e = off[ perm[ i ] + 1 ];
      const int d = noff[ i ];
      for( int k = b; k < e; k++ ) {
         ncol[ d + k - b ] = iperm ? iperm[ col[ k ] ] : col[ k ];
         nval[ d + k - b ] = val[ k ];
      }
      if constexpr( SORT ) {
         for( int k = d + 1; k < d + ( e - b ); k++ ) {
            const int ck = ncol[ k ];
            const Real vk = nval[ k ];
            int j = k - 1;
            while( j >= d && ncol[ j ] > ck ) {
               ncol[ j + 1 ] = ncol[ j ];
               nval[ j + 1 ] = nval[ j ];
               j--;
            }
            ncol[ j + 1 ] = ck;
            nval[ j + 1 ] = vk;
         }
      }
   }
}

// stored column c -> iperm[c]; padding slots (-1) are left alone. The slots
// keep their order: rows are not re-sorted, exactly as TNL leaves them.
__global__ void
perm_columns_kernel( int32_t* col, int64_t n, const int32_t* __restrict__ iperm )
{
   for( int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x ) {
      const int c = col[ i ];
      if( c >= 0 )
         col[ i ] = iperm[ c ];
   }
}

template< typename T >
__global__ void
reorder_array_kernel( const T* __restrict__ src, T* __restrict__ dst, const int32_t* __restrict__ perm, int64_t n )
{
   for( int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x )
      dst[ i ] = src[ perm[ i ] ];
}

static int
pgrid( int64_t n )
{
   return (int) std::max< int64_t >( 1, std::min< int64_t >( ( n + 255 ) / 256, (int64_t) num_sms() * 16 ) );
}

// a device copy of a host or device permutation, range-checked against `bound`
static b2s_status
stage_perm( const int32_t* p, int64_t n, int32_t bound, b2s_memory where, DevBuf& buf, const int32_t*& dp,
            cudaStream_t s )
{
   if( where == B2S_HOST ) {
      B2S_TRY( buf.alloc( (size_t) std::max< int64_t >( n, 1 ) * sizeof( int32_t ) ) );
      if( n > 0 )
         B2S_TRY( copy_h2d( buf.p, p, (size_t) n * sizeof( int32_t ), s ) );
      dp = buf.as< int32_t >();
   }
   else
      dp = p;
   DevBuf flag;
   B2S_TRY( flag.alloc( sizeof( int ) ) );
   B2S_TRY_CUDA( cudaMemsetAsync( flag.p, 0, sizeof( int ), s ) );
   if( n > 0 ) {
      perm_check_kernel<<< pgrid( n ), 256, 0, s >>>( dp, n, bound, flag.as< int >() );
      B2S_TRY_CUDA( cudaGetLastError() );
   }
   int h = 0;
   B2S_TRY( copy_d2h( &h, flag.p, sizeof( int ), s ) );
   if( h ) {
      set_error( "permutation index outside [0, %d)", bound );
      return B2S_INVALID_ARG;
   }
   return B2S_OK;
}

// New CSR arrays of the row-permuted (and optionally column-mapped, sorted) matrix,
// built into a fresh handle with the options of `A`.
static b2s_status
permuted_csr( const b2s_matrix_t* A, const int32_t* perm, const int32_t* iperm, bool sort, cudaStream_t s,
              b2s_matrix* out )
{
   const int32_t rows = A->rows;
   DevBuf len, noff, ncol, nval;
   B2S_TRY( len.alloc( ( (size_t) rows + 1 ) * sizeof( int64_t ) ) );
   B2S_TRY( noff.alloc( ( (size_t) rows + 1 ) * sizeof( int32_t ) ) );
   B2S_TRY( ncol.alloc( (size_t) std::max< int64_t >( A->nnz, 1 ) * sizeof( int32_t ) ) );
   const size_t es = A->dtype == B2S_F64 ? 8 : 4;
   B2S_TRY( nval.alloc( (size_t) std::max< int64_t >( A->nnz, 1 ) * es ) );
   perm_lengths_kernel<<< pgrid( (int64_t) rows + 1 ), 256, 0, s >>>( A->offsets.as< int32_t >(), perm, rows,
                                                                        len.as< int64_t >() );
   B2S_TRY_CUDA( cudaGetLastError() );
   B2S_TRY( scan_exclusive_i64( len.as< int64_t >(), (int64_t) rows + 1, s ) );
   i64_to_i32_kernel<<< pgrid( (int64_t) rows + 1 ), 256, 0, s >>>( len.as< int64_t >(), noff.as< int32_t >(),
                                                                      (int64_t) rows + 1 );
   B2S_TRY_CUDA( cudaGetLastError() );
   if( rows > 0 ) {
#define B2S_PERM_COPY( T, SORT )                                                                                     \
   perm_rows_copy_kernel< T, SORT ><<< pgrid( rows ), 256, 0, s >>>(                                                 \
      A->offsets.as< int32_t >(), A->columns.as< int32_t >(), A->values.as< T >(), perm, iperm, rows,                \
      noff.as< int32_t >(), ncol.as< int32_t >(), nval.as< T >() )
      if( A->dtype == B2S_F64 ) {
         if( sort )
            B2S_PERM_COPY( double, true );
         else
            B2S_PERM_COPY( double, false );
      }
      else {
         if( sort )
            B2S_PERM_COPY( float, true );
         else
            B2S_PERM_COPY( float, false );
      }
#undef B2S_PERM_COPY
      B2S_TRY_CUDA( cudaGetLastError() );
   }
   b2s_matrix_opts mo;
   b2s_matrix_opts_default( &mo );
   mo.csr_kernel = A->csr_kernel;
   mo.threads_per_row = A->tpr;
   mo.keep_fp32_copy = A->values32.p != nullptr ? 1 : 0;
   mo.csr_row_groups = A->csr_group_opt;
   return b2s_matrix_create( B2S_CSR, (b2s_dtype) A->dtype, rows, A->cols, A->nnz, noff.as< int32_t >(),
                             ncol.as< int32_t >(), nval.p, (b2s_dtype) A->dtype, B2S_DEVICE, &mo,
                             reinterpret_cast< b2s_stream >( s ), out );
}

}  // namespace b2s

using namespace b2s;

extern "C" {

b2s_status
b2s_matrix_permute_rows( b2s_matrix A, const int32_t* perm, b2s_memory where, b2s_stream stream )
{
   clear_error();
   B2S_NO_BINARY( A, "row permutation" );
   B2S_CHECK_ARG( A && ( perm || A->rows == 0 ), "NULL argument" );
   if( A->symmetric ) {
      set_error( "permuteMatrixRows is not provided for SymmetricMatrix (lower-triangle) storage" );
      return B2S_UNSUPPORTED;
   }
   B2S_CHECK_ARG( where == B2S_HOST || where == B2S_DEVICE, "where" );
   if( A->format != B2S_CSR ) {
      set_error( "row permutation works on CSR matrices: permute the CSR matrix, then convert" );
      return B2S_UNSUPPORTED;
   }
   cudaStream_t s = as_stream( stream );
   DevBuf pbuf;
   const int32_t* dp = nullptr;
   B2S_TRY( stage_perm( perm, A->rows, A->rows, where, pbuf, dp, s ) );
   b2s_matrix tmp = nullptr;
   B2S_TRY( permuted_csr( A, dp, nullptr, false, s, &tmp ) );
   // the permuted matrix takes the place of A (same handle for the caller)
   std::unique_ptr< b2s_matrix_t > hold( tmp );
   B2S_TRY_CUDA( cudaStreamSynchronize( s ) );
   *A = std::move( *tmp );
   return B2S_OK;
}

b2s_status
b2s_matrix_permute_columns( b2s_matrix A, const int32_t* iperm, b2s_memory where, b2s_stream stream )
{
   clear_error();
   B2S_NO_BINARY( A, "column permutation" );
   B2S_CHECK_ARG( A && ( iperm || A->cols == 0 ), "NULL argument" );
   if( A->symmetric ) {
      set_error( "permuteMatrixColumns is not provided for SymmetricMatrix (lower-triangle) storage" );
      return B2S_UNSUPPORTED;
   }
   B2S_CHECK_ARG( where == B2S_HOST || where == B2S_DEVICE, "where" );
   if( A->format == B2S_MULTIDIAGONAL ) {
      set_error( "a Multidiagonal matrix has no column indices to permute: convert it to a sparse layout first" );
      return B2S_UNSUPPORTED;
   }
   cudaStream_t s = as_stream( stream );
   DevBuf pbuf;
   const int32_t* dp = nullptr;
   B2S_TRY( stage_perm( iperm, A->cols, A->cols, where, pbuf, dp, s ) );
   if( A->alloc_elems > 0 ) {
      perm_columns_kernel<<< pgrid( A->alloc_elems ), 256, 0, s >>>( A->columns.as< int32_t >(), A->alloc_elems, dp );
      B2S_TRY_CUDA( cudaGetLastError() );
   }
   // the Jacobi diagonal follows the new column indices
   B2S_TRY( build_diagonal( A, s ) );
   B2S_TRY_CUDA( cudaStreamSynchronize( s ) );
   return B2S_OK;
}

b2s_status
b2s_matrix_reorder( b2s_matrix src, const int32_t* perm, const int32_t* iperm, b2s_memory where, b2s_stream stream,
                    b2s_matrix* out )
{
   clear_error();
   B2S_NO_BINARY( src, "reordering" );
   B2S_CHECK_ARG( src && out && ( ( perm && iperm ) || src->rows == 0 ), "NULL argument" );
   if( src->symmetric ) {
      set_error( "reorderSparseMatrix is not provided for SymmetricMatrix (lower-triangle) storage" );
      return B2S_UNSUPPORTED;
   }
   B2S_CHECK_ARG( where == B2S_HOST || where == B2S_DEVICE, "where" );
   *out = nullptr;
   if( src->format != B2S_CSR ) {
      set_error( "reordering works on CSR matrices" );
      return B2S_UNSUPPORTED;
   }
   cudaStream_t s = as_stream( stream );
   DevBuf pb, ib;
   const int32_t *dp = nullptr, *di = nullptr;
   B2S_TRY( stage_perm( perm, src->rows, src->rows, where, pb, dp, s ) );
   B2S_TRY( stage_perm( iperm, src->cols, src->cols, where, ib, di, s ) );
   return permuted_csr( src, dp, di, true, s, out );
}

b2s_status
b2s_reorder_array( int32_t element_size, int64_t n, const void* src, void* dest, const int32_t* perm,
                   b2s_stream stream )
{
   clear_error();
   B2S_CHECK_ARG( element_size == 4 || element_size == 8, "element_size must be 4 or 8" );
   B2S_CHECK_ARG( n >= 0 && ( n == 0 || ( src && dest && perm ) ), "NULL argument" );
   B2S_CHECK_ARG( src != dest || n == 0, "src and dest must differ" );
   cudaStream_t s = as_stream( stream );
   DevBuf pbuf;
   const int32_t* dp = nullptr;
   B2S_TRY( stage_perm( perm, n, n > INT32_MAX ? INT32_MAX : (int32_t) n, B2S_DEVICE, pbuf, dp, s ) );
   if( n == 0 )
      return B2S_OK;
   if( element_size == 4 )
      reorder_array_kernel< int32_t ><<< pgrid( n ), 256, 0, s >>>( static_cast< const int32_t* >( src ),
                                                                    static_cast< int32_t* >( dest ), dp, n );
   else
      reorder_array_kernel< int64_t ><<< pgrid( n ), 256, 0, s >>>( static_cast< const int64_t* >( src ),
                                                                    static_cast< int64_t* >( dest ), dp, n );
   B2S_TRY_CUDA( cudaGetLastError() );
   return B2S_OK;
}

}  // extern "C"
