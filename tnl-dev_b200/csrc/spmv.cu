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

HostPipe::~HostPipe()
{
   int cur = -1;
   cudaGetDevice( &cur );
   if( device >= 0 && device != cur )
      cudaSetDevice( device );
   for( cudaEvent_t e : x_ready )
      cudaEventDestroy( e );
   for( cudaEvent_t e : y_ready )
      cudaEventDestroy( e );
   if( exec )
      cudaGraphExecDestroy( exec );
   if( start )
      cudaEventDestroy( start );
   if( done )
      cudaEventDestroy( done );
   if( up )
      cudaStreamDestroy( up );
   if( down )
      cudaStreamDestroy( down );
   if( work )
      cudaStreamDestroy( work );
   if( device >= 0 && device != cur && cur >= 0 )
      cudaSetDevice( cur );
}

// gmax[g] = the largest column of rows [32 g, 32 g + 32) (-1: none)
__global__ void
group_xmax_kernel( const int32_t* __restrict__ off, const int32_t* __restrict__ col, int32_t rows, int* __restrict__ gmax )
{
   const int lane = threadIdx.x & 31;
   const int64_t warps = (int64_t) gridDim.x * ( blockDim.x / 32 );
   for( int64_t base = ( blockIdx.x * (int64_t) blockDim.x + threadIdx.x - lane ); base < rows; base += 32 * warps ) {
      const int64_t r = base + lane;
      int m = -1;
      if( r < rows )
         for( int k = off[ r ]; k < off[ r + 1 ]; k++ )
            m = max( m, col[ k ] );
      m = __reduce_max_sync( 0xffffffffu, m );
      if( lane == 0 )
         gmax[ base / 32 ] = m;
   }
}

// Host vectors on a CSR matrix (row-group kernel): x goes up in chunks on one
// stream, and after x chunk k has arrived one product computes every row whose
// columns all lie in chunks 0..k and that no earlier product took (the row
// cuts follow the running maximum column of 32-row groups, so each product
// waits for the chunk that just arrived); y goes to the host as the products
// finish. The PCIe upload, the products and the download overlap.
constexpr int32_t kPipeMinRows = 1 << 16;
#ifndef B2S_PIPE_CHUNK_BYTES
#define B2S_PIPE_CHUNK_BYTES ( 2u << 20 )
#endif
constexpr size_t kPipeChunkBytes = B2S_PIPE_CHUNK_BYTES;

template< typename Real >
static b2s_status
build_pipe( b2s_matrix_t* A, cudaStream_t s )
{
   std::unique_ptr< HostPipe > P( new HostPipe() );
   P->device = current_device();
   const int32_t rows = A->rows, cols = A->cols;
   const size_t xbytes = (size_t) cols * sizeof( Real );
   const int K = (int) std::max< size_t >( 2, std::min< size_t >( 32, ( xbytes + kPipeChunkBytes - 1 ) / kPipeChunkBytes ) );
   const int32_t cpc = (int32_t) std::max< int64_t >( 1, ( (int64_t) cols + K - 1 ) / K );
   const int nxc = (int) ( ( (int64_t) cols + cpc - 1 ) / cpc );
   for( int k = 0; k <= nxc; k++ )
      P->x_cut.push_back( (int32_t) std::min< int64_t >( (int64_t) k * cpc, cols ) );
   const int64_t groups = ( (int64_t) rows + 31 ) / 32;
   DevBuf dmax;
   B2S_TRY( dmax.alloc( (size_t) std::max< int64_t >( groups, 1 ) * sizeof( int ) ) );
   group_xmax_kernel<<< (int) std::min< int64_t >( ( rows + 255 ) / 256, (int64_t) num_sms() * 32 ), 256, 0, s >>>(
      A->offsets.as< int32_t >(), A->columns.as< int32_t >(), rows, dmax.as< int >() );
   B2S_TRY_CUDA( cudaGetLastError() );
   std::vector< int > gmax( (size_t) groups );
   if( groups > 0 )
      B2S_TRY( copy_d2h( gmax.data(), dmax.p, (size_t) groups * sizeof( int ), s ) );
   // rows ready after x chunk k: the groups whose running maximum column lies
   // below x_cut[k + 1] (the last chunk takes every remaining row)
   P->row_cut.push_back( 0 );
   int64_t g = 0;
   int run = -1;
   for( int k = 0; k < nxc; k++ ) {
      const int limit = P->x_cut[ k + 1 ];
      while( g < groups && ( k == nxc - 1 || std::max( run, gmax[ g ] ) < limit ) ) {
         run = std::max( run, gmax[ g ] );
         g++;
      }
      const int32_t cut = (int32_t) std::min< int64_t >( g * 32, rows );
      if( cut > P->row_cut.back() ) {
         P->row_cut.push_back( cut );
         P->need.push_back( k );
      }
   }
   if( P->row_cut.back() < rows ) {  // rows only when the matrix has no columns
      P->row_cut.push_back( rows );
      P->need.push_back( -1 );
   }
   const int nrc = (int) P->need.size();
   B2S_TRY_CUDA( cudaStreamCreateWithFlags( &P->up, cudaStreamNonBlocking ) );
   B2S_TRY_CUDA( cudaStreamCreateWithFlags( &P->down, cudaStreamNonBlocking ) );
   B2S_TRY_CUDA( cudaStreamCreateWithFlags( &P->work, cudaStreamNonBlocking ) );
   B2S_TRY_CUDA( cudaEventCreateWithFlags( &P->start, cudaEventDisableTiming ) );
   B2S_TRY_CUDA( cudaEventCreateWithFlags( &P->done, cudaEventDisableTiming ) );
   P->x_ready.resize( nxc, nullptr );
   P->y_ready.resize( nrc, nullptr );
   for( auto& e : P->x_ready )
      B2S_TRY_CUDA( cudaEventCreateWithFlags( &e, cudaEventDisableTiming ) );
   for( auto& e : P->y_ready )
      B2S_TRY_CUDA( cudaEventCreateWithFlags( &e, cudaEventDisableTiming ) );
   A->pipe = std::move( P );
   return B2S_OK;
}

// The pipeline, once P.start has been recorded behind the work that must
// come first: x chunks on `up`, products on `cs`; `done` is recorded when y
// is on the host and x is no longer read. `y_mapped` (page-locked y, its
// device-side address): the products write y straight into host memory — the
// SMs' PCIe writes overlap the copy engine's x chunks, where chunked copies
// in both directions on two streams interfere (measured on B200: 16.8 MB up
// and down in 8 + 8 chunks 490 us, the same upload beside a kernel writing the
// 16.8 MB into host memory 375 us). Otherwise y chunks go down on `down`.
template< typename Real >
static b2s_status
pipe_body( b2s_matrix_t* A, HostPipe& P, const Real* x, Real* y, Real* y_mapped, Real alpha, cudaStream_t cs )
{
   Real* sx = A->stage_x.as< Real >();
   Real* sy = A->stage_y.as< Real >();
   B2S_TRY_CUDA( cudaStreamWaitEvent( P.up, P.start, 0 ) );
   B2S_TRY_CUDA( cudaStreamWaitEvent( P.down, P.start, 0 ) );
   B2S_TRY_CUDA( cudaStreamWaitEvent( cs, P.start, 0 ) );
   const int nxc = (int) P.x_ready.size(), nrc = (int) P.y_ready.size();
   for( int k = 0; k < nxc; k++ ) {
      const int32_t a = P.x_cut[ k ], b = P.x_cut[ k + 1 ];
      B2S_TRY_CUDA( cudaMemcpyAsync( sx + a, x + a, (size_t) ( b - a ) * sizeof( Real ), cudaMemcpyHostToDevice, P.up ) );
      B2S_TRY_CUDA( cudaEventRecord( P.x_ready[ k ], P.up ) );
   }
   YSink< Real > sink{ y_mapped ? y_mapped : sy, alpha, Real( 0 ), keeper_mode( alpha, Real( 0 ) ) };
   for( int c = 0; c < nrc; c++ ) {
      const int32_t a = P.row_cut[ c ], b = P.row_cut[ c + 1 ];
      if( P.need[ c ] >= 0 )
         B2S_TRY_CUDA( cudaStreamWaitEvent( cs, P.x_ready[ P.need[ c ] ], 0 ) );
      B2S_TRY( ( spmv_dispatch< Real, YSink< Real > >( A, A->values.as< Real >(), sx, a, b, sink, RedScratch{}, cs ) ) );
      if( ! y_mapped ) {
         B2S_TRY_CUDA( cudaEventRecord( P.y_ready[ c ], cs ) );
         B2S_TRY_CUDA( cudaStreamWaitEvent( P.down, P.y_ready[ c ], 0 ) );
         B2S_TRY_CUDA(
            cudaMemcpyAsync( y + a, sy + a, (size_t) ( b - a ) * sizeof( Real ), cudaMemcpyDeviceToHost, P.down ) );
      }
   }
   if( y_mapped ) {
      // the last product wrote the last of y; `down` only joins
      B2S_TRY_CUDA( cudaEventRecord( P.y_ready[ nrc - 1 ], cs ) );
      B2S_TRY_CUDA( cudaStreamWaitEvent( P.down, P.y_ready[ nrc - 1 ], 0 ) );
   }
   B2S_TRY_CUDA( cudaStreamWaitEvent( P.down, P.x_ready[ nxc - 1 ], 0 ) );
   B2S_TRY_CUDA( cudaEventRecord( P.done, P.down ) );
   return B2S_OK;
}

static bool
is_pinned( const void* p )
{
   cudaPointerAttributes at;
   if( cudaPointerGetAttributes( &at, p ) != cudaSuccess ) {
      cudaGetLastError();
      return false;
   }
   return at.type == cudaMemoryTypeHost;
}

template< typename Real >
static b2s_status
spmv_host_pipelined( b2s_matrix_t* A, const Real* x, Real* y, Real alpha, cudaStream_t s )
{
   if( ! A->pipe || A->pipe->device != current_device() )
      B2S_TRY( build_pipe< Real >( A, s ) );
   HostPipe& P = *A->pipe;
   if( is_pinned( x ) && is_pinned( y ) ) {
      // y's device-side address (page-locked memory is mapped under unified
      // addressing); without one the products go through the staging buffer
      Real* ym = nullptr;
      if( cudaHostGetDevicePointer( reinterpret_cast< void** >( &ym ), y, 0 ) != cudaSuccess ) {
         cudaGetLastError();
         ym = nullptr;
      }
      // page-locked vectors: the pipeline is captured once (on the library's own
      // streams) and replayed as one graph launch on the caller's stream
      if( ! P.exec || P.gx != x || P.gy != y || P.galpha != (double) alpha ) {
         if( P.exec ) {
            cudaGraphExecDestroy( P.exec );
            P.exec = nullptr;
         }
         cudaGraph_t g = nullptr;
         B2S_TRY_CUDA( cudaStreamBeginCapture( P.up, cudaStreamCaptureModeThreadLocal ) );
         b2s_status st = B2S_OK;
         if( cudaEventRecord( P.start, P.up ) != cudaSuccess )
            st = B2S_CUDA_ERROR;
         if( st == B2S_OK )
            st = pipe_body< Real >( A, P, x, y, ym, alpha, P.work );
         if( st == B2S_OK && cudaStreamWaitEvent( P.up, P.done, 0 ) != cudaSuccess )
            st = B2S_CUDA_ERROR;
         const cudaError_t ee = cudaStreamEndCapture( P.up, &g );
         if( st != B2S_OK || ee != cudaSuccess ) {
            if( g )
               cudaGraphDestroy( g );
            cudaGetLastError();
            set_error( "capture of the host-vector SpMV pipeline failed" );
            return st != B2S_OK ? st : B2S_CUDA_ERROR;
         }
         const cudaError_t ie = cudaGraphInstantiate( &P.exec, g, 0 );
         cudaGraphDestroy( g );
         if( ie != cudaSuccess ) {
            P.exec = nullptr;
            set_error( "graph instantiation: %s", cudaGetErrorString( ie ) );
            return B2S_CUDA_ERROR;
         }
         P.gx = x;
         P.gy = y;
         P.galpha = alpha;
      }
      B2S_TRY_CUDA( cudaGraphLaunch( P.exec, s ) );
   }
   else {
      // pageable vectors: the same pipeline issued directly
      B2S_TRY_CUDA( cudaEventRecord( P.start, s ) );
      B2S_TRY( pipe_body< Real >( A, P, x, y, nullptr, alpha, s ) );
      B2S_TRY_CUDA( cudaStreamWaitEvent( s, P.done, 0 ) );
   }
   B2S_TRY_CUDA( cudaStreamSynchronize( s ) );
   return B2S_OK;
}

// SymmetricMatrix (SparseMatrixView.hpp:413-476): y *= beta over the whole
// vector (unless beta is 1), then for every row i of [rb, re): each stored
// element (i, j, v) with j < i adds alpha v x_i to y_j, and alpha times the
// row's sum of v x_j (all its stored elements, in order) is added to y_i —
// both by atomics, as TNL does on the GPU.
template< typename Real >
__global__ void
scale_kernel( int64_t n, Real beta, Real* __restrict__ y )
{
   for( int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x )
      y[ i ] = beta * y[ i ];
}

template< typename Real >
__global__ void
csr_symmetric_kernel( const int32_t* __restrict__ off, const int32_t* __restrict__ col, const Real* __restrict__ val,
                      const Real* __restrict__ x, Real* y, Real alpha, int32_t rb, int32_t re )
{
   for( int64_t r = rb + blockIdx.x * (int64_t) blockDim.x + threadIdx.x; r < re; r += (int64_t) gridDim.x * blockDim.x ) {
      const Real xr = x[ r ];
      Real sum = 0;
      for( int k = off[ r ]; k < off[ r + 1 ]; k++ ) {
         const int j = col[ k ];
         const Real v = val[ k ];
         if( j < r )
            atomicAdd( y + j, alpha * v * xr );
         sum += v * x[ j ];
      }
      atomicAdd( y + r, alpha * sum );
   }
}

template< typename Real >
static b2s_status
spmv_symmetric( const b2s_matrix_t* A, const Real* x, Real* y, Real alpha, Real beta, int32_t rb, int32_t re,
                cudaStream_t s )
{
   const int64_t n = A->rows;
   const int cap = num_sms() * 8;
   if( beta != Real( 1 ) && n > 0 ) {
      scale_kernel< Real ><<< (int) std::min< int64_t >( ( n + 255 ) / 256, cap ), 256, 0, s >>>( n, beta, y );
      B2S_TRY_CUDA( cudaGetLastError() );
   }
   if( re > rb && A->format != B2S_CSR )
      return spmv_symmetric_layout( A, A->values.p, x, y, (double) alpha, rb, re, s );
   if( re > rb ) {
      csr_symmetric_kernel< Real ><<< (int) std::min< int64_t >( ( re - rb + 255 ) / 256, cap ), 256, 0, s >>>(
         A->offsets.as< int32_t >(), A->columns.as< int32_t >(), A->values.as< Real >(), x, y, alpha, rb, re );
      B2S_TRY_CUDA( cudaGetLastError() );
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
   // pipelined when the chunked products are the whole-matrix product bit for
   // bit: the row-group kernel sums every row alike whatever the row range
   if( where == B2S_HOST && A->format == B2S_CSR && A->csr_kernel == B2S_CSR_ADAPTIVE && A->csr_group &&
       ! A->symmetric && beta == 0.0 && rb == 0 && re == A->rows && A->rows >= kPipeMinRows && A->cols > 0 ) {
      const size_t bx = (size_t) A->cols * sizeof( Real ), by = (size_t) A->rows * sizeof( Real );
      if( A->stage_x.bytes < bx )
         B2S_TRY( A->stage_x.alloc( bx ) );
      if( A->stage_y.bytes < by )
         B2S_TRY( A->stage_y.alloc( by ) );
      return spmv_host_pipelined< Real >( A, static_cast< const Real* >( x ), static_cast< Real* >( y ), (Real) alpha,
                                          s );
   }
   if( where == B2S_HOST ) {
      // host vectors: stage through the handle's device buffers on the caller's stream
      const size_t bx = (size_t) std::max( A->cols, 1 ) * sizeof( Real );
      const size_t by = (size_t) std::max( A->rows, 1 ) * sizeof( Real );
      if( A->stage_x.bytes < bx )
         B2S_TRY( A->stage_x.alloc( bx ) );
      if( A->stage_y.bytes < by )
         B2S_TRY( A->stage_y.alloc( by ) );
      B2S_TRY_CUDA( cudaMemcpyAsync( A->stage_x.p, x, (size_t) A->cols * sizeof( Real ), cudaMemcpyHostToDevice, s ) );
      if( beta != 0.0 || rb != 0 || re != A->rows || A->symmetric )
         B2S_TRY_CUDA( cudaMemcpyAsync( A->stage_y.p, y, (size_t) A->rows * sizeof( Real ), cudaMemcpyHostToDevice, s ) );
      dx = A->stage_x.as< Real >();
      dy = A->stage_y.as< Real >();
   }
   if( A->symmetric ) {
      B2S_TRY( spmv_symmetric< Real >( A, dx, dy, (Real) alpha, (Real) beta, rb, re, s ) );
      if( where == B2S_HOST ) {
         B2S_TRY_CUDA( cudaMemcpyAsync( y, dy, (size_t) A->rows * sizeof( Real ), cudaMemcpyDeviceToHost, s ) );
         B2S_TRY_CUDA( cudaStreamSynchronize( s ) );
      }
      return B2S_OK;
   }
   SpmvArgs< Real > a{ A, A->values.as< Real >(), dx, rb, re };
   B2S_TRY( spmv_plain< Real >( a, dy, (Real) alpha, (Real) beta, s ) );
   if( where == B2S_HOST ) {
      B2S_TRY_CUDA( cudaMemcpyAsync( y, dy, (size_t) A->rows * sizeof( Real ), cudaMemcpyDeviceToHost, s ) );
      B2S_TRY_CUDA( cudaStreamSynchronize( s ) );
   }
   return B2S_OK;
}

// a binary matrix's product with vectors of element size es (x and y staged
// through the handle's buffers when they are host memory)
static b2s_status
spmv_binary_public( b2s_matrix A, const void* x, void* y, int vdt, double alpha, double beta, int32_t rb, int32_t re,
                    b2s_memory where, cudaStream_t s )
{
   const size_t es = vdt == B2S_F64 ? 8 : 4;
   const void* dx = x;
   void* dy = y;
   if( where == B2S_HOST ) {
      const size_t bx = (size_t) std::max( A->cols, 1 ) * es, by = (size_t) std::max( A->rows, 1 ) * es;
      if( A->stage_x.bytes < bx )
         B2S_TRY( A->stage_x.alloc( bx ) );
      if( A->stage_y.bytes < by )
         B2S_TRY( A->stage_y.alloc( by ) );
      B2S_TRY_CUDA( cudaMemcpyAsync( A->stage_x.p, x, (size_t) A->cols * es, cudaMemcpyHostToDevice, s ) );
      B2S_TRY_CUDA( cudaMemcpyAsync( A->stage_y.p, y, (size_t) A->rows * es, cudaMemcpyHostToDevice, s ) );
      dx = A->stage_x.p;
      dy = A->stage_y.p;
   }
   B2S_TRY( spmv_binary( A, dx, dy, vdt, alpha, beta, rb, re, s ) );
   if( where == B2S_HOST ) {
      B2S_TRY_CUDA( cudaMemcpyAsync( y, dy, (size_t) A->rows * es, cudaMemcpyDeviceToHost, s ) );
      B2S_TRY_CUDA( cudaStreamSynchronize( s ) );
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
   if( A->dtype == B2S_BOOL )
      return spmv_binary_public( A, x, y, B2S_F64, alpha, beta, row_begin, row_end, where, as_stream( stream ) );
   if( A->dtype == B2S_F64 )
      return spmv_public< double >( A, x, y, alpha, beta, row_begin, row_end, where, as_stream( stream ) );
   return spmv_public< float >( A, x, y, alpha, beta, row_begin, row_end, where, as_stream( stream ) );
}

extern "C" b2s_status
b2s_spmv_ex( b2s_matrix A, const void* x, void* y, b2s_dtype vectors, double alpha, double beta, int32_t row_begin,
             int32_t row_end, b2s_memory where, b2s_stream stream )
{
   clear_error();
   B2S_CHECK_ARG( A, "matrix handle is NULL" );
   B2S_CHECK_ARG( vectors == B2S_F64 || vectors == B2S_F32, "vectors must be B2S_F64 or B2S_F32" );
   if( A->dtype != B2S_BOOL ) {
      B2S_CHECK_ARG( (int) vectors == A->dtype, "vectors of another type than the matrix values" );
      return b2s_spmv( A, x, y, alpha, beta, row_begin, row_end, where, stream );
   }
   B2S_CHECK_ARG( where == B2S_HOST || where == B2S_DEVICE, "where" );
   if( row_end == 0 )
      row_end = A->rows;
   B2S_CHECK_ARG( row_begin >= 0 && row_begin <= row_end && row_end <= A->rows, "row range" );
   B2S_CHECK_ARG( ( x || A->cols == 0 ) && ( y || A->rows == 0 ), "x/y NULL" );
   return spmv_binary_public( A, x, y, vectors, alpha, beta, row_begin, row_end, where, as_stream( stream ) );
}
