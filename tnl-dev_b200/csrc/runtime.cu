// Runtime pieces of libb2sparse: error text, device buffers, grid sizing,
// host/device copies, the device-wide scan (TNL Algorithms/scan.h analogue)
// and the public reduce / vector primitives (Algorithms/reduce.h,
// Containers/Expressions/ExpressionTemplates.h:391-476).
#include "b2s_internal.cuh"

#include <cstdarg>
#include <map>
#include <mutex>
#include <tuple>

namespace b2s {

static thread_local std::string g_last_error;

void
set_error( const char* fmt, ... )
{
   char buf[ 1024 ];
   va_list ap;
   va_start( ap, fmt );
   vsnprintf( buf, sizeof( buf ), fmt, ap );
   va_end( ap );
   g_last_error = buf;
}

void
clear_error()
{
   g_last_error.clear();
}

int
current_device()
{
   int d = 0;
   cudaGetDevice( &d );
   return d;
}

int
num_sms()
{
   static int cache[ 64 ] = { 0 };
   const int d = current_device();
   if( d < 0 || d >= 64 )
      return 148;
   if( cache[ d ] == 0 ) {
      int v = 0;
      if( cudaDeviceGetAttribute( &v, cudaDevAttrMultiProcessorCount, d ) != cudaSuccess || v <= 0 )
         v = 148;
      cache[ d ] = v;
   }
   return cache[ d ];
}

int
resident_blocks( const void* kernel, int block )
{
   static std::mutex mu;
   static std::map< std::tuple< const void*, int, int >, int > cache;
   const auto key = std::make_tuple( kernel, block, current_device() );
   std::lock_guard< std::mutex > lock( mu );
   auto it = cache.find( key );
   if( it != cache.end() )
      return it->second;
   int occ = 0;
   if( cudaOccupancyMaxActiveBlocksPerMultiprocessor( &occ, kernel, block, 0 ) != cudaSuccess || occ < 1 ) {
      cudaGetLastError();
      occ = 1;
   }
   cache.emplace( key, occ );
   return occ;
}

int
reduce_grid( int64_t n, int per_thread )
{
   const int64_t want = ( n + (int64_t) kReduceBlock * per_thread - 1 ) / ( (int64_t) kReduceBlock * per_thread );
   int g = (int) std::min< int64_t >( want, (int64_t) num_sms() * 8 );
   if( g > kMaxReduceGrid )
      g = kMaxReduceGrid;
   return g < 1 ? 1 : g;
}

static thread_local const AllocCtx* t_alloc_ctx = nullptr;

void
set_thread_alloc_ctx( const AllocCtx* ctx )
{
   t_alloc_ctx = ctx;
}

const AllocCtx*
thread_alloc_ctx()
{
   return t_alloc_ctx;
}

b2s_status
DevBuf::alloc( size_t n )
{
   release();
   if( n == 0 )
      return B2S_OK;
   // pad so that 16-byte vector loads and bulk copies never leave the allocation
   const size_t padded = ( n + 255 ) / 256 * 256 + 256;
   cudaError_t e;
   const AllocCtx* ctx = t_alloc_ctx;
   if( ctx ) {
      // stream-ordered; the synchronize makes the memory usable on any stream
      e = cudaMallocFromPoolAsync( &p, padded, ctx->pool, ctx->stream );
      if( e == cudaSuccess )
         e = cudaStreamSynchronize( ctx->stream );
   }
   else
      e = cudaMalloc( &p, padded );
   if( e != cudaSuccess ) {
      p = nullptr;
      set_error( "device allocation of %zu bytes: %s", padded, cudaGetErrorString( e ) );
      cudaGetLastError();
      return e == cudaErrorMemoryAllocation ? B2S_OOM : B2S_CUDA_ERROR;
   }
   pooled = ctx != nullptr;
   pool_stream = ctx ? ctx->stream : nullptr;
   bytes = n;
   return B2S_OK;
}

void
DevBuf::release()
{
   if( p ) {
      // pool memory goes back on the stream it came from; the owner has
      // finished every kernel that used it before releasing it
      if( pooled )
         cudaFreeAsync( p, pool_stream );
      else
         cudaFree( p );
   }
   p = nullptr;
   bytes = 0;
   pooled = false;
   pool_stream = nullptr;
}

b2s_status
Scratch::init( int nslots, cudaStream_t s )
{
   if( slots >= nslots && buf.p )
      return B2S_OK;
   const size_t dbl = (size_t) nslots * 4 * kMaxReduceGrid * sizeof( double );
   B2S_TRY( buf.alloc( dbl + nslots * sizeof( unsigned int ) + 64 ) );
   partials = buf.as< double >();
   counters = reinterpret_cast< unsigned int* >( reinterpret_cast< char* >( buf.p ) + dbl );
   B2S_TRY_CUDA( cudaMemsetAsync( counters, 0, nslots * sizeof( unsigned int ), s ) );
   slots = nslots;
   return B2S_OK;
}

b2s_status
copy_h2d( void* dst, const void* src, size_t bytes, cudaStream_t s )
{
   if( bytes == 0 )
      return B2S_OK;
   B2S_TRY_CUDA( cudaMemcpyAsync( dst, src, bytes, cudaMemcpyHostToDevice, s ) );
   B2S_TRY_CUDA( cudaStreamSynchronize( s ) );
   return B2S_OK;
}

b2s_status
copy_d2h( void* dst, const void* src, size_t bytes, cudaStream_t s )
{
   if( bytes == 0 )
      return B2S_OK;
   B2S_TRY_CUDA( cudaMemcpyAsync( dst, src, bytes, cudaMemcpyDeviceToHost, s ) );
   B2S_TRY_CUDA( cudaStreamSynchronize( s ) );
   return B2S_OK;
}

// ---------------------------------------------------------------------------
// Device-wide exclusive scan (int64): tiles of 2048 elements, a block scan per
// tile, recursion over tile totals, then a uniform add.
constexpr int kScanThreads = 512;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

__global__ void
scan_tiles_kernel( int64_t* data, int64_t n, int64_t* tile_sums )
{
   __shared__ int64_t warp_tot[ kScanThreads / 32 ];
   const int64_t base = (int64_t) blockIdx.x * kScanTile + (int64_t) threadIdx.x * kScanItems;
   int64_t v[ kScanItems ];
   int64_t local = 0;
#pragma unroll
   for( int i = 0; i < kScanItems; i++ ) {
      v[ i ] = ( base + i < n ) ? data[ base + i ] : 0;
      local += v[ i ];
   }
   // inclusive warp scan of thread totals
   const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
   int64_t inc = local;
#pragma unroll
   for( int o = 1; o < 32; o <<= 1 ) {
      const int64_t t = __shfl_up_sync( 0xffffffffu, inc, o );
      if( lane >= o )
         inc += t;
   }
   if( lane == 31 )
      warp_tot[ warp ] = inc;
   __syncthreads();
   if( warp == 0 ) {
      int64_t w = lane < kScanThreads / 32 ? warp_tot[ lane ] : 0;
#pragma unroll
      for( int o = 1; o < 32; o <<= 1 ) {
         const int64_t t = __shfl_up_sync( 0xffffffffu, w, o );
         if( lane >= o )
            w += t;
      }
      if( lane < kScanThreads / 32 )
         warp_tot[ lane ] = w;  // inclusive over warps
   }
   __syncthreads();
   int64_t run = inc - local + ( warp > 0 ? warp_tot[ warp - 1 ] : 0 );
#pragma unroll
   for( int i = 0; i < kScanItems; i++ ) {
      if( base + i < n )
         data[ base + i ] = run;
      run += v[ i ];
   }
   if( threadIdx.x == kScanThreads - 1 )
      tile_sums[ blockIdx.x ] = run;
}

__global__ void
scan_add_kernel( int64_t* data, int64_t n, const int64_t* tile_offsets )
{
   const int64_t add = tile_offsets[ blockIdx.x ];
   const int64_t base = (int64_t) blockIdx.x * kScanTile;
   for( int i = threadIdx.x; i < kScanTile; i += kScanThreads )
      if( base + i < n )
         data[ base + i ] += add;
}

b2s_status
scan_exclusive_i64( int64_t* data, int64_t n, cudaStream_t s )
{
   if( n <= 0 )
      return B2S_OK;
   const int64_t tiles = ( n + kScanTile - 1 ) / kScanTile;
   DevBuf sums;
   B2S_TRY( sums.alloc( tiles * sizeof( int64_t ) ) );
   scan_tiles_kernel<<< (unsigned) tiles, kScanThreads, 0, s >>>( data, n, sums.as< int64_t >() );
   B2S_TRY_CUDA( cudaGetLastError() );
   if( tiles > 1 ) {
      B2S_TRY( scan_exclusive_i64( sums.as< int64_t >(), tiles, s ) );
      scan_add_kernel<<< (unsigned) tiles, kScanThreads, 0, s >>>( data, n, sums.as< int64_t >() );
      B2S_TRY_CUDA( cudaGetLastError() );
   }
   // keep `sums` alive until the kernels that read it have run
   B2S_TRY_CUDA( cudaStreamSynchronize( s ) );
   return B2S_OK;
}

__global__ void
i32_to_i64_kernel( const int32_t* in, int64_t* out, int64_t n )
{
   for( int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x )
      out[ i ] = in[ i ];
}

__global__ void
i64_to_i32_kernel( const int64_t* in, int32_t* out, int64_t n, int64_t* shift_inclusive, const int32_t* orig )
{
   for( int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x )
      out[ i ] = (int32_t) ( shift_inclusive ? in[ i ] + orig[ i ] : in[ i ] );
}

// ---------------------------------------------------------------------------
// Reductions and vector updates on raw device vectors.
template< typename Real, int MODE >
__global__ void __launch_bounds__( kReduceBlock )
reduce_kernel( int64_t n, const Real* __restrict__ a, const Real* __restrict__ b, RedScratch rs, double* result )
{
   double acc[ 1 ] = { 0.0 };
   for( int64_t i = blockIdx.x * (int64_t) kReduceBlock + threadIdx.x; i < n; i += (int64_t) gridDim.x * kReduceBlock ) {
      const double u = (double) a[ i ];
      acc[ 0 ] += MODE == 0 ? u * (double) b[ i ] : u * u;
   }
   double tot[ 1 ];
   if( grid_reduce< 1, kReduceBlock >( acc, rs, tot ) && threadIdx.x == 0 )
      *result = MODE == 0 ? tot[ 0 ] : sqrt( tot[ 0 ] );
}

// dest[i] = src[idx[i]]; an index outside [0, src_size) yields 0 (never a read
// outside the array)
template< typename T >
__global__ void
gather_kernel( int64_t n, const T* __restrict__ src, int64_t src_size, const int32_t* __restrict__ idx,
               T* __restrict__ dest )
{
   for( int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x ) {
      const int32_t k = idx[ i ];
      dest[ i ] = ( k >= 0 && k < src_size ) ? src[ k ] : T( 0 );
   }
}

template< typename Real >
__global__ void
axpby_kernel( int64_t n, Real alpha, const Real* __restrict__ x, Real beta, Real* __restrict__ y )
{
   for( int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x )
      y[ i ] = beta == Real( 0 ) ? alpha * x[ i ] : alpha * x[ i ] + beta * y[ i ];
}

// Scratch for the stateless reduction entry points: allocated stream-ordered
// per call.
template< typename Real, int MODE >
static b2s_status
reduce_call( int64_t n, const void* a, const void* b, double* result, cudaStream_t s )
{
   const int grid = reduce_grid( n, 4 );
   void* mem = nullptr;
   const size_t bytes = (size_t) grid * sizeof( double ) + 64;
   B2S_TRY_CUDA( cudaMallocAsync( &mem, bytes, s ) );
   RedScratch rs{ static_cast< double* >( mem ),
                  reinterpret_cast< unsigned int* >( static_cast< char* >( mem ) + (size_t) grid * sizeof( double ) ) };
   cudaError_t e = cudaMemsetAsync( rs.counter, 0, sizeof( unsigned int ), s );
   if( e == cudaSuccess ) {
      reduce_kernel< Real, MODE ><<< grid, kReduceBlock, 0, s >>>( n, static_cast< const Real* >( a ),
                                                                    static_cast< const Real* >( b ), rs, result );
      e = cudaGetLastError();
   }
   cudaFreeAsync( mem, s );
   if( e != cudaSuccess ) {
      set_error( "reduction launch: %s", cudaGetErrorString( e ) );
      return B2S_CUDA_ERROR;
   }
   return B2S_OK;
}

}  // namespace b2s

using namespace b2s;

extern "C" {

const char*
b2s_status_string( b2s_status s )
{
   switch( s ) {
      case B2S_OK: return "ok";
      case B2S_NOT_CONVERGED: return "not converged (iteration limit)";
      case B2S_NAN: return "residue is NaN";
      case B2S_DIVERGED: return "residue exceeded the divergence residue";
      case B2S_OOM: return "device out of memory";
      case B2S_CUDA_ERROR: return "CUDA error";
      case B2S_TIMEOUT: return "wait timed out";
      case B2S_INVALID_ARG: return "invalid argument";
      case B2S_INDEX_OVERFLOW: return "storage exceeds 32-bit indexing";
      case B2S_UNSUPPORTED: return "unsupported option";
      case B2S_BREAKDOWN: return "Krylov breakdown";
      case B2S_BUDGET: return "memory budget exceeded";
      case B2S_CANCELLED: return "request cancelled";
      case B2S_IO_ERROR: return "file i/o error";
   }
   return "unknown status";
}

const char*
b2s_last_error( void )
{
   return g_last_error.c_str();
}

int
b2s_abi_version( void )
{
   return B2S_ABI_VERSION;
}

b2s_status
b2s_dot( b2s_dtype dtype, int64_t n, const void* a, const void* b, double* result, b2s_stream stream )
{
   clear_error();
   B2S_CHECK_ARG( n >= 0 && result, "dot: n >= 0 and result required" );
   B2S_CHECK_ARG( n == 0 || ( a && b ), "dot: null vector" );
   if( dtype == B2S_F64 )
      return reduce_call< double, 0 >( n, a, b, result, as_stream( stream ) );
   if( dtype == B2S_F32 )
      return reduce_call< float, 0 >( n, a, b, result, as_stream( stream ) );
   set_error( "dot: bad dtype" );
   return B2S_INVALID_ARG;
}

b2s_status
b2s_norm2( b2s_dtype dtype, int64_t n, const void* a, double* result, b2s_stream stream )
{
   clear_error();
   B2S_CHECK_ARG( n >= 0 && result && ( n == 0 || a ), "norm2: bad arguments" );
   if( dtype == B2S_F64 )
      return reduce_call< double, 1 >( n, a, a, result, as_stream( stream ) );
   if( dtype == B2S_F32 )
      return reduce_call< float, 1 >( n, a, a, result, as_stream( stream ) );
   set_error( "norm2: bad dtype" );
   return B2S_INVALID_ARG;
}

b2s_status
b2s_axpby( b2s_dtype dtype, int64_t n, double alpha, const void* x, double beta, void* y, b2s_stream stream )
{
   clear_error();
   B2S_CHECK_ARG( n >= 0 && ( n == 0 || ( x && y ) ), "axpby: bad arguments" );
   if( n == 0 )
      return B2S_OK;
   const int grid = (int) std::min< int64_t >( ( n + 255 ) / 256, (int64_t) num_sms() * 16 );
   cudaStream_t s = as_stream( stream );
   if( dtype == B2S_F64 )
      axpby_kernel< double ><<< grid, 256, 0, s >>>( n, alpha, static_cast< const double* >( x ), beta,
                                                      static_cast< double* >( y ) );
   else if( dtype == B2S_F32 )
      axpby_kernel< float ><<< grid, 256, 0, s >>>( n, (float) alpha, static_cast< const float* >( x ), (float) beta,
                                                     static_cast< float* >( y ) );
   else {
      set_error( "axpby: bad dtype" );
      return B2S_INVALID_ARG;
   }
   B2S_TRY_CUDA( cudaGetLastError() );
   return B2S_OK;
}

b2s_status
b2s_gather( int32_t element_size, int64_t n, const void* src, int64_t src_size, const int32_t* idx, void* dest,
            b2s_stream stream )
{
   clear_error();
   B2S_CHECK_ARG( element_size == 4 || element_size == 8, "gather: element_size must be 4 or 8" );
   B2S_CHECK_ARG( n >= 0 && src_size >= 0 && ( n == 0 || ( src && idx && dest ) ), "gather: bad arguments" );
   if( n == 0 )
      return B2S_OK;
   const int grid = (int) std::min< int64_t >( ( n + 255 ) / 256, (int64_t) num_sms() * 16 );
   cudaStream_t s = as_stream( stream );
   if( element_size == 8 )
      gather_kernel< int64_t ><<< grid, 256, 0, s >>>( n, static_cast< const int64_t* >( src ), src_size, idx,
                                                       static_cast< int64_t* >( dest ) );
   else
      gather_kernel< int32_t ><<< grid, 256, 0, s >>>( n, static_cast< const int32_t* >( src ), src_size, idx,
                                                       static_cast< int32_t* >( dest ) );
   B2S_TRY_CUDA( cudaGetLastError() );
   return B2S_OK;
}

b2s_status
b2s_scan_i32( int64_t n, int32_t* data, int32_t inclusive, b2s_stream stream )
{
   clear_error();
   B2S_CHECK_ARG( n >= 0 && ( n == 0 || data ), "scan: bad arguments" );
   if( n == 0 )
      return B2S_OK;
   cudaStream_t s = as_stream( stream );
   DevBuf tmp, orig;
   B2S_TRY( tmp.alloc( n * sizeof( int64_t ) ) );
   const int grid = (int) std::min< int64_t >( ( n + 255 ) / 256, (int64_t) num_sms() * 16 );
   i32_to_i64_kernel<<< grid, 256, 0, s >>>( data, tmp.as< int64_t >(), n );
   B2S_TRY_CUDA( cudaGetLastError() );
   if( inclusive ) {
      B2S_TRY( orig.alloc( n * sizeof( int32_t ) ) );
      B2S_TRY_CUDA( cudaMemcpyAsync( orig.p, data, n * sizeof( int32_t ), cudaMemcpyDeviceToDevice, s ) );
   }
   B2S_TRY( scan_exclusive_i64( tmp.as< int64_t >(), n, s ) );
   i64_to_i32_kernel<<< grid, 256, 0, s >>>( tmp.as< int64_t >(), data, n,
                                              inclusive ? tmp.as< int64_t >() : nullptr, orig.as< int32_t >() );
   B2S_TRY_CUDA( cudaGetLastError() );
   B2S_TRY_CUDA( cudaStreamSynchronize( s ) );
   return B2S_OK;
}

}  // extern "C"
