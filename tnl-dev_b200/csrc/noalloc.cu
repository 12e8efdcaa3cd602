// Allocation-free variant of the device-wide int32 prefix sum (b2s_scan_i32).
//
// b2s_scan_i32 obtains its working memory (an int64 copy of the data and the
// per-tile totals) from cudaMalloc on every call. Some callers cannot allow
// that: an application that hands out every byte of device memory through its
// own pool allocator or runs under a fixed memory budget (a cudaMalloc beside
// the pool can fail, or fragment the memory the pool expects to own), and
// latency-critical host code that cannot afford the device-wide
// synchronization that cudaFree implies. b2s_scan_i32_noalloc serves them: its
// only working memory is the file-scope array below, which every GPU that
// loads the library holds until the process exits.
//
// Limits and sharing rules:
//  * at most kNoAllocScanMax = kNoAllocTiles * 2048 = 67,108,864 elements per
//    call; larger inputs are rejected with B2S_INVALID_ARG;
//  * all calls on a device share the array and it keeps the previous call's
//    contents. Nothing in it has to start at zero: every slot a call reads was
//    written earlier in that same call. Calls that overlap on the GPU (on two
//    streams, or from two host threads without ordering) race on the array;
//  * the first call on each device looks up the array's device address
//    (cudaGetSymbolAddress, with that device current) and caches it together
//    with the ID of the CUDA context it belongs to. A later call in another
//    context of that device (after cudaDeviceReset the library's kernels and
//    this array are loaded again, possibly elsewhere) looks the address up
//    anew. Make the first call on a device, and the first one after a
//    cudaDeviceReset, before any stream capture begins;
//  * the call is asynchronous on `stream`, as a kernel launch is: it returns
//    once its three kernels are queued. Synchronize with the stream before
//    reading `data` on the host, and before starting a call on another stream.
#include "b2s_internal.cuh"

#include <cuda.h>  // context types only; the two driver calls are reached through the runtime

#include <mutex>

namespace b2s {

constexpr int kNaThreads = 512;
constexpr int kNaItems = 4;
constexpr int kNaTile = kNaThreads * kNaItems;  // 2048 elements per tile
constexpr int kNoAllocTiles = 32768;
constexpr int64_t kNoAllocScanMax = (int64_t) kNoAllocTiles * kNaTile;

// Working memory of b2s_scan_i32_noalloc: one int64 total per tile.
static __device__ __align__( 256 ) int64_t g_noalloc_scan_tiles[ kNoAllocTiles ];

// Host-side cache of the array's device address, per device, tagged with the
// context it was looked up in.
struct NaEntry
{
   int64_t* ptr = nullptr;
   unsigned long long ctx = 0;
};
static std::mutex g_na_mutex;
static NaEntry g_na[ 64 ];

using CtxGetCurrentFn = CUresult ( * )( CUcontext* );
using CtxGetIdFn = CUresult ( * )( CUcontext, unsigned long long* );

// Process-unique ID of the calling thread's current context (cuCtxGetId), or 0
// when no context is current or the driver cannot tell.
static unsigned long long
current_context_id()
{
   static CtxGetCurrentFn get_current = nullptr;
   static CtxGetIdFn get_id = nullptr;
   static std::once_flag once;
   std::call_once( once,
                   []
                   {
                      cudaDriverEntryPointQueryResult q1 = cudaDriverEntryPointSymbolNotFound, q2 = q1;
                      void *f1 = nullptr, *f2 = nullptr;
                      if( cudaGetDriverEntryPoint( "cuCtxGetCurrent", &f1, cudaEnableDefault, &q1 ) == cudaSuccess
                          && cudaGetDriverEntryPoint( "cuCtxGetId", &f2, cudaEnableDefault, &q2 ) == cudaSuccess
                          && q1 == cudaDriverEntryPointSuccess && q2 == cudaDriverEntryPointSuccess ) {
                         get_current = reinterpret_cast< CtxGetCurrentFn >( f1 );
                         get_id = reinterpret_cast< CtxGetIdFn >( f2 );
                      }
                      cudaGetLastError();
                   } );
   if( ! get_current || ! get_id )
      return 0;
   CUcontext c = nullptr;
   unsigned long long id = 0;
   if( get_current( &c ) != CUDA_SUCCESS || c == nullptr || get_id( c, &id ) != CUDA_SUCCESS )
      return 0;
   return id;
}

static b2s_status
noalloc_scratch( int64_t** out )
{
   int dev = 0;
   B2S_TRY_CUDA( cudaGetDevice( &dev ) );
   if( dev < 0 || dev >= 64 ) {
      set_error( "scan_noalloc: device ordinal %d not supported", dev );
      return B2S_INVALID_ARG;
   }
   std::lock_guard< std::mutex > lock( g_na_mutex );
   NaEntry& e = g_na[ dev ];
   const unsigned long long ctx = current_context_id();
   if( ! e.ptr || ctx == 0 || ctx != e.ctx ) {
      // host code only sees a stand-in for the array: ask the runtime for the
      // address the kernels of this device (in its current context) must use
      void* p = nullptr;
      B2S_TRY_CUDA( cudaGetSymbolAddress( &p, g_noalloc_scan_tiles ) );
      e.ptr = static_cast< int64_t* >( p );
      e.ctx = current_context_id();
   }
   *out = e.ptr;
   return B2S_OK;
}

// Inclusive block scan of one int64 per thread; returns the block total too.
__device__ __forceinline__ int64_t
na_block_inclusive( int64_t v, int64_t& total )
{
   __shared__ int64_t warp_tot[ kNaThreads / 32 ];
   const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
   for( int o = 1; o < 32; o <<= 1 ) {
      const int64_t t = __shfl_up_sync( 0xffffffffu, v, o );
      if( lane >= o )
         v += t;
   }
   if( lane == 31 )
      warp_tot[ warp ] = v;
   __syncthreads();
   if( warp == 0 ) {
      int64_t w = lane < kNaThreads / 32 ? warp_tot[ lane ] : 0;
#pragma unroll
      for( int o = 1; o < 32; o <<= 1 ) {
         const int64_t t = __shfl_up_sync( 0xffffffffu, w, o );
         if( lane >= o )
            w += t;
      }
      if( lane < kNaThreads / 32 )
         warp_tot[ lane ] = w;
   }
   __syncthreads();
   const int64_t r = v + ( warp > 0 ? warp_tot[ warp - 1 ] : 0 );
   total = warp_tot[ kNaThreads / 32 - 1 ];
   __syncthreads();
   return r;
}

// 1. total of every tile
__global__ void __launch_bounds__( kNaThreads )
na_tile_totals_kernel( const int32_t* __restrict__ data, int64_t n, int64_t* tiles )
{
   const int64_t base = (int64_t) blockIdx.x * kNaTile + (int64_t) threadIdx.x * kNaItems;
   int64_t s = 0;
#pragma unroll
   for( int i = 0; i < kNaItems; i++ )
      if( base + i < n )
         s += data[ base + i ];
   int64_t total;
   na_block_inclusive( s, total );
   if( threadIdx.x == 0 )
      tiles[ blockIdx.x ] = total;
}

// 2. exclusive scan of the tile totals in place (one block)
__global__ void __launch_bounds__( kNaThreads )
na_scan_tiles_kernel( int64_t* tiles, int ntiles )
{
   const int per = ( ntiles + kNaThreads - 1 ) / kNaThreads;
   const int b = threadIdx.x * per;
   int64_t s = 0;
   for( int i = b; i < b + per && i < ntiles; i++ )
      s += tiles[ i ];
   int64_t total;
   const int64_t inc = na_block_inclusive( s, total );
   int64_t run = inc - s;
   for( int i = b; i < b + per && i < ntiles; i++ ) {
      const int64_t v = tiles[ i ];
      tiles[ i ] = run;
      run += v;
   }
}

// 3. scan inside every tile plus the tile's offset
__global__ void __launch_bounds__( kNaThreads )
na_tile_scan_kernel( int32_t* data, int64_t n, const int64_t* __restrict__ tiles, int inclusive )
{
   const int64_t base = (int64_t) blockIdx.x * kNaTile + (int64_t) threadIdx.x * kNaItems;
   int64_t v[ kNaItems ];
   int64_t s = 0;
#pragma unroll
   for( int i = 0; i < kNaItems; i++ ) {
      v[ i ] = base + i < n ? data[ base + i ] : 0;
      s += v[ i ];
   }
   int64_t total;
   const int64_t inc = na_block_inclusive( s, total );
   int64_t run = tiles[ blockIdx.x ] + inc - s;
#pragma unroll
   for( int i = 0; i < kNaItems; i++ ) {
      if( inclusive )
         run += v[ i ];
      if( base + i < n )
         data[ base + i ] = (int32_t) run;
      if( ! inclusive )
         run += v[ i ];
   }
}

}  // namespace b2s

using namespace b2s;

extern "C" b2s_status
b2s_scan_i32_noalloc( int64_t n, int32_t* data, int32_t inclusive, b2s_stream stream )
{
   clear_error();
   B2S_CHECK_ARG( n >= 0 && ( n == 0 || data ), "scan_noalloc: bad arguments" );
   if( n > kNoAllocScanMax ) {
      set_error( "scan_noalloc: n = %lld exceeds the fixed working array (at most %lld elements)", (long long) n,
                 (long long) kNoAllocScanMax );
      return B2S_INVALID_ARG;
   }
   int64_t* tiles = nullptr;
   B2S_TRY( noalloc_scratch( &tiles ) );
   if( n == 0 )
      return B2S_OK;
   cudaStream_t s = as_stream( stream );
   const int ntiles = (int) ( ( n + kNaTile - 1 ) / kNaTile );
   na_tile_totals_kernel<<< ntiles, kNaThreads, 0, s >>>( data, n, tiles );
   B2S_TRY_CUDA( cudaGetLastError() );
   na_scan_tiles_kernel<<< 1, kNaThreads, 0, s >>>( tiles, ntiles );
   B2S_TRY_CUDA( cudaGetLastError() );
   na_tile_scan_kernel<<< ntiles, kNaThreads, 0, s >>>( data, n, tiles, inclusive ? 1 : 0 );
   B2S_TRY_CUDA( cudaGetLastError() );
   return B2S_OK;
}
