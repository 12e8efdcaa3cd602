// Matrix assembly on the device and MatrixMarket input/output.
//
// b2s_matrix_from_coo — TNL assembles a sparse matrix with
//   setRowCapacities( counts ) + setElement / addElement per element
//   (Matrices/SparseMatrix.hpp:284-304, SparseMatrixView.hpp:256-340):
// each row keeps its elements sorted by column; an element whose column is
// already in the row is merged (setElement: value = 0 * old + new, so the last
// write wins; addElement: value = old + new), in the order of the calls.
// Here the whole triplet list is assembled at once on the device:
//   1. key = row << colbits | column, payload = the triplet's position;
//   2. stable LSD radix sort of (key, position), 8 bits per pass (skipped when
//      the keys already come sorted) — equal keys keep their input order;
//   3. runs of equal keys merged in input order with TNL's arithmetic, one
//      thread per run; row counts of the merged elements -> CSR offsets;
//   4. the target layout built from that CSR with the triplet counts as row
//      capacities (TNL's capacity of a row is the number of calls for it, so
//      padded layouts keep the slots of merged duplicates as padding) and
//      explicit zeros kept (setElement stores zeros).
// CSR is the exception: TNL's CSR row would keep those unused slots with
// column -1, which its own CSR kernels then read as x[-1]; here CSR rows hold
// exactly the merged elements.
//
// b2s_mtx_read / b2s_matrix_read_mtx — Matrices/MatrixReader.hpp:21-359:
// the same header checks, the same tokenisation (split on ' ', empty tokens
// skipped, exactly three per element line, atoi / atof), symmetric files
// expanded into both triangles in TNL's order, the same errors. The file is
// parsed by several host threads over line-aligned chunks.
//
// b2s_matrix_write_mtx — Matrices/MatrixWriter.hpp:103-128: TNL's header,
// rows in order, elements in storage order, zero values skipped, the value
// printed with the stream's default six significant digits.
#include "b2s_internal.cuh"

#include <algorithm>
#include <cerrno>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

using namespace b2s;

namespace b2s {

// ---------------------------------------------------------------------------
// Stable LSD radix sort of 64-bit keys with an int32 payload.
constexpr int kRadixBlock = 512;
constexpr int kRadixWarps = kRadixBlock / 32;
constexpr int kRadixItems = 8;
constexpr int kRadixTile = kRadixBlock * kRadixItems;

// element e of tile t handled by warp w, item i, lane l: e = t*TILE + (w*ITEMS + i)*32 + l,
// so (w, i, l) order is input order inside the tile
__device__ __forceinline__ int64_t
radix_elem( int w, int i, int lane )
{
   return (int64_t) blockIdx.x * kRadixTile + ( w * kRadixItems + i ) * 32 + lane;
}

// counts[d * nblocks + b] = elements of tile b with digit d
__global__ void __launch_bounds__( kRadixBlock )
radix_hist_kernel( const uint64_t* __restrict__ keys, int64_t n, int shift, int64_t* __restrict__ counts )
{
   __shared__ int hist[ 256 ];
   for( int d = threadIdx.x; d < 256; d += kRadixBlock )
      hist[ d ] = 0;
   __syncthreads();
   const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
   for( int i = 0; i < kRadixItems; i++ ) {
      const int64_t e = radix_elem( w, i, lane );
      if( e < n )
         atomicAdd( &hist[ ( keys[ e ] >> shift ) & 255 ], 1 );
   }
   __syncthreads();
   for( int d = threadIdx.x; d < 256; d += kRadixBlock )
      counts[ (int64_t) d * gridDim.x + blockIdx.x ] = hist[ d ];
}

// stable scatter: position = offs[d][b] + elements of digit d in earlier warps
// of the tile + earlier items / lanes of this warp
__global__ void __launch_bounds__( kRadixBlock )
radix_scatter_kernel( const uint64_t* __restrict__ kin, const int32_t* __restrict__ vin, int64_t n, int shift,
                      const int64_t* __restrict__ offs, uint64_t* __restrict__ kout, int32_t* __restrict__ vout )
{
   __shared__ int whist[ kRadixWarps ][ 256 ];
   __shared__ int64_t base[ 256 ];
   for( int t = threadIdx.x; t < kRadixWarps * 256; t += kRadixBlock )
      ( &whist[ 0 ][ 0 ] )[ t ] = 0;
   for( int d = threadIdx.x; d < 256; d += kRadixBlock )
      base[ d ] = offs[ (int64_t) d * gridDim.x + blockIdx.x ];
   __syncthreads();
   const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
   uint64_t k[ kRadixItems ];
   int32_t v[ kRadixItems ];
   int dg[ kRadixItems ], lo[ kRadixItems ];
#pragma unroll
   for( int i = 0; i < kRadixItems; i++ ) {
      const int64_t e = radix_elem( w, i, lane );
      const bool in = e < n;
      k[ i ] = in ? kin[ e ] : 0;
      v[ i ] = in ? vin[ e ] : 0;
      dg[ i ] = in ? (int) ( ( k[ i ] >> shift ) & 255 ) : 256;  // 256: outside the array
      const unsigned peers = __match_any_sync( 0xffffffffu, dg[ i ] );
      const int rank = __popc( peers & ( ( 1u << lane ) - 1u ) );
      const int run = in ? whist[ w ][ dg[ i ] ] : 0;
      lo[ i ] = run + rank;
      __syncwarp();
      if( in && lane == __ffs( peers ) - 1 )
         whist[ w ][ dg[ i ] ] = run + __popc( peers );
      __syncwarp();
   }
   __syncthreads();
   // per digit: exclusive prefix over the warps of the tile
   for( int d = threadIdx.x; d < 256; d += kRadixBlock ) {
      int acc = 0;
      for( int ww = 0; ww < kRadixWarps; ww++ ) {
         const int t = whist[ ww ][ d ];
         whist[ ww ][ d ] = acc;
         acc += t;
      }
   }
   __syncthreads();
#pragma unroll
   for( int i = 0; i < kRadixItems; i++ ) {
      if( dg[ i ] < 256 ) {
         const int64_t pos = base[ dg[ i ] ] + whist[ w ][ dg[ i ] ] + lo[ i ];
         kout[ pos ] = k[ i ];
         vout[ pos ] = v[ i ];
      }
   }
}

__global__ void
sorted_check_kernel( const uint64_t* __restrict__ keys, int64_t n, int* unsorted )
{
   for( int64_t i = 1 + blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x )
      if( keys[ i ] < keys[ i - 1 ] ) {
         atomicExch( unsorted, 1 );
         return;
      }
}

static int
grid_of( int64_t n, int threads = 256 )
{
   const int64_t g = ( n + threads - 1 ) / threads;
   return (int) std::max< int64_t >( 1, std::min< int64_t >( g, (int64_t) num_sms() * 32 ) );
}

// Sorts keys[0, n) (with payload idx) stably on their low `bits` bits; the
// result is in *keys / *idx (the buffers may be swapped with the spares).
static b2s_status
radix_sort( DevBuf& keys, DevBuf& idx, DevBuf& keys2, DevBuf& idx2, int64_t n, int bits, cudaStream_t s )
{
   if( n <= 1 || bits <= 0 )
      return B2S_OK;
   DevBuf flag;
   B2S_TRY( flag.alloc( sizeof( int ) ) );
   B2S_TRY_CUDA( cudaMemsetAsync( flag.p, 0, sizeof( int ), s ) );
   sorted_check_kernel<<< grid_of( n ), 256, 0, s >>>( keys.as< uint64_t >(), n, flag.as< int >() );
   B2S_TRY_CUDA( cudaGetLastError() );
   int unsorted = 0;
   B2S_TRY( copy_d2h( &unsorted, flag.p, sizeof( int ), s ) );
   if( ! unsorted )
      return B2S_OK;
   const int64_t nb = ( n + kRadixTile - 1 ) / kRadixTile;
   if( nb > INT32_MAX / 2 ) {
      set_error( "radix sort: too many elements" );
      return B2S_INVALID_ARG;
   }
   DevBuf counts;
   B2S_TRY( counts.alloc( (size_t) nb * 256 * sizeof( int64_t ) ) );
   for( int shift = 0; shift < bits; shift += 8 ) {
      radix_hist_kernel<<< (unsigned) nb, kRadixBlock, 0, s >>>( keys.as< uint64_t >(), n, shift, counts.as< int64_t >() );
      B2S_TRY_CUDA( cudaGetLastError() );
      B2S_TRY( scan_exclusive_i64( counts.as< int64_t >(), nb * 256, s ) );
      radix_scatter_kernel<<< (unsigned) nb, kRadixBlock, 0, s >>>( keys.as< uint64_t >(), idx.as< int32_t >(), n, shift,
                                                                  counts.as< int64_t >(), keys2.as< uint64_t >(),
                                                                  idx2.as< int32_t >() );
      B2S_TRY_CUDA( cudaGetLastError() );
      std::swap( keys, keys2 );
      std::swap( idx, idx2 );
   }
   return B2S_OK;
}

// ---------------------------------------------------------------------------
// COO assembly kernels
__global__ void
coo_keys_kernel( int64_t n, const int32_t* __restrict__ ri, const int32_t* __restrict__ ci, int32_t rows, int32_t cols,
                 int cbits, uint64_t* __restrict__ keys, int32_t* __restrict__ idx, int* bad )
{
   for( int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x ) {
      const int32_t r = ri[ i ], c = ci[ i ];
      if( r < 0 || r >= rows || c < 0 || c >= cols ) {
         atomicExch( bad, 1 );
         keys[ i ] = 0;
      }
      else
         keys[ i ] = ( (uint64_t) r << cbits ) | (uint64_t) c;
      idx[ i ] = (int32_t) i;
   }
}

// head[k] = 1 where a run of equal keys starts; caps[row] counts every triplet
__global__ void
coo_heads_kernel( int64_t n, const uint64_t* __restrict__ keys, int cbits, int64_t* __restrict__ head,
                  int32_t* __restrict__ caps )
{
   for( int64_t k = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; k < n; k += (int64_t) gridDim.x * blockDim.x ) {
      head[ k ] = ( k == 0 || keys[ k ] != keys[ k - 1 ] ) ? 1 : 0;
      atomicAdd( &caps[ keys[ k ] >> cbits ], 1 );
   }
}

// one thread per run: the merged value in input order with TNL's arithmetic
template< typename Real, typename Tin >
__global__ void
coo_merge_kernel( int64_t n, const uint64_t* __restrict__ keys, const int32_t* __restrict__ idx,
                  const Tin* __restrict__ vals, const int64_t* __restrict__ uidx, int cbits, int add,
                  int32_t* __restrict__ out_col, Real* __restrict__ out_val, int32_t* __restrict__ row_count )
{
   const uint64_t cmask = ( cbits >= 64 ) ? ~0ull : ( ( 1ull << cbits ) - 1ull );
   for( int64_t k = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; k < n; k += (int64_t) gridDim.x * blockDim.x ) {
      const uint64_t key = keys[ k ];
      if( k > 0 && keys[ k - 1 ] == key )
         continue;  // not the head of its run
      Real v = (Real) vals[ idx[ k ] ];
      for( int64_t j = k + 1; j < n && keys[ j ] == key; j++ ) {
         const Real nv = (Real) vals[ idx[ j ] ];
         // addElement( row, col, value, multiplicator ): multiplicator * old + value
         v = add ? Real( 1 ) * v + nv : Real( 0 ) * v + nv;
      }
      const int64_t u = uidx[ k ];
      out_col[ u ] = (int32_t) ( key & cmask );
      out_val[ u ] = v;
      atomicAdd( &row_count[ key >> cbits ], 1 );
   }
}

// capacities given by the caller: each row's distinct columns must fit
__global__ void
caps_check_kernel( const int32_t* __restrict__ caps, const int32_t* __restrict__ used, int32_t rows,
                   int64_t* __restrict__ caps64, int* bad )
{
   for( int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i <= rows; i += (int64_t) gridDim.x * blockDim.x ) {
      if( i == rows ) {
         caps64[ i ] = 0;
         continue;
      }
      const int32_t c = caps[ i ];
      if( c < used[ i ] || c < 0 )
         atomicMin( bad, (int) i );
      caps64[ i ] = c;
   }
}

__global__ void
counts_to_i64_kernel( const int32_t* __restrict__ c, int32_t n, int64_t* __restrict__ out )
{
   for( int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i <= n; i += (int64_t) gridDim.x * blockDim.x )
      out[ i ] = i < n ? c[ i ] : 0;
}

__global__ void
i64_to_i32_kernel( const int64_t* __restrict__ in, int64_t n, int32_t* __restrict__ out )
{
   for( int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x )
      out[ i ] = (int32_t) in[ i ];
}

static int
bits_for( int64_t v )  // bits needed for values in [0, v)
{
   int b = 0;
   while( b < 63 && ( 1ll << b ) < v )
      b++;
   return b;
}

template< typename Real, typename Tin >
static b2s_status
assemble( b2s_format format, b2s_dtype dtype, int32_t rows, int32_t cols, int64_t n, const int32_t* ri,
          const int32_t* ci, const Tin* vals, int add, const int32_t* caps_user, const b2s_matrix_opts& o,
          cudaStream_t s, b2s_matrix* out )
{
   const int cbits = bits_for( cols ), rbits = bits_for( rows );
   DevBuf keys, idx, keys2, idx2, flag;
   B2S_TRY( keys.alloc( (size_t) std::max< int64_t >( n, 1 ) * sizeof( uint64_t ) ) );
   B2S_TRY( idx.alloc( (size_t) std::max< int64_t >( n, 1 ) * sizeof( int32_t ) ) );
   B2S_TRY( flag.alloc( sizeof( int ) ) );
   B2S_TRY_CUDA( cudaMemsetAsync( flag.p, 0, sizeof( int ), s ) );
   if( n > 0 ) {
      coo_keys_kernel<<< grid_of( n ), 256, 0, s >>>( n, ri, ci, rows, cols, cbits, keys.as< uint64_t >(),
                                                      idx.as< int32_t >(), flag.as< int >() );
      B2S_TRY_CUDA( cudaGetLastError() );
   }
   int bad = 0;
   B2S_TRY( copy_d2h( &bad, flag.p, sizeof( int ), s ) );
   if( bad ) {
      set_error( "triplet index outside the %d x %d matrix", rows, cols );
      return B2S_INVALID_ARG;
   }
   if( n > 1 ) {
      B2S_TRY( keys2.alloc( (size_t) n * sizeof( uint64_t ) ) );
      B2S_TRY( idx2.alloc( (size_t) n * sizeof( int32_t ) ) );
      B2S_TRY( radix_sort( keys, idx, keys2, idx2, n, rbits + cbits, s ) );
      keys2.release();
      idx2.release();
   }
   // runs -> unique positions; row capacities (triplet counts)
   DevBuf head, caps, rcount, off64, off;
   B2S_TRY( head.alloc( (size_t) std::max< int64_t >( n, 1 ) * sizeof( int64_t ) ) );
   B2S_TRY( caps.alloc( (size_t) std::max( rows, 1 ) * sizeof( int32_t ) ) );
   B2S_TRY( rcount.alloc( (size_t) std::max( rows, 1 ) * sizeof( int32_t ) ) );
   B2S_TRY_CUDA( cudaMemsetAsync( caps.p, 0, (size_t) std::max( rows, 1 ) * sizeof( int32_t ), s ) );
   B2S_TRY_CUDA( cudaMemsetAsync( rcount.p, 0, (size_t) std::max( rows, 1 ) * sizeof( int32_t ), s ) );
   int64_t nu = 0;
   if( n > 0 ) {
      coo_heads_kernel<<< grid_of( n ), 256, 0, s >>>( n, keys.as< uint64_t >(), cbits, head.as< int64_t >(),
                                                       caps.as< int32_t >() );
      B2S_TRY_CUDA( cudaGetLastError() );
      int64_t last_head = 0;
      B2S_TRY( copy_d2h( &last_head, head.as< int64_t >() + n - 1, sizeof( int64_t ), s ) );
      B2S_TRY( scan_exclusive_i64( head.as< int64_t >(), n, s ) );
      B2S_TRY( copy_d2h( &nu, head.as< int64_t >() + n - 1, sizeof( int64_t ), s ) );
      nu += last_head;
   }
   if( nu > INT32_MAX ) {
      set_error( "assembled matrix exceeds 32-bit indices" );
      return B2S_INDEX_OVERFLOW;
   }
   DevBuf ucol, uval;
   B2S_TRY( ucol.alloc( (size_t) std::max< int64_t >( nu, 1 ) * sizeof( int32_t ) ) );
   B2S_TRY( uval.alloc( (size_t) std::max< int64_t >( nu, 1 ) * sizeof( Real ) ) );
   if( n > 0 ) {
      coo_merge_kernel< Real, Tin ><<< grid_of( n ), 256, 0, s >>>( n, keys.as< uint64_t >(), idx.as< int32_t >(), vals,
                                                                    head.as< int64_t >(), cbits, add, ucol.as< int32_t >(),
                                                                    uval.as< Real >(), rcount.as< int32_t >() );
      B2S_TRY_CUDA( cudaGetLastError() );
   }
   keys.release();
   idx.release();
   head.release();
   B2S_TRY( off64.alloc( ( (size_t) rows + 1 ) * sizeof( int64_t ) ) );
   B2S_TRY( off.alloc( ( (size_t) rows + 1 ) * sizeof( int32_t ) ) );
   counts_to_i64_kernel<<< grid_of( (int64_t) rows + 1 ), 256, 0, s >>>( rcount.as< int32_t >(), rows,
                                                                          off64.as< int64_t >() );
   B2S_TRY_CUDA( cudaGetLastError() );
   B2S_TRY( scan_exclusive_i64( off64.as< int64_t >(), (int64_t) rows + 1, s ) );
   i64_to_i32_kernel<<< grid_of( (int64_t) rows + 1 ), 256, 0, s >>>( off64.as< int64_t >(), (int64_t) rows + 1,
                                                                      off.as< int32_t >() );
   B2S_TRY_CUDA( cudaGetLastError() );
   int64_t caps_total = n;
   const int32_t* caps_used = caps.as< int32_t >();
   if( caps_user ) {
      // setRowCapacities( caps ): check that every row's elements fit, sum the capacities
      DevBuf c64, badf;
      B2S_TRY( c64.alloc( ( (size_t) rows + 1 ) * sizeof( int64_t ) ) );
      B2S_TRY( badf.alloc( sizeof( int ) ) );
      const int none = INT32_MAX;
      B2S_TRY( copy_h2d( badf.p, &none, sizeof( int ), s ) );
      caps_check_kernel<<< grid_of( (int64_t) rows + 1 ), 256, 0, s >>>( caps_user, rcount.as< int32_t >(), rows,
                                                                         c64.as< int64_t >(), badf.as< int >() );
      B2S_TRY_CUDA( cudaGetLastError() );
      int badrow = INT32_MAX;
      B2S_TRY( copy_d2h( &badrow, badf.p, sizeof( int ), s ) );
      if( badrow != INT32_MAX ) {
         set_error( "The capacity of the sparse matrix row number %d was exceeded.", badrow );
         return B2S_INVALID_ARG;
      }
      B2S_TRY( scan_exclusive_i64( c64.as< int64_t >(), (int64_t) rows + 1, s ) );
      B2S_TRY( copy_d2h( &caps_total, c64.as< int64_t >() + rows, sizeof( int64_t ), s ) );
      caps_used = caps_user;
   }
   return matrix_from_assembled( format, dtype, rows, cols, nu, off.as< int32_t >(), ucol.as< int32_t >(), uval.p,
                                 caps_used, caps_total, o, s, out );
}

// ---------------------------------------------------------------------------
// MatrixMarket text parsing (host)

// TNL's String::split( ' ', SkipEmpty ) of one line
static int
split_spaces( const char* b, const char* e, const char** tb, const char** te, int maxt )
{
   int nt = 0;
   const char* p = b;
   while( p < e ) {
      while( p < e && *p == ' ' )
         p++;
      if( p >= e )
         break;
      const char* q = p;
      while( q < e && *q != ' ' )
         q++;
      if( nt < maxt ) {
         tb[ nt ] = p;
         te[ nt ] = q;
      }
      nt++;
      p = q;
   }
   return nt;
}

// atoi / atof of one token (the token is copied so conversion stops at its end)
static long
tok_atoi( const char* b, const char* e )
{
   char buf[ 64 ];
   const size_t len = std::min< size_t >( (size_t) ( e - b ), sizeof( buf ) - 1 );
   std::memcpy( buf, b, len );
   buf[ len ] = 0;
   return std::strtol( buf, nullptr, 10 );
}

static double
tok_atof( const char* b, const char* e )
{
   char small[ 128 ];
   const size_t len = (size_t) ( e - b );
   if( len < sizeof( small ) ) {
      std::memcpy( small, b, len );
      small[ len ] = 0;
      return std::strtod( small, nullptr );
   }
   std::string big( b, e );
   return std::strtod( big.c_str(), nullptr );
}

static bool
tok_eq( const char* b, const char* e, const char* lit )
{
   const size_t n = std::strlen( lit );
   return (size_t) ( e - b ) == n && std::memcmp( b, lit, n ) == 0;
}

struct MtxChunk
{
   std::vector< int32_t > r, c;
   std::vector< double > v;
   std::string error;
};

static void
parse_chunk( const char* b, const char* e, int32_t rows, int32_t cols, bool sym, MtxChunk& out )
{
   const char* p = b;
   while( p < e ) {
      const char* nl = static_cast< const char* >( std::memchr( p, '\n', (size_t) ( e - p ) ) );
      const char* le = nl ? nl : e;
      if( le > p && *p != '%' ) {
         const char *tb[ 3 ], *te[ 3 ];
         const int nt = split_spaces( p, le, tb, te, 3 );
         if( nt != 3 ) {
            out.error = "Wrong number of parameters in the matrix row at line:" + std::string( p, le );
            return;
         }
         const long row = tok_atoi( tb[ 0 ], te[ 0 ] ), col = tok_atoi( tb[ 1 ], te[ 1 ] );
         const double val = tok_atof( tb[ 2 ], te[ 2 ] );
         if( col > cols || row > rows ) {
            out.error = "There is an element at position " + std::to_string( row ) + ", " + std::to_string( col ) +
                        " out of the matrix dimensions " + std::to_string( rows ) + " x " + std::to_string( cols ) + ".";
            return;
         }
         if( row < 1 || col < 1 ) {
            out.error = "Row or column index below 1 at line:" + std::string( p, le );
            return;
         }
         out.r.push_back( (int32_t) row - 1 );
         out.c.push_back( (int32_t) col - 1 );
         out.v.push_back( val );
         if( sym && row != col ) {
            out.r.push_back( (int32_t) col - 1 );
            out.c.push_back( (int32_t) row - 1 );
            out.v.push_back( val );
         }
      }
      p = le + 1;
   }
}

static b2s_status
parse_mtx( const char* path, b2s_mtx& m, std::vector< int32_t >& R, std::vector< int32_t >& Cc, std::vector< double >& V )
{
   FILE* f = std::fopen( path, "rb" );
   if( ! f ) {
      set_error( "I am not able to open the file %s", path );
      return B2S_IO_ERROR;
   }
   std::string buf;
   {
      char tmp[ 1 << 16 ];
      size_t got;
      while( ( got = std::fread( tmp, 1, sizeof( tmp ), f ) ) > 0 )
         buf.append( tmp, got );
      std::fclose( f );
   }
   const char* p = buf.data();
   const char* end = p + buf.size();
   auto next_line = [ & ]( const char*& q, const char*& le ) -> bool
   {
      if( q >= end )
         return false;
      const char* nl = static_cast< const char* >( std::memchr( q, '\n', (size_t) ( end - q ) ) );
      le = nl ? nl : end;
      return true;
   };
   // header line: %%MatrixMarket matrix coordinate real general|symmetric
   const char* le = nullptr;
   if( ! next_line( p, le ) ) {
      set_error( "Unknown format of the source file. We expect line like this: %%%%MatrixMarket matrix coordinate real general" );
      return B2S_INVALID_ARG;
   }
   {
      const char *tb[ 8 ], *te[ 8 ];
      const int nt = split_spaces( p, le, tb, te, 8 );
      if( nt < 5 || ! tok_eq( tb[ 0 ], te[ 0 ], "%%MatrixMarket" ) ) {
         set_error( "Unknown format of the source file. We expect line like this: %%%%MatrixMarket matrix coordinate "
                    "real general" );
         return B2S_INVALID_ARG;
      }
      if( ! tok_eq( tb[ 1 ], te[ 1 ], "matrix" ) ) {
         set_error( "Keyword 'matrix' is expected in the header line: %s", std::string( p, le ).c_str() );
         return B2S_INVALID_ARG;
      }
      if( ! tok_eq( tb[ 2 ], te[ 2 ], "coordinates" ) && ! tok_eq( tb[ 2 ], te[ 2 ], "coordinate" ) ) {
         set_error( "Error: Only 'coordinates' format is supported now, not %s", std::string( tb[ 2 ], te[ 2 ] ).c_str() );
         return B2S_INVALID_ARG;
      }
      if( ! tok_eq( tb[ 3 ], te[ 3 ], "real" ) ) {
         set_error( "Only 'real' matrices are supported, not %s", std::string( tb[ 3 ], te[ 3 ] ).c_str() );
         return B2S_INVALID_ARG;
      }
      m.symmetric = 0;
      if( ! tok_eq( tb[ 4 ], te[ 4 ], "general" ) ) {
         if( tok_eq( tb[ 4 ], te[ 4 ], "symmetric" ) )
            m.symmetric = 1;
         else {
            set_error( "Only 'general' matrices are supported, not %s", std::string( tb[ 4 ], te[ 4 ] ).c_str() );
            return B2S_INVALID_ARG;
         }
      }
   }
   p = le + 1;
   // dimensions line: the first line that does not start with '%'
   for( ;; ) {
      if( ! next_line( p, le ) ) {
         set_error( "Wrong number of parameters in the matrix header - should be 3." );
         return B2S_INVALID_ARG;
      }
      if( le > p && *p == '%' ) {
         p = le + 1;
         continue;
      }
      const char *tb[ 3 ], *te[ 3 ];
      if( split_spaces( p, le, tb, te, 3 ) != 3 ) {
         set_error( "Wrong number of parameters in the matrix header - should be 3." );
         return B2S_INVALID_ARG;
      }
      const long rows = tok_atoi( tb[ 0 ], te[ 0 ] ), cols = tok_atoi( tb[ 1 ], te[ 1 ] );
      if( rows <= 0 || cols <= 0 ) {
         set_error( "Row or column index is negative." );
         return B2S_INVALID_ARG;
      }
      if( rows > INT32_MAX || cols > INT32_MAX ) {
         set_error( "matrix dimensions exceed 32-bit indices" );
         return B2S_INDEX_OVERFLOW;
      }
      m.rows = (int32_t) rows;
      m.cols = (int32_t) cols;
      p = le + 1;
      break;
   }
   // element lines, parsed in line-aligned chunks by several threads
   const int64_t rest = end > p ? end - p : 0;
   int nthreads = (int) std::min< int64_t >( std::max( 1u, std::thread::hardware_concurrency() ), 16 );
   if( rest < ( 1 << 20 ) )
      nthreads = 1;
   std::vector< const char* > cut( nthreads + 1 );
   cut[ 0 ] = p;
   cut[ nthreads ] = end > p ? end : p;
   for( int t = 1; t < nthreads; t++ ) {
      const char* q = p + rest * t / nthreads;
      q = std::max( q, cut[ t - 1 ] );
      const char* nl = q < end ? static_cast< const char* >( std::memchr( q, '\n', (size_t) ( end - q ) ) ) : nullptr;
      cut[ t ] = nl ? nl + 1 : end;
   }
   std::vector< MtxChunk > parts( nthreads );
   std::vector< std::thread > th;
   for( int t = 0; t < nthreads; t++ )
      th.emplace_back( [ &, t ] { parse_chunk( cut[ t ], cut[ t + 1 ], m.rows, m.cols, m.symmetric != 0, parts[ t ] ); } );
   for( auto& t : th )
      t.join();
   size_t total = 0;
   for( auto& c : parts ) {
      if( ! c.error.empty() ) {  // the first error in file order
         set_error( "%s", c.error.c_str() );
         return B2S_INVALID_ARG;
      }
      total += c.r.size();
   }
   if( total > (size_t) INT32_MAX ) {
      set_error( "more than 2^31 - 1 matrix elements" );
      return B2S_INDEX_OVERFLOW;
   }
   R.reserve( total );
   Cc.reserve( total );
   V.reserve( total );
   for( auto& c : parts ) {
      R.insert( R.end(), c.r.begin(), c.r.end() );
      Cc.insert( Cc.end(), c.c.begin(), c.c.end() );
      V.insert( V.end(), c.v.begin(), c.v.end() );
   }
   // TNL's row-length check: a row may not hold more elements than there are columns
   std::vector< int64_t > len( (size_t) m.rows, 0 );
   for( int32_t r : R )
      if( ++len[ r ] > m.cols ) {
         set_error( "There are more elements ( %lld ) than the matrix columns ( %d ) at the row %d.",
                    (long long) len[ r ], m.cols, r + 1 );
         return B2S_INVALID_ARG;
      }
   m.count = (int64_t) total;
   return B2S_OK;
}

}  // namespace b2s

extern "C" {

// (r, c) -> (max, min): the lower-triangle position of a SymmetricMatrix element
__global__ void
lower_swap_kernel( const int32_t* ri, const int32_t* ci, int64_t n, int32_t* ro, int32_t* co )
{
   for( int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x ) {
      const int32_t r = ri[ i ], c = ci[ i ];
      ro[ i ] = r < c ? c : r;
      co[ i ] = r < c ? r : c;
   }
}

// unit values for the triplets of a binary matrix
__global__ void
unit_values_kernel( float* v, int64_t n )
{
   for( int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x )
      v[ i ] = 1.0f;
}

b2s_status
b2s_matrix_from_coo( b2s_format format, b2s_dtype dtype, int32_t rows, int32_t cols, int64_t count,
                     const int32_t* row_indexes, const int32_t* column_indexes, const void* values,
                     b2s_dtype values_dtype, b2s_memory where, int32_t duplicates, const int32_t* row_capacities,
                     const b2s_matrix_opts* opts, b2s_stream stream, b2s_matrix* out )
{
   clear_error();
   B2S_CHECK_ARG( out, "out handle is NULL" );
   *out = nullptr;
   B2S_CHECK_ARG( format >= B2S_CSR && format <= B2S_MULTIDIAGONAL, "format" );
   B2S_CHECK_ARG( dtype == B2S_F64 || dtype == B2S_F32 || dtype == B2S_BOOL, "dtype" );
   B2S_CHECK_ARG( values_dtype == B2S_F64 || values_dtype == B2S_F32, "values_dtype" );
   B2S_CHECK_ARG( where == B2S_HOST || where == B2S_DEVICE, "where" );
   B2S_CHECK_ARG( duplicates == B2S_DUP_SET || duplicates == B2S_DUP_ADD, "duplicates" );
   B2S_CHECK_ARG( rows >= 0 && cols >= 0 && count >= 0, "negative size" );
   B2S_CHECK_ARG( count <= INT32_MAX, "more than 2^31 - 1 triplets" );
   B2S_CHECK_ARG( count == 0 || ( row_indexes && column_indexes && ( values || dtype == B2S_BOOL ) ),
                  "NULL triplet arrays" );
   b2s_matrix_opts o;
   b2s_matrix_opts_default( &o );
   if( opts )
      o = *opts;
   cudaStream_t s = as_stream( stream );
   if( format == B2S_MULTIDIAGONAL && ( dtype == B2S_BOOL || o.symmetric ) ) {
      set_error( "a Multidiagonal matrix holds FP64 or FP32 values of a general matrix" );
      return B2S_UNSUPPORTED;
   }
   if( dtype == B2S_BOOL ) {
      // binary matrix: setElement / addElement store the column whatever the
      // value (a binary row keeps no values, SparseMatrix.hpp:297-302), so the
      // triplets are assembled with unit values and only the columns are kept
      if( o.symmetric || o.keep_fp32_copy ) {
         set_error( "binary matrices are general matrices without an FP32 copy" );
         return B2S_UNSUPPORTED;
      }
      std::vector< float > host_ones;
      DevBuf dev_ones;
      const void* ones = nullptr;
      if( where == B2S_HOST ) {
         host_ones.assign( (size_t) std::max< int64_t >( count, 1 ), 1.0f );
         ones = host_ones.data();
      }
      else {
         B2S_TRY( dev_ones.alloc( (size_t) std::max< int64_t >( count, 1 ) * sizeof( float ) ) );
         unit_values_kernel<<< (int) std::min< int64_t >( ( std::max< int64_t >( count, 1 ) + 255 ) / 256,
                                                          (int64_t) num_sms() * 8 ),
                                256, 0, s >>>( dev_ones.as< float >(), std::max< int64_t >( count, 1 ) );
         B2S_TRY_CUDA( cudaGetLastError() );
         ones = dev_ones.p;
      }
      b2s_matrix m = nullptr;
      B2S_TRY( b2s_matrix_from_coo( format, B2S_F32, rows, cols, count, row_indexes, column_indexes, ones, B2S_F32,
                                    where, B2S_DUP_SET, row_capacities, &o, stream, &m ) );
      m->values.release();
      m->values32.release();
      m->diagonal.release();
      m->dtype = B2S_BOOL;
      *out = m;
      return B2S_OK;
   }
   const size_t vs = values_dtype == B2S_F64 ? 8 : 4;
   const int32_t* ri = row_indexes;
   const int32_t* ci = column_indexes;
   const void* vv = values;
   DevBuf dr, dc, dv, dcaps;
   const int32_t* caps = row_capacities;
   if( where == B2S_HOST && row_capacities && rows > 0 ) {
      B2S_TRY( dcaps.alloc( (size_t) rows * sizeof( int32_t ) ) );
      B2S_TRY( copy_h2d( dcaps.p, row_capacities, (size_t) rows * sizeof( int32_t ), s ) );
      caps = dcaps.as< int32_t >();
   }
   if( where == B2S_HOST && count > 0 ) {
      B2S_TRY( dr.alloc( (size_t) count * sizeof( int32_t ) ) );
      B2S_TRY( dc.alloc( (size_t) count * sizeof( int32_t ) ) );
      B2S_TRY( dv.alloc( (size_t) count * vs ) );
      B2S_TRY( copy_h2d( dr.p, row_indexes, (size_t) count * sizeof( int32_t ), s ) );
      B2S_TRY( copy_h2d( dc.p, column_indexes, (size_t) count * sizeof( int32_t ), s ) );
      B2S_TRY( copy_h2d( dv.p, values, (size_t) count * vs, s ) );
      ri = dr.as< int32_t >();
      ci = dc.as< int32_t >();
      vv = dv.p;
   }
   if( o.symmetric ) {
      // SymmetricMatrix::setElement / addElement store (i, j) with i < j at (j, i)
      // (SparseMatrixView.hpp:285-289)
      if( rows != cols ) {
         set_error( "SymmetricMatrix must be square" );
         return B2S_INVALID_ARG;
      }
      if( count > 0 ) {
         // host triplets were staged into dr / dc above and are swapped in place
         // (each element by its own thread); device triplets get new arrays
         if( where == B2S_DEVICE ) {
            B2S_TRY( dr.alloc( (size_t) count * sizeof( int32_t ) ) );
            B2S_TRY( dc.alloc( (size_t) count * sizeof( int32_t ) ) );
         }
         lower_swap_kernel<<< (int) std::min< int64_t >( ( count + 255 ) / 256, (int64_t) num_sms() * 8 ), 256, 0, s >>>(
            ri, ci, count, dr.as< int32_t >(), dc.as< int32_t >() );
         B2S_TRY_CUDA( cudaGetLastError() );
         ri = dr.as< int32_t >();
         ci = dc.as< int32_t >();
      }
   }
   const int add = duplicates == B2S_DUP_ADD;
   if( dtype == B2S_F64 )
      return values_dtype == B2S_F64 ? assemble< double, double >( format, dtype, rows, cols, count, ri, ci,
                                                                   (const double*) vv, add, caps, o, s, out )
                                     : assemble< double, float >( format, dtype, rows, cols, count, ri, ci,
                                                                  (const float*) vv, add, caps, o, s, out );
   return values_dtype == B2S_F64 ? assemble< float, double >( format, dtype, rows, cols, count, ri, ci,
                                                               (const double*) vv, add, caps, o, s, out )
                                  : assemble< float, float >( format, dtype, rows, cols, count, ri, ci,
                                                              (const float*) vv, add, caps, o, s, out );
}

b2s_status
b2s_mtx_read( const char* path, b2s_mtx** out )
{
   clear_error();
   B2S_CHECK_ARG( path && out, "NULL argument" );
   *out = nullptr;
   b2s_mtx m;
   std::memset( &m, 0, sizeof( m ) );
   std::vector< int32_t > R, Cc;
   std::vector< double > V;
   B2S_TRY( parse_mtx( path, m, R, Cc, V ) );
   std::unique_ptr< b2s_mtx, void ( * )( b2s_mtx* ) > res( static_cast< b2s_mtx* >( std::calloc( 1, sizeof( b2s_mtx ) ) ),
                                                          b2s_mtx_free );
   if( ! res ) {
      set_error( "host allocation failed" );
      return B2S_OOM;
   }
   *res = m;
   res->row_indexes = nullptr;
   res->column_indexes = nullptr;
   res->values = nullptr;
   const size_t n = (size_t) m.count;
   res->row_indexes = static_cast< int32_t* >( std::malloc( std::max< size_t >( n, 1 ) * sizeof( int32_t ) ) );
   res->column_indexes = static_cast< int32_t* >( std::malloc( std::max< size_t >( n, 1 ) * sizeof( int32_t ) ) );
   res->values = static_cast< double* >( std::malloc( std::max< size_t >( n, 1 ) * sizeof( double ) ) );
   if( ! res->row_indexes || ! res->column_indexes || ! res->values ) {
      set_error( "host allocation failed" );
      return B2S_OOM;
   }
   if( n ) {
      std::memcpy( res->row_indexes, R.data(), n * sizeof( int32_t ) );
      std::memcpy( res->column_indexes, Cc.data(), n * sizeof( int32_t ) );
      std::memcpy( res->values, V.data(), n * sizeof( double ) );
   }
   *out = res.release();
   return B2S_OK;
}

void
b2s_mtx_free( b2s_mtx* m )
{
   if( ! m )
      return;
   std::free( m->row_indexes );
   std::free( m->column_indexes );
   std::free( m->values );
   std::free( m );
}

b2s_status
b2s_matrix_read_mtx( const char* path, b2s_format format, b2s_dtype dtype, const b2s_matrix_opts* opts,
                     b2s_stream stream, b2s_matrix* out )
{
   clear_error();
   B2S_CHECK_ARG( path && out, "NULL argument" );
   *out = nullptr;
   b2s_mtx* m = nullptr;
   B2S_TRY( b2s_mtx_read( path, &m ) );
   const b2s_status st = b2s_matrix_from_coo( format, dtype, m->rows, m->cols, m->count, m->row_indexes,
                                              m->column_indexes, m->values, B2S_F64, B2S_HOST, B2S_DUP_SET, nullptr, opts,
                                              stream, out );
   b2s_mtx_free( m );
   return st;
}

b2s_status
b2s_matrix_write_mtx( b2s_matrix A, const char* path )
{
   clear_error();
   B2S_NO_BINARY( A, "MatrixMarket output" );
   B2S_CHECK_ARG( A && path, "NULL argument" );
   if( A->symmetric ) {
      set_error( "MatrixWriter::writeMtx is not provided for SymmetricMatrix (lower-triangle) storage" );
      return B2S_UNSUPPORTED;
   }
   // the rows in storage order without padding; zero values are kept for the
   // header's count and skipped when printed, as TNL's writer does
   cudaStream_t s = nullptr;
   DevBuf doff, dcol, dval;
   int64_t nnz = 0;
   B2S_TRY( layout_to_csr( A, false, doff, dcol, dval, nnz, s ) );
   const int32_t rows = A->rows;
   std::vector< int32_t > off( (size_t) rows + 1 ), col( (size_t) std::max< int64_t >( nnz, 1 ) );
   std::vector< double > val( (size_t) std::max< int64_t >( nnz, 1 ) );
   B2S_TRY( copy_d2h( off.data(), doff.p, off.size() * sizeof( int32_t ), s ) );
   if( nnz > 0 ) {
      B2S_TRY( copy_d2h( col.data(), dcol.p, (size_t) nnz * sizeof( int32_t ), s ) );
      if( A->dtype == B2S_F64 )
         B2S_TRY( copy_d2h( val.data(), dval.p, (size_t) nnz * sizeof( double ), s ) );
      else {
         std::vector< float > valf( (size_t) nnz );
         B2S_TRY( copy_d2h( valf.data(), dval.p, (size_t) nnz * sizeof( float ), s ) );
         for( int64_t k = 0; k < nnz; k++ )
            val[ k ] = valf[ k ];
      }
   }
   // getNonzeroElementsCount(): stored elements that are not padding
   // (SparseMatrixView.hpp:184-194), explicit zeros included
   const int64_t nonzeros = nnz;
   FILE* f = std::fopen( path, "wb" );
   if( ! f ) {
      set_error( "cannot open %s for writing", path );
      return B2S_IO_ERROR;
   }
   std::string out;
   out.reserve( 1 << 20 );
   char line[ 128 ];
   out += "%%MatrixMarket matrix coordinate real general\n%%\n%% This file was generated by TNL (www.tnl-project.org)\n";
   // "%%" << setw( 9 ) << " ROWS " << setw( 9 ) << " COLUMNS " << setw( 12 ) << " ELEMENTS "
   std::snprintf( line, sizeof( line ), "%%%%%9s%9s%12s\n", " ROWS ", " COLUMNS ", " ELEMENTS " );
   out += line;
   std::snprintf( line, sizeof( line ), "%9d %9d %12lld\n", rows, A->cols, (long long) nonzeros );
   out += line;
   bool ok = true;
   for( int32_t r = 0; r < rows && ok; r++ ) {
      for( int32_t k = off[ r ]; k < off[ r + 1 ]; k++ ) {
         if( val[ k ] == 0.0 )
            continue;
         // ostream << value: %g with six significant digits (the float itself for FP32 matrices)
         std::snprintf( line, sizeof( line ), "%9d%9d%12g\n", r + 1, col[ k ] + 1, val[ k ] );
         out += line;
      }
      if( out.size() > ( 1u << 20 ) ) {
         ok = std::fwrite( out.data(), 1, out.size(), f ) == out.size();
         out.clear();
      }
   }
   if( ok && ! out.empty() )
      ok = std::fwrite( out.data(), 1, out.size(), f ) == out.size();
   ok = ( std::fclose( f ) == 0 ) && ok;
   if( ! ok ) {
      set_error( "write to %s failed", path );
      return B2S_IO_ERROR;
   }
   return B2S_OK;
}

}  // extern "C"
