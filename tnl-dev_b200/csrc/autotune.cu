// Autotuner of the SpMV layout: builds the matrix in every candidate segment
// layout / CSR kernel / threads-per-row / slice size, times vectorProduct on
// the device, and reports the fastest. TNL picks the layout at compile time
// (the Segments template argument of SparseMatrix); this is the run-time
// counterpart of that choice.
//
// Candidates (each skipped when its allocated slots exceed
// `max_storage_ratio` x nnz or 32-bit indexing):
//   CSR adaptive (32-row groups where they fit, and warp windows), CSR vector with 1..32 threads per row
//   (up to 4x the mean row length), Ellpack, SlicedEllpack with slice
//   8 / 16 / 32 / 64, ChunkedEllpack, BiEllpack.
// Timing: `reps` products after two warm-ups, CUDA events on the caller's
// stream around each product; before each one (outside the events) a 256 MiB
// write and a 256 MiB read evict L2, so every candidate pays for its own HBM
// traffic (back-to-back products, warm_l2 = 1, let a matrix not much larger
// than L2 run partly from it: 7 TB/s "measured" on a 217 MB matrix).
#include "b2s_internal.cuh"

#include <algorithm>
#include <cstring>
#include <vector>

using namespace b2s;

namespace b2s {

struct TuneCand
{
   int32_t format, csr_kernel, tpr, slice, groups;
};

// L2 eviction between timed products: write one buffer larger than L2, then
// read another, so that the write's dirty lines are back in HBM too
constexpr int64_t kFlushFloats = ( 256ll << 20 ) / 4;

__global__ void
tune_flush_kernel( float* __restrict__ w, const float* __restrict__ r, int64_t n, float* sink )
{
   float acc = 0;
   for( int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x ) {
      w[ i ] = 1.0f;
      acc += r[ i ];
   }
   if( acc == 12345.0f )
      *sink = acc;
}

struct L2Flush
{
   DevBuf w, r;
   b2s_status
   init( cudaStream_t s )
   {
      B2S_TRY( w.alloc( (size_t) kFlushFloats * 4 + 16 ) );
      B2S_TRY( r.alloc( (size_t) kFlushFloats * 4 ) );
      B2S_TRY_CUDA( cudaMemsetAsync( r.p, 0, (size_t) kFlushFloats * 4, s ) );
      return B2S_OK;
   }
   void
   run( cudaStream_t s ) const
   {
      tune_flush_kernel<<< num_sms() * 8, 256, 0, s >>>( w.as< float >(), r.as< float >(), kFlushFloats,
                                                          w.as< float >() + kFlushFloats );
   }
};

static b2s_status
time_candidate( b2s_matrix src, const TuneCand& c, b2s_dtype dtype, int reps, double max_ratio, const L2Flush* flush,
                cudaStream_t s, double& us, int64_t& storage, int32_t& groups_ran, bool& skipped )
{
   skipped = false;
   groups_ran = c.groups;
   b2s_matrix_opts mo;
   b2s_matrix_opts_default( &mo );
   mo.csr_kernel = c.csr_kernel;
   mo.threads_per_row = c.tpr;
   mo.slice_size = c.slice;
   mo.csr_row_groups = c.groups;
   b2s_matrix m = nullptr;
   b2s_status st = b2s_matrix_convert( src, (b2s_format) c.format, dtype, &mo, s, &m );
   // a pattern with more diagonals than a Multidiagonal matrix holds is no candidate
   if( st == B2S_INDEX_OVERFLOW || st == B2S_OOM || ( st == B2S_UNSUPPORTED && c.format == B2S_MULTIDIAGONAL ) ) {
      cudaGetLastError();
      skipped = true;
      return B2S_OK;
   }
   if( st != B2S_OK )
      return st;
   b2s_matrix_info info;
   b2s_matrix_get_info( m, &info );
   storage = info.storage_size;
   if( info.csr_path != 0 )
      groups_ran = info.csr_path == 1 ? 0 : -1;  // the CSR adaptive kernel that was built
   // the slots the layout holds on the device (BiEllpack allocates only those
   // it addresses, not TNL's nominal 32 x groupPointers[last])
   if( info.nnz > 0 && (double) m->alloc_elems > max_ratio * (double) info.nnz ) {
      b2s_matrix_destroy( m );
      skipped = true;
      return B2S_OK;
   }
   const size_t es = dtype == B2S_F64 ? 8 : 4;
   DevBuf x, y;
   st = x.alloc( (size_t) std::max( info.cols, 1 ) * es );
   if( st == B2S_OK )
      st = y.alloc( (size_t) std::max( info.rows, 1 ) * es );
   if( st != B2S_OK ) {
      b2s_matrix_destroy( m );
      return st;
   }
   // x = 1 (TNL's SpMV benchmark input), y = 0
   if( info.cols > 0 ) {
      std::vector< double > h( (size_t) info.cols, 1.0 );
      std::vector< float > hf( (size_t) info.cols, 1.0f );
      B2S_TRY( copy_h2d( x.p, dtype == B2S_F64 ? (const void*) h.data() : (const void*) hf.data(),
                         (size_t) info.cols * es, s ) );
   }
   std::vector< cudaEvent_t > ev( 2 * (size_t) std::max( reps, 1 ), nullptr );
   for( auto& e : ev )
      B2S_TRY_CUDA( cudaEventCreate( &e ) );
   for( int i = 0; i < 2 && st == B2S_OK; i++ )
      st = b2s_spmv( m, x.p, y.p, 1.0, 0.0, 0, 0, B2S_DEVICE, s );
   for( int i = 0; i < reps && st == B2S_OK; i++ ) {
      // cold: L2 evicted before each product; warm: events around the whole run
      if( flush )
         flush->run( s );
      if( flush || i == 0 )
         cudaEventRecord( ev[ 2 * i ], s );
      st = b2s_spmv( m, x.p, y.p, 1.0, 0.0, 0, 0, B2S_DEVICE, s );
      if( flush || i == reps - 1 )
         cudaEventRecord( ev[ flush ? 2 * i + 1 : 1 ], s );
   }
   if( st == B2S_OK ) {
      cudaError_t e = cudaStreamSynchronize( s );
      if( e != cudaSuccess ) {
         set_error( "autotune: %s", cudaGetErrorString( e ) );
         st = B2S_CUDA_ERROR;
      }
   }
   double total = 0;
   if( st == B2S_OK ) {
      for( int i = 0; i < ( flush ? reps : 1 ); i++ ) {
         float ms = 0;
         cudaEventElapsedTime( &ms, ev[ 2 * i ], ev[ 2 * i + 1 ] );
         total += ms;
      }
   }
   for( auto& e : ev )
      cudaEventDestroy( e );
   b2s_matrix_destroy( m );
   us = 1e3 * total / std::max( reps, 1 );
   return st;
}

}  // namespace b2s

extern "C" {

void
b2s_tune_opts_default( b2s_tune_opts* o )
{
   if( ! o )
      return;
   std::memset( o, 0, sizeof( *o ) );
   o->reps = 10;
   o->max_storage_ratio = 3.0;
}

b2s_status
b2s_autotune_spmv( b2s_matrix src, b2s_dtype dtype, const b2s_tune_opts* opts, b2s_stream stream, b2s_tune_result* best,
                   b2s_tune_entry* table, int32_t capacity, int32_t* count )
{
   clear_error();
   B2S_NO_BINARY( src, "the autotuner" );
   B2S_CHECK_ARG( src && best, "NULL argument" );
   B2S_CHECK_ARG( src->format == B2S_CSR, "the autotuner starts from a CSR matrix" );
   B2S_CHECK_ARG( dtype == B2S_F64 || dtype == B2S_F32, "dtype" );
   b2s_tune_opts o;
   b2s_tune_opts_default( &o );
   if( opts )
      o = *opts;
   if( o.reps < 1 )
      o.reps = 1;
   if( o.max_storage_ratio <= 0 )
      o.max_storage_ratio = 3.0;
   cudaStream_t s = as_stream( stream );
   L2Flush flush;
   if( ! o.warm_l2 )
      B2S_TRY( flush.init( s ) );
   std::vector< TuneCand > cands;
   cands.push_back( { B2S_CSR, B2S_CSR_ADAPTIVE, 0, 0, 0 } );
   if( src->csr_group )  // the nnz-window kernel as well
      cands.push_back( { B2S_CSR, B2S_CSR_ADAPTIVE, 0, 0, -1 } );
   for( int t = 1; t <= 32; t *= 2 )
      if( t == 1 || t <= 4.0 * src->mean_row )
         cands.push_back( { B2S_CSR, B2S_CSR_VECTOR, t, 0, 0 } );
   cands.push_back( { B2S_ELLPACK, 0, 0, 0, 0 } );
   for( int ss : { 8, 16, 32, 64 } )
      cands.push_back( { B2S_SLICED_ELLPACK, 0, 0, ss, 0 } );
   cands.push_back( { B2S_CHUNKED_ELLPACK, 0, 0, 0, 0 } );
   cands.push_back( { B2S_BIELLPACK, 0, 0, 0, 0 } );
   cands.push_back( { B2S_MULTIDIAGONAL, 0, 0, 0, 0 } );
   std::memset( best, 0, sizeof( *best ) );
   best->spmv_us = 1e300;
   int32_t n_out = 0, timed = 0;
   for( const auto& c : cands ) {
      double us = 0;
      int64_t storage = 0;
      bool skipped = false;
      int32_t groups_ran = c.groups;
      B2S_TRY( time_candidate( src, c, dtype, o.reps, o.max_storage_ratio, o.warm_l2 ? nullptr : &flush, s, us, storage,
                               groups_ran, skipped ) );
      if( table && n_out < capacity ) {
         b2s_tune_entry& e = table[ n_out ];
         std::memset( &e, 0, sizeof( e ) );
         e.format = c.format;
         e.csr_kernel = c.csr_kernel;
         e.threads_per_row = c.tpr;
         e.slice_size = c.slice == 0 && c.format == B2S_SLICED_ELLPACK ? b2s::kSliceSize : c.slice;
         e.skipped = skipped ? 1 : 0;
         e.csr_row_groups = groups_ran;
         e.storage_size = storage;
         e.spmv_us = skipped ? -1.0 : us;
      }
      n_out++;
      if( skipped )
         continue;
      timed++;
      if( us < best->spmv_us ) {
         best->format = c.format;
         best->csr_kernel = c.csr_kernel;
         best->threads_per_row = c.tpr;
         best->slice_size = c.slice;
         best->csr_row_groups = groups_ran;
         best->spmv_us = us;
      }
   }
   best->candidates = timed;
   if( count )
      *count = n_out;
   if( timed == 0 ) {
      set_error( "autotune: no candidate layout could be built" );
      return B2S_UNSUPPORTED;
   }
   return B2S_OK;
}

}  // extern "C"
