// Serving loop: a device-resident request server for linear solves.
//
// Requests (a CSR matrix, a right-hand side and solver options, all in host
// memory) queue in arrival order. Each of `max_inflight` worker threads owns
// a slot: it admits the next request whose estimated device footprint fits
// in what is left of the memory budget, builds the matrix in HBM, runs the
// solve on its own streams, copies the solution back and releases the
// memory. Requests that arrive while others are on the GPU are admitted as
// soon as a slot and enough budget are free, and their kernels overlap with
// the running ones on the device (continuous batching).
//
// Admission: first-come first-served, except that a request that does not
// fit may be overtaken by later ones that do; after kMaxOvertakes overtakes
// nothing passes it any more (no starvation of large requests). A request
// larger than the whole budget fails at once with B2S_BUDGET.
//
// Device memory of admitted requests comes from a pool owned by the server,
// allocated and freed in stream order on the worker's stream, so one request
// setting up or tearing down never waits for the kernels of the others.
//
// Every result is the same, bit for bit, whether the request runs alone or
// among others: each solve has private vectors and reduction scratch, and
// every reduction has a fixed order.
//
// TNL has no serving layer; this is an addition on top of its solvers.
#include "b2s_internal.cuh"

#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

namespace b2s {

constexpr int kMaxOvertakes = 64;
constexpr int32_t kGraphRows = 1 << 18;
// Requests below this many rows run in plain FP64 even when they ask for mixed
// precision (their working set fits in L2, the FP32 path saves no bandwidth
// and its recurrences take more iterations).
constexpr int32_t kMixedMinRows = 1 << 19;

static int64_t
clock_ns()
{
   return std::chrono::duration_cast< std::chrono::nanoseconds >(
             std::chrono::steady_clock::now().time_since_epoch() )
      .count();
}

struct ServerReq
{
   int64_t ticket = 0;
   b2s_request r{};
   int64_t est_bytes = 0;
   int overtaken = 0;
   bool done = false;
   b2s_request_result res{};
   std::string msg;
};

// Device bytes a request holds at its peak: the matrix (CSR arrays, window
// tables, diagonal, FP32 copy for mixed precision, build temporaries), the
// solver's vectors, reduction scratch and, for GMRES, the Krylov basis.
static int64_t
estimate_bytes( const b2s_request& r )
{
   const int64_t n = r.rows, nnz = r.nnz;
   const bool mixed = r.opts.precision == B2S_PRECISION_MIXED;
   const int64_t pad = 512;
   int64_t m = 0;
   m += nnz * ( 8 + 4 ) + ( n + 1 ) * 4 + 2 * pad;      // values, columns, offsets
   m += ( nnz / kWinNnzF64 + nnz / kWinNnzF32 + 4 ) * 4;  // window tables
   m += n * 8 + 16 * pad;                                // diagonal, small buffers
   if( r.format != B2S_CSR )
      m += nnz * ( 8 + 4 ) + n * 16;                     // padded layout (CSR staging freed later)
   m += ( n + 1 ) * 4 + nnz * ( 4 + 8 ) + n * 4;          // build temporaries
   if( mixed )
      m += nnz * 4 + n * 4;                              // FP32 values and diagonal
   const int64_t ln = ( n + 63 ) / 64 * 64;
   const int64_t es = mixed ? 4 : 8;
   int64_t s = 10 * ln * es + ( mixed ? 2 * ln * 8 : 0 );
   s += (int64_t) 10 * 4 * kMaxReduceGrid * 8 + 64 * kMaxReduceGrid * 8 + 8 * pad;
   if( r.opts.solver == B2S_GMRES ) {
      const int64_t M = std::max( r.opts.gmres_restarting_max, 1 );
      s += ( M + 1 ) * ( ( n + 31 ) / 32 * 32 ) * es + ( ( M + 1 ) * M + 5 * ( M + 1 ) ) * 8;
   }
   if( r.opts.solver == B2S_BICGSTABL ) {
      const int64_t L = std::max( r.opts.bicgstab_ell, 1 );
      s += 2 * ( L + 1 ) * ( ( n + 31 ) / 32 * 32 ) * es + ( L * L + 4 * ( L + 1 ) ) * 8 + 64;
   }
   return m + s + ( 2 << 20 );
}

}  // namespace b2s

using namespace b2s;

struct b2s_server_t
{
   b2s_server_opts o{};
   int device = 0;
   cudaMemPool_t pool = nullptr;
   std::mutex mu;
   std::condition_variable cv_work, cv_done;
   std::deque< std::shared_ptr< ServerReq > > pending;
   std::map< int64_t, std::shared_ptr< ServerReq > > live;  // submitted, not yet collected
   int64_t next_ticket = 1;
   int64_t reserved = 0, peak_reserved = 0;
   int inflight = 0, peak_inflight = 0;
   int64_t completed = 0;
   bool stop = false;
   std::vector< std::thread > workers;

   void worker_main();
   bool pick( std::shared_ptr< ServerReq >& out );
   void run( ServerReq& q, cudaStream_t ws );
};

// Called with the lock held: the request to admit next, if any.
bool
b2s_server_t::pick( std::shared_ptr< ServerReq >& out )
{
   const int64_t free_bytes = o.memory_budget - reserved;
   for( size_t i = 0; i < pending.size(); i++ ) {
      auto& q = pending[ i ];
      if( q->est_bytes <= free_bytes ) {
         for( size_t j = 0; j < i; j++ )
            pending[ j ]->overtaken++;
         out = q;
         pending.erase( pending.begin() + (long) i );
         return true;
      }
      if( q->overtaken >= kMaxOvertakes )
         return false;  // the oldest waiting request must go next
   }
   return false;
}

void
b2s_server_t::run( ServerReq& q, cudaStream_t ws )
{
   const b2s_request& r = q.r;
   b2s_matrix A = nullptr;
   b2s_solver S = nullptr;
   b2s_matrix_opts mo;
   b2s_matrix_opts_default( &mo );
   mo.keep_fp32_copy = r.opts.precision == B2S_PRECISION_MIXED ? 1 : 0;
   b2s_status st = b2s_matrix_create( (b2s_format) r.format, B2S_F64, r.rows, r.rows, r.nnz, r.offsets, r.columns,
                                      r.values, B2S_F64, B2S_HOST, &mo, ws, &A );
   // a request's solver is used once: below kGraphRows rows, capturing and
   // instantiating its iteration graphs costs more than it saves
   b2s_solve_opts so = r.opts;
   if( r.rows < kGraphRows )
      so.graphs = 1;
   if( st == B2S_OK )
      st = b2s_solver_create( A, &so, &S );
   b2s_solve_report rep{};
   q.res.t_built_ns = clock_ns();
   if( st == B2S_OK )
      st = b2s_solve( S, r.b, r.x, B2S_HOST, ws, &rep );
   q.res.t_solved_ns = clock_ns();
   if( st != B2S_OK )
      q.msg = b2s_last_error();
   if( S )
      b2s_solver_destroy( S );
   if( A )
      b2s_matrix_destroy( A );
   cudaStreamSynchronize( ws );  // the frees of this request are ordered
   q.res.status = st;
   q.res.report = rep;
}

void
b2s_server_t::worker_main()
{
   cudaSetDevice( device );
   cudaStream_t ws = nullptr, ss = nullptr;
   cudaEvent_t e0 = nullptr, e1 = nullptr;
   cudaStreamCreateWithFlags( &ws, cudaStreamNonBlocking );
   cudaStreamCreateWithFlags( &ss, cudaStreamNonBlocking );
   cudaEventCreate( &e0 );
   cudaEventCreate( &e1 );
   AllocCtx ctx{ pool, ws, ss, e0, e1 };
   set_thread_alloc_ctx( &ctx );
   for( ;; ) {
      std::shared_ptr< ServerReq > q;
      {
         std::unique_lock< std::mutex > lk( mu );
         for( ;; ) {
            if( stop )
               break;
            if( pick( q ) )
               break;
            cv_work.wait( lk );
         }
         if( ! q )
            break;
         reserved += q->est_bytes;
         inflight++;
         peak_reserved = std::max( peak_reserved, reserved );
         peak_inflight = std::max( peak_inflight, inflight );
         q->res.t_admit_ns = clock_ns();
      }
      run( *q, ws );
      {
         std::lock_guard< std::mutex > lk( mu );
         q->res.t_done_ns = clock_ns();
         q->done = true;
         reserved -= q->est_bytes;
         inflight--;
         completed++;
      }
      cv_done.notify_all();
      cv_work.notify_all();
   }
   set_thread_alloc_ctx( nullptr );
   cudaStreamSynchronize( ws );
   cudaStreamSynchronize( ss );
   cudaEventDestroy( e0 );
   cudaEventDestroy( e1 );
   cudaStreamDestroy( ss );
   cudaStreamDestroy( ws );
}

extern "C" {

void
b2s_server_opts_default( b2s_server_opts* o )
{
   if( ! o )
      return;
   std::memset( o, 0, sizeof( *o ) );
   o->memory_budget = (int64_t) 150 * 1000 * 1000 * 1000;
   o->max_inflight = 8;
}

int64_t
b2s_server_clock_ns( void )
{
   return clock_ns();
}

b2s_status
b2s_server_create( const b2s_server_opts* opts, b2s_server* out )
{
   clear_error();
   B2S_CHECK_ARG( out, "NULL argument" );
   *out = nullptr;
   b2s_server_opts o;
   b2s_server_opts_default( &o );
   if( opts )
      o = *opts;
   B2S_CHECK_ARG( o.max_inflight >= 1 && o.max_inflight <= 256, "max_inflight in [1, 256]" );
   B2S_CHECK_ARG( o.memory_budget > 0, "memory_budget > 0" );
   std::unique_ptr< b2s_server_t > sv( new b2s_server_t() );
   B2S_TRY_CUDA( cudaGetDevice( &sv->device ) );
   size_t free_b = 0, total_b = 0;
   B2S_TRY_CUDA( cudaMemGetInfo( &free_b, &total_b ) );
   // never promise more than the device has free now, less a reserve for
   // the CUDA context and other users
   const int64_t cap = (int64_t) free_b - ( (int64_t) 2 << 30 );
   if( o.memory_budget > cap )
      o.memory_budget = std::max< int64_t >( cap, (int64_t) 64 << 20 );
   sv->o = o;
   cudaMemPoolProps props{};
   props.allocType = cudaMemAllocationTypePinned;
   props.location.type = cudaMemLocationTypeDevice;
   props.location.id = sv->device;
   B2S_TRY_CUDA( cudaMemPoolCreate( &sv->pool, &props ) );
   uint64_t keep = (uint64_t) o.memory_budget;  // freed memory stays in the pool up to the budget
   B2S_TRY_CUDA( cudaMemPoolSetAttribute( sv->pool, cudaMemPoolAttrReleaseThreshold, &keep ) );
   for( int i = 0; i < o.max_inflight; i++ )
      sv->workers.emplace_back( [ p = sv.get() ] { p->worker_main(); } );
   *out = sv.release();
   return B2S_OK;
}

b2s_status
b2s_server_submit( b2s_server sv, const b2s_request* req, int64_t* ticket )
{
   clear_error();
   B2S_CHECK_ARG( sv && req && ticket, "NULL argument" );
   B2S_CHECK_ARG( req->rows >= 0 && req->nnz >= 0, "rows / nnz" );
   B2S_CHECK_ARG( req->rows == 0 || ( req->offsets && req->b && req->x ), "NULL request arrays" );
   B2S_CHECK_ARG( req->nnz == 0 || ( req->columns && req->values ), "NULL request arrays" );
   B2S_CHECK_ARG( req->format >= B2S_CSR && req->format <= B2S_MULTIDIAGONAL, "format" );
   auto q = std::make_shared< ServerReq >();
   q->r = *req;
   const int32_t min_rows = sv->o.mixed_min_rows == 0 ? kMixedMinRows : sv->o.mixed_min_rows;
   if( q->r.opts.precision == B2S_PRECISION_MIXED && min_rows > 0 && q->r.rows < min_rows )
      q->r.opts.precision = B2S_PRECISION_PLAIN;  // same FP64 tolerance, fewer iterations
   q->res.precision = q->r.opts.precision;
   q->est_bytes = estimate_bytes( q->r );
   q->res.t_submit_ns = clock_ns();
   q->res.device_bytes = q->est_bytes;
   {
      std::lock_guard< std::mutex > lk( sv->mu );
      B2S_CHECK_ARG( ! sv->stop, "server is shutting down" );
      q->ticket = sv->next_ticket++;
      *ticket = q->ticket;
      sv->live[ q->ticket ] = q;
      if( q->est_bytes > sv->o.memory_budget ) {
         // can never be admitted
         q->res.status = B2S_BUDGET;
         q->res.t_admit_ns = q->res.t_done_ns = q->res.t_submit_ns;
         q->msg = "request needs more device memory than the server's whole budget";
         q->done = true;
         sv->completed++;
      }
      else
         sv->pending.push_back( q );
   }
   sv->cv_work.notify_one();
   sv->cv_done.notify_all();
   return B2S_OK;
}

b2s_status
b2s_server_wait( b2s_server sv, int64_t ticket, double timeout_seconds, b2s_request_result* out )
{
   clear_error();
   B2S_CHECK_ARG( sv && out, "NULL argument" );
   std::unique_lock< std::mutex > lk( sv->mu );
   auto it = sv->live.find( ticket );
   if( it == sv->live.end() ) {
      set_error( "unknown or already collected ticket %lld", (long long) ticket );
      return B2S_INVALID_ARG;
   }
   auto q = it->second;
   const auto until = std::chrono::steady_clock::now()
                    + std::chrono::duration_cast< std::chrono::steady_clock::duration >(
                         std::chrono::duration< double >( timeout_seconds < 0 ? 1e9 : timeout_seconds ) );
   while( ! q->done ) {
      if( sv->cv_done.wait_until( lk, until ) == std::cv_status::timeout && ! q->done ) {
         set_error( "request %lld not finished within %.3f s", (long long) ticket, timeout_seconds );
         return B2S_TIMEOUT;
      }
   }
   *out = q->res;
   sv->live.erase( it );
   if( q->res.status != B2S_OK && ! q->msg.empty() )
      set_error( "%s", q->msg.c_str() );
   return B2S_OK;
}

b2s_status
b2s_server_get_stats( b2s_server sv, b2s_server_stats* out )
{
   clear_error();
   B2S_CHECK_ARG( sv && out, "NULL argument" );
   std::lock_guard< std::mutex > lk( sv->mu );
   std::memset( out, 0, sizeof( *out ) );
   out->memory_budget = sv->o.memory_budget;
   out->reserved_bytes = sv->reserved;
   out->peak_reserved_bytes = sv->peak_reserved;
   out->pending = (int64_t) sv->pending.size();
   out->inflight = sv->inflight;
   out->peak_inflight = sv->peak_inflight;
   out->completed = sv->completed;
   return B2S_OK;
}

b2s_status
b2s_server_destroy( b2s_server sv )
{
   clear_error();
   if( ! sv )
      return B2S_OK;
   {
      std::lock_guard< std::mutex > lk( sv->mu );
      sv->stop = true;
      // requests never admitted are cancelled
      for( auto& q : sv->pending ) {
         q->res.status = B2S_CANCELLED;
         q->res.t_admit_ns = q->res.t_done_ns = clock_ns();
         q->done = true;
      }
      sv->pending.clear();
   }
   sv->cv_work.notify_all();
   for( auto& t : sv->workers )
      t.join();
   sv->cv_done.notify_all();
   if( sv->pool )
      cudaMemPoolDestroy( sv->pool );
   delete sv;
   return B2S_OK;
}

}  // extern "C"
