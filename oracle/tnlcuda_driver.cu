// COMPARISON LEG ONLY — the reference timed beside the product, never the product.
//
// TNL's own Devices::Cuda path, compiled here for sm_100a from the unmodified
// reference headers (header-only library) and exposed behind a flat C ABI so
// that bench.py can time the reference's GPU kernels on the same matrices and
// the same GPU as this library's:
//
//   * SparseMatrix< Real, Devices::Cuda, int, GeneralMatrix, Segments >,
//     filled by operator=( host CSR matrix )   Matrices/SparseMatrix.hpp:1069-1193
//   * vectorProduct                            Matrices/SparseMatrixView.hpp:390-490
//     segments CSRScalar (TNL's CUDA default, Segments/CSR.h:580-605),
//     CSRVector, CSRLight, CSRAdaptive, Ellpack, SlicedEllpack (32),
//     ChunkedEllpack, BiEllpack, all in Devices::Cuda's default organization
//   * Solvers::Linear::CG / BICGStab / GMRES::solve   Solvers/Linear/*.hpp
//
// TNL launches every kernel synchronously (Cuda/KernelLaunch.h: the launch is
// followed by cudaStreamSynchronize), so a timed call includes that wait.
//
// Built by oracle/Makefile (`make cuda-ref TNL_SRC=...`) into
// oracle/_ref/libtnlcuda.so.

#include <TNL/Matrices/SparseMatrix.h>
#include <TNL/Algorithms/Segments/CSR.h>
#include <TNL/Algorithms/Segments/Ellpack.h>
#include <TNL/Algorithms/Segments/SlicedEllpack.h>
#include <TNL/Algorithms/Segments/ChunkedEllpack.h>
#include <TNL/Algorithms/Segments/BiEllpack.h>
#include <TNL/Solvers/Linear/CG.h>
#include <TNL/Solvers/Linear/BICGStab.h>
#include <TNL/Solvers/Linear/GMRES.h>
#include <TNL/Config/ParameterContainer.h>

#include <chrono>
#include <cstring>
#include <memory>
#include <string>

using namespace TNL;
namespace Seg = TNL::Algorithms::Segments;
using Host = TNL::Devices::Host;
using CudaDev = TNL::Devices::Cuda;

template< typename Real, typename Device, template< typename, typename, typename > class S >
using Mat = Matrices::SparseMatrix< Real, Device, int, Matrices::GeneralMatrix, S >;

// the padded layouts in Devices::Cuda's default organization (ColumnMajorOrder)
template< typename D, typename I, typename A >
using Ell32 = Seg::Ellpack< D, I, A, Seg::ColumnMajorOrder, 32 >;
template< typename D, typename I, typename A >
using SEll32 = Seg::SlicedEllpack< D, I, A, Seg::ColumnMajorOrder, 32 >;
template< typename D, typename I, typename A >
using ChEll = Seg::ChunkedEllpack< D, I, A, Seg::ColumnMajorOrder >;
template< typename D, typename I, typename A >
using BiEll32 = Seg::BiEllpack< D, I, A, Seg::ColumnMajorOrder, 32 >;

// A 256 MiB read after a 256 MiB write: evicts L2 between timed calls (the
// same flush the library's own products are timed with).
__global__ void
flush_kernel( float* w, const float* r, long long n, float* sink )
{
   float s = 0;
   for( long long i = blockIdx.x * (long long) blockDim.x + threadIdx.x; i < n; i += (long long) gridDim.x * blockDim.x ) {
      w[ i ] = 1.0f;
      s += r[ i ];
   }
   if( s == 12345.0f )
      *sink = s;
}

struct Flush
{
   float *w = nullptr, *r = nullptr, *sink = nullptr;
   long long n = ( 256ll << 20 ) / 4;
   Flush()
   {
      if( cudaMalloc( &w, n * 4 ) != cudaSuccess || cudaMalloc( &r, n * 4 ) != cudaSuccess
          || cudaMalloc( &sink, 4 ) != cudaSuccess )
         throw std::runtime_error( "flush buffers" );
      cudaMemset( r, 0, n * 4 );
   }
   ~Flush()
   {
      cudaFree( w );
      cudaFree( r );
      cudaFree( sink );
   }
   void
   run()
   {
      flush_kernel<<< 148 * 8, 256 >>>( w, r, n, sink );
   }
};

struct CudaMatrixBase
{
   virtual ~CudaMatrixBase() = default;
   virtual void
   spmv( const double* x, double* y ) = 0;
   virtual double
   timeSpmv( const double* x, int warmup, int loops, double* best ) = 0;
};

template< typename Real >
static Mat< Real, Host, Seg::CSRDefault >
hostCsr( int rows, int cols, const int* offsets, const int* columns, const double* values )
{
   Mat< Real, Host, Seg::CSRDefault > csr( rows, cols );
   Containers::Vector< int, Host, int > caps( rows );
   for( int i = 0; i < rows; i++ )
      caps[ i ] = offsets[ i + 1 ] - offsets[ i ];
   csr.setRowCapacities( caps );
   auto& v = csr.getValues();
   auto& c = csr.getColumnIndexes();
   for( long long k = 0; k < offsets[ rows ]; k++ ) {
      v[ k ] = (Real) values[ k ];
      c[ k ] = columns[ k ];
   }
   return csr;
}

template< typename Real, template< typename, typename, typename > class S >
struct CudaMatrix : CudaMatrixBase
{
   Mat< Real, CudaDev, S > A;
   Containers::Vector< Real, CudaDev, int > xv, yv;
   Flush flush;

   void
   load( const double* x )
   {
      Containers::Vector< Real, Host, int > h( A.getColumns() );
      for( int i = 0; i < A.getColumns(); i++ )
         h[ i ] = (Real) x[ i ];
      xv = h;
      yv.setSize( A.getRows() );
      yv = 0;
   }
   void
   spmv( const double* x, double* y ) override
   {
      load( x );
      A.vectorProduct( xv, yv );
      Containers::Vector< Real, Host, int > h;
      h = yv;
      for( int i = 0; i < A.getRows(); i++ )
         y[ i ] = (double) h[ i ];
   }
   // mean and best device time of one vectorProduct call (CUDA events on the
   // legacy default stream TNL launches on; L2 evicted before every call)
   double
   timeSpmv( const double* x, int warmup, int loops, double* best ) override
   {
      load( x );
      for( int i = 0; i < warmup; i++ ) {
         flush.run();
         A.vectorProduct( xv, yv );
      }
      cudaEvent_t a, b;
      cudaEventCreate( &a );
      cudaEventCreate( &b );
      double sum = 0, mn = 1e30;
      for( int i = 0; i < loops; i++ ) {
         flush.run();
         cudaEventRecord( a, 0 );
         A.vectorProduct( xv, yv );
         cudaEventRecord( b, 0 );
         cudaEventSynchronize( b );
         float ms = 0;
         cudaEventElapsedTime( &ms, a, b );
         sum += ms;
         mn = ms < mn ? ms : mn;
      }
      cudaEventDestroy( a );
      cudaEventDestroy( b );
      *best = mn;
      return sum / loops;
   }
};

template< typename Real, template< typename, typename, typename > class S >
static CudaMatrixBase*
make( int rows, int cols, const int* offsets, const int* columns, const double* values )
{
   auto* m = new CudaMatrix< Real, S >();
   m->A = hostCsr< Real >( rows, cols, offsets, columns, values );
   return m;
}

template< typename Real >
static CudaMatrixBase*
makeFormat( int format, int rows, int cols, const int* offsets, const int* columns, const double* values )
{
   switch( format ) {
      case 0:
         return make< Real, Seg::CSRScalar >( rows, cols, offsets, columns, values );
      case 1:
         return make< Real, Seg::CSRVector >( rows, cols, offsets, columns, values );
      case 2:
         return make< Real, Seg::CSRLight >( rows, cols, offsets, columns, values );
      case 3:
         return make< Real, Seg::CSRAdaptive >( rows, cols, offsets, columns, values );
      case 4:
         return make< Real, Ell32 >( rows, cols, offsets, columns, values );
      case 5:
         return make< Real, SEll32 >( rows, cols, offsets, columns, values );
      case 6:
         return make< Real, ChEll >( rows, cols, offsets, columns, values );
      case 7:
         return make< Real, BiEll32 >( rows, cols, offsets, columns, values );
      default:
         return nullptr;
   }
}

template< typename Real >
static int
solveImpl( int solver, int rows, const int* offsets, const int* columns, const double* values, const double* b, double* x,
           double rtol, long long maxit, long long* iters, double* seconds )
{
   using M = Mat< Real, CudaDev, Seg::CSRScalar >;
   auto A = std::make_shared< M >();
   *A = hostCsr< Real >( rows, rows, offsets, columns, values );
   Containers::Vector< Real, Host, int > bh( rows ), xh( rows );
   for( int i = 0; i < rows; i++ ) {
      bh[ i ] = (Real) b[ i ];
      xh[ i ] = (Real) x[ i ];
   }
   Containers::Vector< Real, CudaDev, int > bd, xd;
   bd = bh;
   xd = xh;
   auto run = [ & ]( auto& s ) -> bool
   {
      s.setMatrix( A );
      s.setConvergenceResidue( rtol );
      s.setMaxIterations( maxit );
      cudaDeviceSynchronize();
      const auto t0 = std::chrono::steady_clock::now();
      const bool ok = s.solve( bd.getConstView(), xd.getView() );
      cudaDeviceSynchronize();
      *seconds = std::chrono::duration< double >( std::chrono::steady_clock::now() - t0 ).count();
      *iters = s.getIterations();
      return ok;
   };
   bool ok = false;
   if( solver == 0 ) {
      Solvers::Linear::CG< M > s;
      ok = run( s );
   }
   else if( solver == 1 ) {
      Solvers::Linear::BICGStab< M > s;
      ok = run( s );
   }
   else {
      Solvers::Linear::GMRES< M > s;
      Config::ParameterContainer p;
      p.addParameter< std::string >( "gmres-variant", "CGSR" );
      p.addParameter< int >( "gmres-restarting-min", 30 );
      p.addParameter< int >( "gmres-restarting-max", 30 );
      p.addParameter< int >( "gmres-restarting-step-min", 3 );
      p.addParameter< int >( "gmres-restarting-step-max", 3 );
      s.setup( p );
      ok = run( s );
   }
   xh = xd;
   for( int i = 0; i < rows; i++ )
      x[ i ] = (double) xh[ i ];
   return ok ? 1 : 0;
}

extern "C" {

// format: 0 CSRScalar (TNL's CUDA default), 1 CSRVector, 2 CSRLight, 3 CSRAdaptive,
//         4 Ellpack, 5 SlicedEllpack(32), 6 ChunkedEllpack, 7 BiEllpack
// real: 0 double, 1 float. NULL when TNL throws.
void*
tnlcuda_create( int format, int real, int rows, int cols, const int* offsets, const int* columns, const double* values )
{
   try {
      return real == 0 ? makeFormat< double >( format, rows, cols, offsets, columns, values )
                       : makeFormat< float >( format, rows, cols, offsets, columns, values );
   }
   catch( ... ) {
      return nullptr;
   }
}

void
tnlcuda_destroy( void* h )
{
   delete static_cast< CudaMatrixBase* >( h );
}

int
tnlcuda_spmv( void* h, const double* x, double* y )
{
   try {
      static_cast< CudaMatrixBase* >( h )->spmv( x, y );
      return 0;
   }
   catch( ... ) {
      return -1;
   }
}

// mean milliseconds per call over `loops` timed calls (best in *best_ms); -1 when TNL throws
double
tnlcuda_spmv_time( void* h, const double* x, int warmup, int loops, double* best_ms )
{
   try {
      return static_cast< CudaMatrixBase* >( h )->timeSpmv( x, warmup, loops, best_ms );
   }
   catch( ... ) {
      return -1;
   }
}

// solver: 0 CG, 1 BiCGStab, 2 GMRES (CGSR, restart 30); CSRScalar matrix on the GPU.
// Returns 1 converged, 0 not, -1 when TNL throws.
int
tnlcuda_solve( int solver, int real, int rows, const int* offsets, const int* columns, const double* values,
               const double* b, double* x, double rtol, long long maxit, long long* iters, double* seconds )
{
   try {
      return real == 0 ? solveImpl< double >( solver, rows, offsets, columns, values, b, x, rtol, maxit, iters, seconds )
                       : solveImpl< float >( solver, rows, offsets, columns, values, b, x, rtol, maxit, iters, seconds );
   }
   catch( ... ) {
      return -1;
   }
}

}  // extern "C"
