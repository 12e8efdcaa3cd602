// TEST INFRASTRUCTURE ONLY — the checker, never the product.
//
// Driver for the reference implementation itself: this translation unit is
// compiled against TNL's own headers (header-only library) and exposes TNL's
// Devices::Host path behind a flat C ABI so that the tests, the fixture
// generator and the CPU baseline in bench.py can call it through ctypes.
// Nothing of TNL is copied here; every call goes into the unmodified headers:
//
//   * SparseMatrix::setRowCapacities / operator=(other format)
//       src/TNL/Matrices/SparseMatrix.hpp:284-304, 1069-1193
//   * SparseMatrix::vectorProduct
//       src/TNL/Matrices/SparseMatrixView.hpp:390-490
//   * SparseMatrix::setElement / addElement
//       src/TNL/Matrices/SparseMatrixView.hpp:256-340
//   * MatrixReader::readMtx, MatrixWriter::writeMtx
//       src/TNL/Matrices/MatrixReader.hpp:51-359, MatrixWriter.hpp:103-128
//   * SparseMatrix::save / load (Object, File)
//       src/TNL/Matrices/SparseMatrix.hpp:1233-1290, Object.hpp, File.hpp
//   * Solvers::Linear::{CG, BICGStab, GMRES, TFQMR, BICGStabL}::solve,
//     Preconditioners::Diagonal, ILU0
//       src/TNL/Solvers/Linear/CG.hpp:11-104, BICGStab.hpp:33-118,
//       GMRES.hpp:72-178, TFQMR.hpp:18-114, BICGStabL.hpp:42-250,
//       Preconditioners/Diagonal.hpp:13-47, Preconditioners/ILU0.hpp:23-144
//
// The segment classes keep their storage in protected members; they are read
// through pointer-to-member accessors taken inside small derived structs,
// which is legal C++ and leaves TNL untouched.
//
// Built by oracle/Makefile into oracle/_ref/libtnlref.so.

#include <TNL/Matrices/SparseMatrix.h>
#include <TNL/Algorithms/Segments/CSR.h>
#include <TNL/Algorithms/Segments/Ellpack.h>
#include <TNL/Algorithms/Segments/SlicedEllpack.h>
#include <TNL/Matrices/MatrixPermutationApplier.h>
#include <TNL/Matrices/SparseOperations.h>
#include <TNL/Matrices/MatrixReader.h>
#include <TNL/Matrices/MatrixWriter.h>
#include <TNL/Algorithms/Segments/ChunkedEllpack.h>
#include <TNL/Algorithms/Segments/BiEllpack.h>
#include <TNL/Solvers/Linear/CG.h>
#include <TNL/Solvers/Linear/BICGStab.h>
#include <TNL/Solvers/Linear/GMRES.h>
#include <TNL/Solvers/Linear/TFQMR.h>
#include <TNL/Solvers/Linear/BICGStabL.h>
#include <TNL/Solvers/Linear/Preconditioners/Diagonal.h>
#include <TNL/Solvers/Linear/Preconditioners/ILU0.h>
#include <TNL/Solvers/Linear/Preconditioners/ILUT.h>
#include <TNL/Solvers/Linear/Jacobi.h>
#include <TNL/Solvers/Linear/SOR.h>
#include <TNL/Matrices/MultidiagonalMatrix.h>
#include <TNL/Config/ParameterContainer.h>

#include <omp.h>
#include <chrono>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

using namespace TNL;
namespace Seg = TNL::Algorithms::Segments;
using Host = TNL::Devices::Host;

// ---------------------------------------------------------------------------
// Segment type aliases with an explicit element organization.
template< typename D, typename I, typename A >
using CSRSeg = Seg::CSRDefault< D, I, A >;
template< typename D, typename I, typename A >
using EllCol = Seg::Ellpack< D, I, A, Seg::ColumnMajorOrder, 32 >;
template< typename D, typename I, typename A >
using EllRow = Seg::Ellpack< D, I, A, Seg::RowMajorOrder, 32 >;
template< typename D, typename I, typename A >
using SEllCol = Seg::SlicedEllpack< D, I, A, Seg::ColumnMajorOrder, 32 >;
template< typename D, typename I, typename A >
using SEllRow = Seg::SlicedEllpack< D, I, A, Seg::RowMajorOrder, 32 >;
// other slice sizes (format codes 5, 6, 7)
template< int SS >
struct SEllSized
{
   template< typename D, typename I, typename A >
   using Col = Seg::SlicedEllpack< D, I, A, Seg::ColumnMajorOrder, SS >;
   template< typename D, typename I, typename A >
   using Row = Seg::SlicedEllpack< D, I, A, Seg::RowMajorOrder, SS >;
};
template< typename T >
struct IsSliced : std::false_type
{};
template< typename D, typename I, typename A, Seg::ElementsOrganization O, int SS >
struct IsSliced< Seg::SlicedEllpack< D, I, A, O, SS > > : std::true_type
{};
template< typename D, typename I, typename A >
using CEllCol = Seg::ChunkedEllpack< D, I, A, Seg::ColumnMajorOrder >;
template< typename D, typename I, typename A >
using CEllRow = Seg::ChunkedEllpack< D, I, A, Seg::RowMajorOrder >;
template< typename D, typename I, typename A >
using BEllCol = Seg::BiEllpack< D, I, A, Seg::ColumnMajorOrder, 32 >;
template< typename D, typename I, typename A >
using BEllRow = Seg::BiEllpack< D, I, A, Seg::RowMajorOrder, 32 >;

using IndexAlloc = typename Allocators::Default< Host >::template Allocator< int >;

// ---------------------------------------------------------------------------
// Accessors for protected segment storage (pointer-to-member through a
// derived type; no TNL code is modified or re-declared).
template< typename S >
struct SlicedAcc : S
{
   static auto p_sliceOffsets() { return &SlicedAcc::sliceOffsets; }
   static auto p_sliceSegmentSizes() { return &SlicedAcc::sliceSegmentSizes; }
   static auto p_size() { return &SlicedAcc::size; }
   static auto p_alignedSize() { return &SlicedAcc::alignedSize; }
};
template< typename S >
struct EllAcc : S
{
   static auto p_segmentSize() { return &EllAcc::segmentSize; }
   static auto p_size() { return &EllAcc::size; }
   static auto p_alignedSize() { return &EllAcc::alignedSize; }
};
template< typename S >
struct ChunkedAcc : S
{
   static auto p_rowToSliceMapping() { return &ChunkedAcc::rowToSliceMapping; }
   static auto p_rowToChunkMapping() { return &ChunkedAcc::rowToChunkMapping; }
   static auto p_chunksToSegmentsMapping() { return &ChunkedAcc::chunksToSegmentsMapping; }
   static auto p_rowPointers() { return &ChunkedAcc::rowPointers; }
   static auto p_slices() { return &ChunkedAcc::slices; }
   static auto p_numberOfSlices() { return &ChunkedAcc::numberOfSlices; }
   static auto p_storageSize() { return &ChunkedAcc::storageSize; }
};
template< typename S >
struct BiAcc : S
{
   static auto p_rowPermArray() { return &BiAcc::rowPermArray; }
   static auto p_groupPointers() { return &BiAcc::groupPointers; }
   static auto p_virtualRows() { return &BiAcc::virtualRows; }
   static auto p_storageSize() { return &BiAcc::storageSize; }
};

// ---------------------------------------------------------------------------
struct Arrays
{
   // name -> int64 copy (index arrays are widened; scalars are 1-element arrays)
   std::vector< std::pair< std::string, std::vector< long long > > > ints;
   void
   put( const std::string& n, std::vector< long long > v )
   {
      ints.emplace_back( n, std::move( v ) );
   }
   template< typename Vec >
   void
   putVec( const std::string& n, const Vec& v, long long count = -1 )
   {
      std::vector< long long > out;
      const long long s = count < 0 ? v.getSize() : count;
      out.resize( s );
      for( long long i = 0; i < s; i++ )
         out[ i ] = v[ i ];
      put( n, std::move( out ) );
   }
   void
   putScalar( const std::string& n, long long s )
   {
      put( n, std::vector< long long >{ s } );
   }
};

struct MatrixBase
{
   virtual ~MatrixBase() = default;
   virtual void
   spmv( const double* x, double* y, double alpha, double beta, int begin, int end ) = 0;
   virtual double
   timeSpmv( const double* x, int loops ) = 0;
   virtual long long
   storageSize() const = 0;
   virtual void
   exportValues( double* out ) const = 0;
   virtual void
   exportColumns( int* out ) const = 0;
   // elements [first, first + count) of the storage arrays (large layouts are
   // compared piece by piece)
   virtual void
   exportValuesRange( double* out, long long first, long long count ) const = 0;
   virtual void
   exportColumnsRange( int* out, long long first, long long count ) const = 0;
   // Matrices/MatrixPermutationApplier.h
   virtual void
   permuteRows( const int* perm ) = 0;
   virtual void
   permuteColumns( const int* iperm ) = 0;
   virtual void
   writeMtx( const char* path ) const = 0;
   // Object::save( fileName ) (SparseMatrix.hpp:1264-1290)
   virtual void
   save( const char* path ) const = 0;
   // SparseMatrix::operator=( const RHSMatrix& ) into another layout
   virtual MatrixBase*
   convertTo( int format, int org ) const = 0;
   Arrays meta;
   int rows = 0, cols = 0;
};

template< typename Real, template< typename, typename, typename > class S >
using Mat = Matrices::SparseMatrix< Real, Host, int, Matrices::GeneralMatrix, S >;

template< typename Real >
static Mat< Real, CSRSeg >
makeCsr( int rows, int cols, const int* offsets, const int* columns, const double* values )
{
   Mat< Real, CSRSeg > csr( rows, cols );
   Containers::Vector< int, Host, int > caps( rows );
   for( int i = 0; i < rows; i++ )
      caps[ i ] = offsets[ i + 1 ] - offsets[ i ];
   csr.setRowCapacities( caps );
   auto& v = csr.getValues();
   auto& c = csr.getColumnIndexes();
   const long long nnz = offsets[ rows ];
   for( long long k = 0; k < nnz; k++ ) {
      v[ k ] = (Real) values[ k ];
      c[ k ] = columns[ k ];
   }
   return csr;
}

template< typename Real, template< typename, typename, typename > class S >
struct MatrixImpl : MatrixBase
{
   Mat< Real, S > A;

   void
   spmv( const double* x, double* y, double alpha, double beta, int begin, int end ) override
   {
      Containers::Vector< Real, Host, int > xv( A.getColumns() ), yv( A.getRows() );
      for( int i = 0; i < A.getColumns(); i++ )
         xv[ i ] = (Real) x[ i ];
      for( int i = 0; i < A.getRows(); i++ )
         yv[ i ] = (Real) y[ i ];
      A.vectorProduct( xv, yv, (Real) alpha, (Real) beta, begin, end );
      for( int i = 0; i < A.getRows(); i++ )
         y[ i ] = (double) yv[ i ];
   }

   double
   timeSpmv( const double* x, int loops ) override
   {
      Containers::Vector< Real, Host, int > xv( A.getColumns() ), yv( A.getRows() );
      for( int i = 0; i < A.getColumns(); i++ )
         xv[ i ] = (Real) x[ i ];
      yv = 0;
      A.vectorProduct( xv, yv );  // warm-up
      auto t0 = std::chrono::steady_clock::now();
      for( int l = 0; l < loops; l++ )
         A.vectorProduct( xv, yv );
      auto t1 = std::chrono::steady_clock::now();
      return std::chrono::duration< double >( t1 - t0 ).count() / loops;
   }

   long long
   storageSize() const override
   {
      return A.getValues().getSize();
   }
   void
   exportValues( double* out ) const override
   {
      const auto& v = A.getValues();
      for( long long i = 0; i < v.getSize(); i++ )
         out[ i ] = (double) v[ i ];
   }
   void
   exportColumns( int* out ) const override
   {
      const auto& c = A.getColumnIndexes();
      for( long long i = 0; i < c.getSize(); i++ )
         out[ i ] = c[ i ];
   }
   void
   exportValuesRange( double* out, long long first, long long count ) const override
   {
      const auto& v = A.getValues();
      for( long long i = 0; i < count; i++ )
         out[ i ] = (double) v[ first + i ];
   }
   void
   exportColumnsRange( int* out, long long first, long long count ) const override
   {
      const auto& c = A.getColumnIndexes();
      for( long long i = 0; i < count; i++ )
         out[ i ] = c[ first + i ];
   }
   void
   permuteRows( const int* perm ) override
   {
      Containers::Array< int, Host, int > p( A.getRows() );
      for( int i = 0; i < A.getRows(); i++ )
         p[ i ] = perm[ i ];
      Matrices::permuteMatrixRows( A, p );
      recapture();
   }
   void
   permuteColumns( const int* iperm ) override
   {
      Containers::Array< int, Host, int > p( A.getColumns() );
      for( int i = 0; i < A.getColumns(); i++ )
         p[ i ] = iperm[ i ];
      Matrices::permuteMatrixColumns( A, p );
   }
   void
   writeMtx( const char* path ) const override
   {
      Matrices::MatrixWriter< Mat< Real, S > >::writeMtx( path, A );
   }
   MatrixBase*
   convertTo( int format, int org ) const override;
   void
   save( const char* path ) const override
   {
      A.save( String( path ) );
   }
   void
   recapture();
};

// Metadata capture per segment family ----------------------------------------
template< typename Segments >
static void
captureMeta( Arrays&, const Segments&, int )
{}

template< typename Real >
static void
captureCsr( Arrays& m, const Mat< Real, CSRSeg >& A )
{
   m.putVec( "offsets", A.getSegments().getOffsets() );
}

template< typename S >
static void
captureEll( Arrays& m, const S& s )
{
   m.putScalar( "segmentSize", s.*( EllAcc< S >::p_segmentSize() ) );
   m.putScalar( "size", s.*( EllAcc< S >::p_size() ) );
   m.putScalar( "alignedSize", s.*( EllAcc< S >::p_alignedSize() ) );
}

template< typename S >
static void
captureSliced( Arrays& m, const S& s )
{
   m.putVec( "sliceOffsets", s.*( SlicedAcc< S >::p_sliceOffsets() ) );
   m.putVec( "sliceSegmentSizes", s.*( SlicedAcc< S >::p_sliceSegmentSizes() ) );
   m.putScalar( "size", s.*( SlicedAcc< S >::p_size() ) );
   m.putScalar( "alignedSize", s.*( SlicedAcc< S >::p_alignedSize() ) );
}

template< typename S >
static void
captureChunked( Arrays& m, const S& s )
{
   const int nslices = s.*( ChunkedAcc< S >::p_numberOfSlices() );
   m.putScalar( "numberOfSlices", nslices );
   m.putScalar( "storageSize", s.*( ChunkedAcc< S >::p_storageSize() ) );
   m.putVec( "rowToChunkMapping", s.*( ChunkedAcc< S >::p_rowToChunkMapping() ) );
   m.putVec( "rowToSliceMapping", s.*( ChunkedAcc< S >::p_rowToSliceMapping() ) );
   m.putVec( "chunksToSegmentsMapping", s.*( ChunkedAcc< S >::p_chunksToSegmentsMapping() ) );
   m.putVec( "rowPointers", s.*( ChunkedAcc< S >::p_rowPointers() ) );
   const auto& sl = s.*( ChunkedAcc< S >::p_slices() );
   std::vector< long long > flat;
   // only the first numberOfSlices entries are defined (the container is sized by rows)
   for( int i = 0; i < nslices; i++ ) {
      flat.push_back( sl[ i ].size );
      flat.push_back( sl[ i ].chunkSize );
      flat.push_back( sl[ i ].firstSegment );
      flat.push_back( sl[ i ].pointer );
   }
   m.put( "slices", flat );
}

template< typename S >
static void
captureBi( Arrays& m, const S& s )
{
   m.putScalar( "virtualRows", s.*( BiAcc< S >::p_virtualRows() ) );
   m.putScalar( "storageSize", s.*( BiAcc< S >::p_storageSize() ) );
   m.putVec( "rowPermArray", s.*( BiAcc< S >::p_rowPermArray() ) );
   m.putVec( "groupPointers", s.*( BiAcc< S >::p_groupPointers() ) );
}

template< typename Real, template< typename, typename, typename > class S >
static void
captureAll( Arrays& meta, const Mat< Real, S >& A )
{
   meta.ints.clear();
   using SegT = typename Mat< Real, S >::SegmentsType;
   const auto& seg = A.getSegments();
   if constexpr( std::is_same< SegT, CSRSeg< Host, int, IndexAlloc > >::value )
      meta.putVec( "offsets", seg.getOffsets() );
   else if constexpr( std::is_same< SegT, EllCol< Host, int, IndexAlloc > >::value
                      || std::is_same< SegT, EllRow< Host, int, IndexAlloc > >::value )
      captureEll( meta, seg );
   else if constexpr( IsSliced< SegT >::value )
      captureSliced( meta, seg );
   else if constexpr( std::is_same< SegT, CEllCol< Host, int, IndexAlloc > >::value
                      || std::is_same< SegT, CEllRow< Host, int, IndexAlloc > >::value )
      captureChunked( meta, seg );
   else if constexpr( std::is_same< SegT, BEllCol< Host, int, IndexAlloc > >::value
                      || std::is_same< SegT, BEllRow< Host, int, IndexAlloc > >::value )
      captureBi( meta, seg );
}

template< typename Real, template< typename, typename, typename > class S >
void
MatrixImpl< Real, S >::recapture()
{
   captureAll< Real, S >( meta, A );
}

template< typename Real, template< typename, typename, typename > class S >
static MatrixBase*
build( int rows, int cols, const int* offsets, const int* columns, const double* values )
{
   auto* M = new MatrixImpl< Real, S >();
   M->rows = rows;
   M->cols = cols;
   auto csr = makeCsr< Real >( rows, cols, offsets, columns, values );
   M->A = csr;  // SparseMatrix::operator=( const RHSMatrix& ) — TNL's own conversion
   using SegT = typename Mat< Real, S >::SegmentsType;
   const auto& seg = M->A.getSegments();
   if constexpr( std::is_same< SegT, CSRSeg< Host, int, IndexAlloc > >::value )
      M->meta.putVec( "offsets", seg.getOffsets() );
   else if constexpr( std::is_same< SegT, EllCol< Host, int, IndexAlloc > >::value
                 || std::is_same< SegT, EllRow< Host, int, IndexAlloc > >::value )
      captureEll( M->meta, seg );
   else if constexpr( IsSliced< SegT >::value )
      captureSliced( M->meta, seg );
   else if constexpr( std::is_same< SegT, CEllCol< Host, int, IndexAlloc > >::value
                      || std::is_same< SegT, CEllRow< Host, int, IndexAlloc > >::value )
      captureChunked( M->meta, seg );
   else if constexpr( std::is_same< SegT, BEllCol< Host, int, IndexAlloc > >::value
                      || std::is_same< SegT, BEllRow< Host, int, IndexAlloc > >::value )
      captureBi( M->meta, seg );
   return M;
}

template< typename Real >
static MatrixBase*
buildCsrDirect( int rows, int cols, const int* offsets, const int* columns, const double* values )
{
   // CSR is stored exactly as given (the matrix a TNL user assembles with
   // setRowCapacities + setElement); no conversion is applied.
   auto* M = new MatrixImpl< Real, CSRSeg >();
   M->rows = rows;
   M->cols = cols;
   M->A = makeCsr< Real >( rows, cols, offsets, columns, values );
   captureCsr< Real >( M->meta, M->A );
   return M;
}

template< typename Real >
static MatrixBase*
dispatch( int format, int org, int rows, int cols, const int* off, const int* col, const double* val )
{
   const bool cm = ( org == 0 );
   switch( format ) {
      case 0:
         return buildCsrDirect< Real >( rows, cols, off, col, val );
      case 1:
         return cm ? build< Real, EllCol >( rows, cols, off, col, val ) : build< Real, EllRow >( rows, cols, off, col, val );
      case 2:
         return cm ? build< Real, SEllCol >( rows, cols, off, col, val ) : build< Real, SEllRow >( rows, cols, off, col, val );
      case 3:
         return cm ? build< Real, CEllCol >( rows, cols, off, col, val ) : build< Real, CEllRow >( rows, cols, off, col, val );
      case 4:
         return cm ? build< Real, BEllCol >( rows, cols, off, col, val ) : build< Real, BEllRow >( rows, cols, off, col, val );
      case 5:
         return cm ? build< Real, SEllSized< 8 >::Col >( rows, cols, off, col, val )
                   : build< Real, SEllSized< 8 >::Row >( rows, cols, off, col, val );
      case 6:
         return cm ? build< Real, SEllSized< 16 >::Col >( rows, cols, off, col, val )
                   : build< Real, SEllSized< 16 >::Row >( rows, cols, off, col, val );
      case 7:
         return cm ? build< Real, SEllSized< 64 >::Col >( rows, cols, off, col, val )
                   : build< Real, SEllSized< 64 >::Row >( rows, cols, off, col, val );
   }
   return nullptr;
}

// ---------------------------------------------------------------------------
// Binary matrices: SparseMatrix< bool, Host, int, GeneralMatrix, S > filled by
// operator= from the double CSR matrix (zero values dropped, only the column
// indexes stored: SparseMatrix.h:23-26, SparseMatrix.hpp:297-302, 1069-1193).
// The product runs in ComputeReal = int (SparseMatrixView.h:22-30): each
// stored column adds (int) x[column], and alpha / beta are passed as ints
// (SparseMatrixView.hpp:423-471).
template< template< typename, typename, typename > class S >
struct BinaryImpl : MatrixBase
{
   Mat< bool, S > A;

   template< typename V >
   void
   product( const V* x, V* y, double alpha, double beta, int begin, int end )
   {
      Containers::Vector< V, Host, int > xv( A.getColumns() ), yv( A.getRows() );
      for( int i = 0; i < A.getColumns(); i++ )
         xv[ i ] = x[ i ];
      for( int i = 0; i < A.getRows(); i++ )
         yv[ i ] = y[ i ];
      A.vectorProduct( xv, yv, alpha, beta, begin, end );
      for( int i = 0; i < A.getRows(); i++ )
         y[ i ] = yv[ i ];
   }
   void
   spmv( const double* x, double* y, double alpha, double beta, int begin, int end ) override
   {
      product< double >( x, y, alpha, beta, begin, end );
   }
   double
   timeSpmv( const double*, int ) override
   {
      return 0;
   }
   long long
   storageSize() const override
   {
      return A.getColumnIndexes().getSize();
   }
   void
   exportValues( double* out ) const override
   {
      for( long long i = 0; i < storageSize(); i++ )
         out[ i ] = 0;  // binary matrices store no values
   }
   void
   exportColumns( int* out ) const override
   {
      const auto& c = A.getColumnIndexes();
      for( long long i = 0; i < c.getSize(); i++ )
         out[ i ] = c[ i ];
   }
   void
   exportValuesRange( double* out, long long, long long count ) const override
   {
      for( long long i = 0; i < count; i++ )
         out[ i ] = 0;
   }
   void
   exportColumnsRange( int* out, long long first, long long count ) const override
   {
      const auto& c = A.getColumnIndexes();
      for( long long i = 0; i < count; i++ )
         out[ i ] = c[ first + i ];
   }
   void
   permuteRows( const int* ) override
   {
      throw std::logic_error( "not used for binary matrices" );
   }
   void
   permuteColumns( const int* ) override
   {
      throw std::logic_error( "not used for binary matrices" );
   }
   void
   writeMtx( const char* ) const override
   {
      throw std::logic_error( "not used for binary matrices" );
   }
   void
   save( const char* ) const override
   {
      throw std::logic_error( "not used for binary matrices" );
   }
   MatrixBase*
   convertTo( int, int ) const override
   {
      throw std::logic_error( "not used for binary matrices" );
   }
};

template< template< typename, typename, typename > class S >
static MatrixBase*
buildBinary( int rows, int cols, const int* offsets, const int* columns, const double* values )
{
   auto* M = new BinaryImpl< S >();
   M->rows = rows;
   M->cols = cols;
   M->A = makeCsr< double >( rows, cols, offsets, columns, values );  // operator=: zeros dropped
   captureAll< bool, S >( M->meta, M->A );
   return M;
}

static MatrixBase*
dispatchBinary( int format, int org, int rows, int cols, const int* off, const int* col, const double* val )
{
   const bool cm = ( org == 0 );
   switch( format ) {
      case 0:
         return buildBinary< CSRSeg >( rows, cols, off, col, val );
      case 1:
         return cm ? buildBinary< EllCol >( rows, cols, off, col, val ) : buildBinary< EllRow >( rows, cols, off, col, val );
      case 2:
         return cm ? buildBinary< SEllCol >( rows, cols, off, col, val ) : buildBinary< SEllRow >( rows, cols, off, col, val );
      case 3:
         return cm ? buildBinary< CEllCol >( rows, cols, off, col, val ) : buildBinary< CEllRow >( rows, cols, off, col, val );
      case 4:
         return cm ? buildBinary< BEllCol >( rows, cols, off, col, val ) : buildBinary< BEllRow >( rows, cols, off, col, val );
   }
   return nullptr;
}

// the product of a binary matrix with float vectors
template< template< typename, typename, typename > class S >
static bool
binaryProductF32( MatrixBase* h, const float* x, float* y, double alpha, double beta, int begin, int end )
{
   auto* b = dynamic_cast< BinaryImpl< S >* >( h );
   if( ! b )
      return false;
   b->template product< float >( x, y, alpha, beta, begin, end );
   return true;
}

// ---------------------------------------------------------------------------
// F::template run< Real, S >() for the segments type of (format, org).
template< typename Real, typename F >
static MatrixBase*
withLayout( int format, int org, F& f )
{
   const bool cm = ( org == 0 );
   switch( format ) {
      case 0:
         return f.template run< Real, CSRSeg >();
      case 1:
         return cm ? f.template run< Real, EllCol >() : f.template run< Real, EllRow >();
      case 2:
         return cm ? f.template run< Real, SEllCol >() : f.template run< Real, SEllRow >();
      case 3:
         return cm ? f.template run< Real, CEllCol >() : f.template run< Real, CEllRow >();
      case 4:
         return cm ? f.template run< Real, BEllCol >() : f.template run< Real, BEllRow >();
      case 5:
         return cm ? f.template run< Real, SEllSized< 8 >::Col >() : f.template run< Real, SEllSized< 8 >::Row >();
      case 6:
         return cm ? f.template run< Real, SEllSized< 16 >::Col >() : f.template run< Real, SEllSized< 16 >::Row >();
      case 7:
         return cm ? f.template run< Real, SEllSized< 64 >::Col >() : f.template run< Real, SEllSized< 64 >::Row >();
   }
   return nullptr;
}

// target = source through TNL's operator= (same Real)
template< typename Real, template< typename, typename, typename > class Src >
struct ConvertFrom
{
   const Mat< Real, Src >& src;
   template< typename R2, template< typename, typename, typename > class S >
   MatrixBase*
   run()
   {
      auto* M = new MatrixImpl< R2, S >();
      M->rows = src.getRows();
      M->cols = src.getColumns();
      M->A = src;
      M->recapture();
      return M;
   }
};

template< typename Real, template< typename, typename, typename > class S >
MatrixBase*
MatrixImpl< Real, S >::convertTo( int format, int org ) const
{
   ConvertFrom< Real, S > f{ A };
   return withLayout< Real >( format, org, f );
}

// setRowCapacities( triplet counts ) + setElement / addElement per triplet, in order
struct FromCoo
{
   int rows, cols;
   long long n;
   const int *ri, *ci;
   const double* v;
   int add;
   const int* rowCaps;
   template< typename Real, template< typename, typename, typename > class S >
   MatrixBase*
   run()
   {
      auto* M = new MatrixImpl< Real, S >();
      M->rows = rows;
      M->cols = cols;
      M->A.setDimensions( rows, cols );
      Containers::Vector< int, Host, int > caps( rows );
      caps = 0;
      for( long long k = 0; k < n; k++ )
         caps[ ri[ k ] ]++;
      if( rowCaps )
         for( int i = 0; i < rows; i++ )
            caps[ i ] = rowCaps[ i ];
      M->A.setRowCapacities( caps );
      for( long long k = 0; k < n; k++ ) {
         if( add )
            M->A.addElement( ri[ k ], ci[ k ], (Real) v[ k ], (Real) 1 );
         else
            M->A.setElement( ri[ k ], ci[ k ], (Real) v[ k ] );
      }
      M->recapture();
      return M;
   }
};

// SparseMatrix::load( fileName ) into the layout (format, org)
struct LoadFile
{
   const char* path;
   template< typename Real, template< typename, typename, typename > class S >
   MatrixBase*
   run()
   {
      auto* M = new MatrixImpl< Real, S >();
      M->A.load( String( path ) );
      M->rows = M->A.getRows();
      M->cols = M->A.getColumns();
      M->recapture();
      return M;
   }
};

struct ReadMtx
{
   const char* path;
   template< typename Real, template< typename, typename, typename > class S >
   MatrixBase*
   run()
   {
      auto* M = new MatrixImpl< Real, S >();
      Matrices::MatrixReader< Mat< Real, S > >::readMtx( path, M->A );
      M->rows = M->A.getRows();
      M->cols = M->A.getColumns();
      M->recapture();
      return M;
   }
};

// Matrices::MultidiagonalMatrix< Real, Host, int, Organization > built with
// setElement from row-major values (rows x diagonals; entries whose column is
// outside the matrix are not set)
struct MdiagBase
{
   virtual ~MdiagBase() = default;
   virtual long long storage() const = 0;
   virtual void values( double* out ) const = 0;
   virtual void spmv( const double* x, double* y, double alpha, double beta, int begin, int end ) = 0;
};

template< typename Real, Algorithms::Segments::ElementsOrganization Org >
struct MdiagImpl : MdiagBase
{
   using M = Matrices::MultidiagonalMatrix< Real, Host, int, Org >;
   M A;
   MdiagImpl( int rows, int cols, int nd, const int* offsets, const double* vals )
   {
      Containers::Vector< int, Host, int > o( nd );
      for( int d = 0; d < nd; d++ )
         o[ d ] = offsets[ d ];
      A.setDimensions( rows, cols, o );
      for( int r = 0; r < rows; r++ )
         for( int d = 0; d < nd; d++ ) {
            const long long c = (long long) r + offsets[ d ];
            if( c >= 0 && c < cols )
               A.setElement( r, (int) c, (Real) vals[ (long long) r * nd + d ] );
         }
   }
   long long storage() const override { return A.getValues().getSize(); }
   void
   values( double* out ) const override
   {
      for( long long k = 0; k < A.getValues().getSize(); k++ )
         out[ k ] = (double) A.getValues()[ k ];
   }
   void
   spmv( const double* x, double* y, double alpha, double beta, int begin, int end ) override
   {
      Containers::Vector< Real, Host, int > xv( A.getColumns() ), yv( A.getRows() );
      for( int i = 0; i < A.getColumns(); i++ )
         xv[ i ] = (Real) x[ i ];
      for( int i = 0; i < A.getRows(); i++ )
         yv[ i ] = (Real) y[ i ];
      A.vectorProduct( xv, yv, (Real) alpha, (Real) beta, begin, end );
      for( int i = 0; i < A.getRows(); i++ )
         y[ i ] = (double) yv[ i ];
   }
};

// ILUT parameters of the solves with precond 3 (tnlref_set_ilut)
static int g_ilut_p = 0;
static double g_ilut_tau = 1e-4;

// ---------------------------------------------------------------------------
// Solvers over the FP64 (or FP32) host CSR matrix.
template< typename Real >
static int
solveImpl( int solver,
           int precond,
           int rows,
           const int* offsets,
           const int* columns,
           const double* values,
           const double* b,
           double* x,
           double rtol,
           long long maxit,
           const char* gmresVariant,
           int restartMin,
           int restartMax,
           int exactResidue,
           int ell,
           long long* iters,
           double* residue,
           double* seconds )
{
   using M = Mat< Real, CSRSeg >;
   using Vec = Containers::Vector< Real, Host, int >;
   auto A = std::make_shared< M >( makeCsr< Real >( rows, rows, offsets, columns, values ) );
   Vec bv( rows ), xv( rows );
   for( int i = 0; i < rows; i++ ) {
      bv[ i ] = (Real) b[ i ];
      xv[ i ] = (Real) x[ i ];
   }
   Config::ParameterContainer params;
   params.addParameter< String >( "gmres-variant", String( gmresVariant ) );
   params.addParameter< int >( "gmres-restarting-min", restartMin );
   params.addParameter< int >( "gmres-restarting-max", restartMax );
   params.addParameter< bool >( "bicgstab-exact-residue", exactResidue != 0 );
   params.addParameter< int >( "bicgstab-ell", ell );
   params.addParameter< int >( "ilut-p", g_ilut_p );
   params.addParameter< double >( "ilut-threshold", g_ilut_tau );

   using Pre = Solvers::Linear::Preconditioners::Preconditioner< M >;
   std::shared_ptr< Pre > pre;
   if( precond == 2 )
      pre = std::make_shared< Solvers::Linear::Preconditioners::ILU0< M > >();
   else if( precond == 3 ) {
      pre = std::make_shared< Solvers::Linear::Preconditioners::ILUT< M > >();
      pre->setup( params );
   }
   else
      pre = std::make_shared< Solvers::Linear::Preconditioners::Diagonal< M > >();
   if( precond )
      pre->update( A );

   bool ok = false;
   auto t0 = std::chrono::steady_clock::now();
   auto run = [ & ]( auto& s )
   {
      s.setup( params );
      s.setMatrix( A );
      if( precond )
         s.setPreconditioner( pre );
      s.setConvergenceResidue( (Real) rtol );
      s.setMaxIterations( (int) maxit );
      ok = s.solve( bv, xv );
      *iters = s.getIterations();
      *residue = (double) s.getResidue();
   };
   if( solver == 0 ) {
      Solvers::Linear::CG< M > s;
      run( s );
   }
   else if( solver == 1 ) {
      Solvers::Linear::BICGStab< M > s;
      run( s );
   }
   else if( solver == 2 ) {
      Solvers::Linear::GMRES< M > s;
      run( s );
   }
   else if( solver == 3 ) {
      Solvers::Linear::TFQMR< M > s;
      run( s );
   }
   else {
      Solvers::Linear::BICGStabL< M > s;
      run( s );
   }
   auto t1 = std::chrono::steady_clock::now();
   *seconds = std::chrono::duration< double >( t1 - t0 ).count();
   for( int i = 0; i < rows; i++ )
      x[ i ] = (double) xv[ i ];
   return ok ? 1 : 0;
}

// Solvers::Linear::Jacobi (Jacobi.hpp:67-128) and SOR (SOR.hpp:66-118) on the
// host CSR matrix with the relaxation parameter and the residue period
template< typename Real >
static int
stationaryImpl( int solver, int rows, const int* offsets, const int* columns, const double* values, const double* b,
                double* x, double rtol, long long maxit, double omega, int period, long long* iters, double* residue )
{
   using M = Mat< Real, CSRSeg >;
   using Vec = Containers::Vector< Real, Host, int >;
   auto A = std::make_shared< M >( makeCsr< Real >( rows, rows, offsets, columns, values ) );
   Vec bv( rows ), xv( rows );
   for( int i = 0; i < rows; i++ ) {
      bv[ i ] = (Real) b[ i ];
      xv[ i ] = (Real) x[ i ];
   }
   bool ok = false;
   auto run = [ & ]( auto& s )
   {
      s.setMatrix( A );
      s.setOmega( (Real) omega );
      s.setResiduePeriod( period );
      s.setConvergenceResidue( (Real) rtol );
      s.setMaxIterations( (int) maxit );
      ok = s.solve( bv, xv );
      *iters = s.getIterations();
      *residue = (double) s.getResidue();
   };
   if( solver == 5 ) {
      Solvers::Linear::Jacobi< M > s;
      run( s );
   }
   else {
      Solvers::Linear::SOR< M > s;
      run( s );
   }
   for( int i = 0; i < rows; i++ )
      x[ i ] = (double) xv[ i ];
   return ok ? 1 : 0;
}

// Preconditioners::ILUT (ILUT.hpp:33-289) with its factors exposed: L (unit
// diagonal implied) and U (rows stored in reverse order) as TNL builds them,
// capacity slots included (column -1 where unused)
struct IlutBase
{
   virtual ~IlutBase() = default;
   virtual void factors( int* Loff, int* Lcol, double* Lval, int* Uoff, int* Ucol, double* Uval ) const = 0;
   virtual long long sizeL() const = 0;
   virtual long long sizeU() const = 0;
   virtual void solve( const double* b, double* x ) const = 0;
};

template< typename Real >
struct IlutImpl : IlutBase
{
   using M = Mat< Real, CSRSeg >;
   struct Access : Solvers::Linear::Preconditioners::ILUT< M >
   {
      using Solvers::Linear::Preconditioners::ILUT< M >::L;
      using Solvers::Linear::Preconditioners::ILUT< M >::U;
   };
   std::shared_ptr< M > A;
   Access pre;
   int n = 0;

   IlutImpl( int rows, const int* offsets, const int* columns, const double* values, int p, double tau )
   {
      n = rows;
      A = std::make_shared< M >( makeCsr< Real >( rows, rows, offsets, columns, values ) );
      Config::ParameterContainer params;
      params.addParameter< int >( "ilut-p", p );
      params.addParameter< double >( "ilut-threshold", tau );
      pre.setup( params );
      pre.update( A );
   }
   long long sizeL() const override { return pre.L.getValues().getSize(); }
   long long sizeU() const override { return pre.U.getValues().getSize(); }
   void
   factors( int* Loff, int* Lcol, double* Lval, int* Uoff, int* Ucol, double* Uval ) const override
   {
      auto put = []( const auto& F, int* off, int* col, double* val )
      {
         const auto& o = F.getSegments().getOffsets();
         for( int i = 0; i < o.getSize(); i++ )
            off[ i ] = o[ i ];
         for( int k = 0; k < F.getValues().getSize(); k++ ) {
            col[ k ] = F.getColumnIndexes()[ k ];
            val[ k ] = (double) F.getValues()[ k ];
         }
      };
      put( pre.L, Loff, Lcol, Lval );
      put( pre.U, Uoff, Ucol, Uval );
   }
   void
   solve( const double* b, double* x ) const override
   {
      Containers::Vector< Real, Host, int > bv( n ), xv( n );
      for( int i = 0; i < n; i++ )
         bv[ i ] = (Real) b[ i ];
      pre.solve( bv.getConstView(), xv.getView() );
      for( int i = 0; i < n; i++ )
         x[ i ] = (double) xv[ i ];
   }
};

// Preconditioners::ILU0< CSR matrix >::update( A ) then solve( b, x ): x = U^-1 L^-1 b
// (Solvers/Linear/Preconditioners/ILU0.hpp:23-144)
template< typename Real >
static void
iluApply( int rows, const int* offsets, const int* columns, const double* values, const double* b, double* x )
{
   using M = Mat< Real, CSRSeg >;
   auto A = std::make_shared< M >( makeCsr< Real >( rows, rows, offsets, columns, values ) );
   Solvers::Linear::Preconditioners::ILU0< M > pre;
   pre.update( A );
   Containers::Vector< Real, Host, int > bv( rows ), xv( rows );
   for( int i = 0; i < rows; i++ )
      bv[ i ] = (Real) b[ i ];
   pre.solve( bv.getConstView(), xv.getView() );
   for( int i = 0; i < rows; i++ )
      x[ i ] = (double) xv[ i ];
}

// ---------------------------------------------------------------------------
// SparseMatrix< Real, Host, int, SymmetricMatrix, CSR >: the lower triangle given
// as CSR; y = alpha A x + beta y over rows [begin, end) (SparseMatrixView.hpp:413-476)
template< typename Real >
static int
symmetricSpmv( int rows, const int* offsets, const int* columns, const double* values, const double* x, double* y,
               double alpha, double beta, int begin, int end )
{
   using S = Matrices::SparseMatrix< Real, Host, int, Matrices::SymmetricMatrix, CSRSeg >;
   S A( rows, rows );
   Containers::Vector< int, Host, int > caps( rows );
   for( int i = 0; i < rows; i++ )
      caps[ i ] = offsets[ i + 1 ] - offsets[ i ];
   A.setRowCapacities( caps );
   auto& v = A.getValues();
   auto& c = A.getColumnIndexes();
   for( long long k = 0; k < offsets[ rows ]; k++ ) {
      v[ k ] = (Real) values[ k ];
      c[ k ] = columns[ k ];
   }
   Containers::Vector< Real, Host, int > xv( rows ), yv( rows );
   for( int i = 0; i < rows; i++ ) {
      xv[ i ] = (Real) x[ i ];
      yv[ i ] = (Real) y[ i ];
   }
   A.vectorProduct( xv, yv, (Real) alpha, (Real) beta, begin, end );
   for( int i = 0; i < rows; i++ )
      y[ i ] = (double) yv[ i ];
   return 0;
}


extern "C" {

void
tnlref_set_threads( int n )
{
   if( n > 0 )
      omp_set_num_threads( n );
}

int
tnlref_get_threads( void )
{
   return omp_get_max_threads();
}

// format: 0 CSR (as given), 1 Ellpack, 2 SlicedEllpack(32), 3 ChunkedEllpack,
//         4 BiEllpack(32), 5/6/7 SlicedEllpack with SliceSize 8/16/64
// org: 0 ColumnMajorOrder (TNL's Devices::Cuda default), 1 RowMajorOrder (Host default)
// real: 0 double, 1 float, 2 bool (binary matrix, formats 0-4, assigned from the CSR)
void*
tnlref_create( int format, int org, int real, int rows, int cols, const int* offsets, const int* columns, const double* values )
{
   try {
      if( real == 0 )
         return dispatch< double >( format, org, rows, cols, offsets, columns, values );
      if( real == 2 )
         return dispatchBinary( format, org, rows, cols, offsets, columns, values );
      return dispatch< float >( format, org, rows, cols, offsets, columns, values );
   }
   catch( ... ) {
      return nullptr;
   }
}

// y = alpha A x + beta y with float vectors for a binary matrix (real == 2 in tnlref_create)
int
tnlref_binary_spmv_f32( void* h, const float* x, float* y, double alpha, double beta, int begin, int end )
{
   try {
      MatrixBase* m = static_cast< MatrixBase* >( h );
      if( binaryProductF32< CSRSeg >( m, x, y, alpha, beta, begin, end )
          || binaryProductF32< EllCol >( m, x, y, alpha, beta, begin, end )
          || binaryProductF32< SEllCol >( m, x, y, alpha, beta, begin, end )
          || binaryProductF32< CEllCol >( m, x, y, alpha, beta, begin, end )
          || binaryProductF32< BEllCol >( m, x, y, alpha, beta, begin, end ) )
         return 0;
      return -1;
   }
   catch( ... ) {
      return -1;
   }
}

void
tnlref_destroy( void* h )
{
   delete static_cast< MatrixBase* >( h );
}

long long
tnlref_storage_size( void* h )
{
   return static_cast< MatrixBase* >( h )->storageSize();
}

void
tnlref_export_values( void* h, double* out )
{
   static_cast< MatrixBase* >( h )->exportValues( out );
}

void
tnlref_export_columns( void* h, int* out )
{
   static_cast< MatrixBase* >( h )->exportColumns( out );
}

int
tnlref_export_range( void* h, int which, long long first, long long count, void* out )
{
   const MatrixBase* m = static_cast< MatrixBase* >( h );
   if( first < 0 || count < 0 || first + count > m->storageSize() )
      return -1;
   if( which == 0 )
      m->exportValuesRange( static_cast< double* >( out ), first, count );
   else
      m->exportColumnsRange( static_cast< int* >( out ), first, count );
   return 0;
}

int
tnlref_meta_count( void* h )
{
   return (int) static_cast< MatrixBase* >( h )->meta.ints.size();
}

const char*
tnlref_meta_name( void* h, int i )
{
   return static_cast< MatrixBase* >( h )->meta.ints[ i ].first.c_str();
}

long long
tnlref_meta_size( void* h, int i )
{
   return (long long) static_cast< MatrixBase* >( h )->meta.ints[ i ].second.size();
}

void
tnlref_meta_get( void* h, int i, long long* out )
{
   const auto& v = static_cast< MatrixBase* >( h )->meta.ints[ i ].second;
   std::memcpy( out, v.data(), v.size() * sizeof( long long ) );
}

int
tnlref_spmv( void* h, const double* x, double* y, double alpha, double beta, int begin, int end )
{
   try {
      static_cast< MatrixBase* >( h )->spmv( x, y, alpha, beta, begin, end );
      return 0;
   }
   catch( ... ) {
      return -1;
   }
}

double
tnlref_spmv_time( void* h, const double* x, int loops )
{
   return static_cast< MatrixBase* >( h )->timeSpmv( x, loops );
}

int
tnlref_spmv_symmetric( int real, int rows, const int* offsets, const int* columns, const double* values, const double* x,
                       double* y, double alpha, double beta, int begin, int end )
{
   try {
      if( real == 0 )
         return symmetricSpmv< double >( rows, offsets, columns, values, x, y, alpha, beta, begin, end );
      return symmetricSpmv< float >( rows, offsets, columns, values, x, y, alpha, beta, begin, end );
   }
   catch( ... ) {
      return -1;
   }
}

// solver: 0 CG, 1 BiCGStab, 2 GMRES, 3 TFQMR, 4 BiCGStab(ell); precond: 0 none, 1 Jacobi (Diagonal), 2 ILU0,
// 3 ILUT (parameters from tnlref_set_ilut)
int
tnlref_solve( int solver,
              int precond,
              int real,
              int rows,
              const int* offsets,
              const int* columns,
              const double* values,
              const double* b,
              double* x,
              double rtol,
              long long maxit,
              const char* gmresVariant,
              int restartMin,
              int restartMax,
              int exactResidue,
              int ell,
              long long* iters,
              double* residue,
              double* seconds )
{
   try {
      if( real == 0 )
         return solveImpl< double >( solver, precond, rows, offsets, columns, values, b, x, rtol, maxit, gmresVariant,
                                     restartMin, restartMax, exactResidue, ell, iters, residue, seconds );
      return solveImpl< float >( solver, precond, rows, offsets, columns, values, b, x, rtol, maxit, gmresVariant,
                                 restartMin, restartMax, exactResidue, ell, iters, residue, seconds );
   }
   catch( ... ) {
      return -1;
   }
}

// MultidiagonalMatrix: real 0 FP64 / 1 FP32, org 0 RowMajor / 1 ColumnMajor;
// NULL when TNL throws
void*
tnlref_mdiag_create( int real, int org, int rows, int cols, int nd, const int* offsets, const double* vals )
{
   using Seg = Algorithms::Segments::ElementsOrganization;
   try {
      if( real == 0 )
         return org ? (MdiagBase*) new MdiagImpl< double, Seg::ColumnMajorOrder >( rows, cols, nd, offsets, vals )
                    : (MdiagBase*) new MdiagImpl< double, Seg::RowMajorOrder >( rows, cols, nd, offsets, vals );
      return org ? (MdiagBase*) new MdiagImpl< float, Seg::ColumnMajorOrder >( rows, cols, nd, offsets, vals )
                 : (MdiagBase*) new MdiagImpl< float, Seg::RowMajorOrder >( rows, cols, nd, offsets, vals );
   }
   catch( ... ) {
      return nullptr;
   }
}

long long
tnlref_mdiag_storage( void* h )
{
   return static_cast< MdiagBase* >( h )->storage();
}

void
tnlref_mdiag_values( void* h, double* out )
{
   static_cast< MdiagBase* >( h )->values( out );
}

void
tnlref_mdiag_spmv( void* h, const double* x, double* y, double alpha, double beta, int begin, int end )
{
   static_cast< MdiagBase* >( h )->spmv( x, y, alpha, beta, begin, end );
}

void
tnlref_mdiag_destroy( void* h )
{
   delete static_cast< MdiagBase* >( h );
}

// ilut-p and ilut-threshold of the solves with precond 3 (ILUT)
void
tnlref_set_ilut( int p, double tau )
{
   g_ilut_p = p;
   g_ilut_tau = tau;
}

// solver: 5 Jacobi, 6 SOR (one OpenMP thread makes SOR's sweep TNL's sequential one)
int
tnlref_solve_stationary( int solver, int real, int rows, const int* offsets, const int* columns, const double* values,
                         const double* b, double* x, double rtol, long long maxit, double omega, int period,
                         long long* iters, double* residue )
{
   try {
      if( real == 0 )
         return stationaryImpl< double >( solver, rows, offsets, columns, values, b, x, rtol, maxit, omega, period, iters,
                                          residue );
      return stationaryImpl< float >( solver, rows, offsets, columns, values, b, x, rtol, maxit, omega, period, iters,
                                      residue );
   }
   catch( ... ) {
      return -1;
   }
}

// ILUT: update( A ) with ilut-p and ilut-threshold; NULL when TNL throws
void*
tnlref_ilut_create( int real, int rows, const int* offsets, const int* columns, const double* values, int p, double tau )
{
   try {
      if( real == 0 )
         return new IlutImpl< double >( rows, offsets, columns, values, p, tau );
      return new IlutImpl< float >( rows, offsets, columns, values, p, tau );
   }
   catch( ... ) {
      return nullptr;
   }
}

void
tnlref_ilut_sizes( void* h, long long* nL, long long* nU )
{
   *nL = static_cast< IlutBase* >( h )->sizeL();
   *nU = static_cast< IlutBase* >( h )->sizeU();
}

void
tnlref_ilut_factors( void* h, int* Loff, int* Lcol, double* Lval, int* Uoff, int* Ucol, double* Uval )
{
   static_cast< IlutBase* >( h )->factors( Loff, Lcol, Lval, Uoff, Ucol, Uval );
}

void
tnlref_ilut_solve( void* h, const double* b, double* x )
{
   static_cast< IlutBase* >( h )->solve( b, x );
}

void
tnlref_ilut_destroy( void* h )
{
   delete static_cast< IlutBase* >( h );
}

// Matrices/MatrixPermutationApplier.h:17-62: new row i = old row perm[i]
int
tnlref_permute_rows( void* h, const int* perm )
{
   try {
      static_cast< MatrixBase* >( h )->permuteRows( perm );
      return 0;
   }
   catch( ... ) {
      return -1;
   }
}

// Matrices/MatrixPermutationApplier.h:64-90: column c -> iperm[c], slots unchanged
int
tnlref_permute_columns( void* h, const int* iperm )
{
   try {
      static_cast< MatrixBase* >( h )->permuteColumns( iperm );
      return 0;
   }
   catch( ... ) {
      return -1;
   }
}

// setRowCapacities( rowCaps, or the triplet counts when NULL ) + setElement
// (add = 0) / addElement( .., 1 ) (add = 1) for every triplet in order; NULL
// when TNL throws
void*
tnlref_from_coo( int format, int org, int real, int rows, int cols, long long n, const int* ri, const int* ci,
                 const double* v, int add, const int* rowCaps )
{
   try {
      FromCoo f{ rows, cols, n, ri, ci, v, add, rowCaps };
      return real == 0 ? withLayout< double >( format, org, f ) : withLayout< float >( format, org, f );
   }
   catch( ... ) {
      return nullptr;
   }
}

// MatrixReader< Matrix >::readMtx( path, matrix ); NULL when TNL throws
void*
tnlref_read_mtx( int format, int org, int real, const char* path )
{
   try {
      ReadMtx f{ path };
      return real == 0 ? withLayout< double >( format, org, f ) : withLayout< float >( format, org, f );
   }
   catch( ... ) {
      return nullptr;
   }
}

// SparseMatrix::operator=( other layout ); NULL when TNL throws
void*
tnlref_convert( void* h, int format, int org )
{
   try {
      return static_cast< MatrixBase* >( h )->convertTo( format, org );
   }
   catch( ... ) {
      return nullptr;
   }
}

int
tnlref_save( void* h, const char* path )
{
   try {
      static_cast< MatrixBase* >( h )->save( path );
      return 0;
   }
   catch( ... ) {
      return -1;
   }
}

// SparseMatrix::load( fileName ); NULL when TNL throws (e.g. another type in the file)
void*
tnlref_load( int format, int org, int real, const char* path )
{
   try {
      LoadFile f{ path };
      return real == 0 ? withLayout< double >( format, org, f ) : withLayout< float >( format, org, f );
   }
   catch( ... ) {
      return nullptr;
   }
}

// MatrixWriter< Matrix >::writeMtx( path, matrix )
int
tnlref_write_mtx( void* h, const char* path )
{
   try {
      static_cast< MatrixBase* >( h )->writeMtx( path );
      return 0;
   }
   catch( ... ) {
      return -1;
   }
}

int
tnlref_ilu0_apply( int real, int rows, const int* offsets, const int* columns, const double* values, const double* b,
                   double* x )
{
   try {
      if( real == 0 )
         iluApply< double >( rows, offsets, columns, values, b, x );
      else
         iluApply< float >( rows, offsets, columns, values, b, x );
      return 0;
   }
   catch( ... ) {
      return -1;
   }
}

// Matrices/SparseOperations_impl.h:253-312 reorderSparseMatrix on a host CSR
// matrix: row i of the result = row perm[i], columns mapped by iperm and sorted
void*
tnlref_reorder( int rows, int cols, const int* offsets, const int* columns, const double* values, const int* perm,
                const int* iperm )
{
   try {
      auto src = makeCsr< double >( rows, cols, offsets, columns, values );
      auto* M = new MatrixImpl< double, CSRSeg >();
      M->rows = rows;
      M->cols = cols;
      Containers::Array< int, Host, int > p( rows ), ip( cols );
      for( int i = 0; i < rows; i++ )
         p[ i ] = perm[ i ];
      for( int i = 0; i < cols; i++ )
         ip[ i ] = iperm[ i ];
      Matrices::reorderSparseMatrix( src, M->A, p, ip );
      M->recapture();
      return M;
   }
   catch( ... ) {
      return nullptr;
   }
}

}  // extern "C"
