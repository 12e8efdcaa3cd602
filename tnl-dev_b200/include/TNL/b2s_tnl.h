// TNL-shaped C++ front end of libb2sparse (header only).
//
// Existing code written against TNL's sparse path —
//   TNL::Matrices::SparseMatrix< Real, Devices::Cuda, Index, GeneralMatrix, Segments >
//   TNL::Solvers::Linear::{CG, BICGStab, GMRES}< Matrix >, Preconditioners::Diagonal
//   TNL::Containers::Vector< Real, Devices::Cuda, Index >, Config::ParameterContainer
// — compiles against these headers and runs on the B200 kernels through the C
// ABI of include/b2s.h. Only the part of TNL's interface that the sparse hot
// path uses is provided. Errors become the exceptions TNL throws
// (Exceptions::CudaBadAlloc, Exceptions::CudaRuntimeError, std::logic_error);
// solve() returns false on non-convergence as TNL's does.
#pragma once

#include <b2s.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <initializer_list>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

namespace TNL {

// ---------------------------------------------------------------------------
namespace Devices {
struct Host
{};
struct Cuda
{};
}  // namespace Devices

namespace Exceptions {
struct CudaBadAlloc : std::bad_alloc
{
   const char* what() const noexcept override { return "Failed to allocate memory on the CUDA device."; }
};
struct CudaRuntimeError : std::runtime_error
{
   using std::runtime_error::runtime_error;
};
}  // namespace Exceptions

namespace detail {
inline void
check( b2s_status s, const char* where )
{
   if( s == B2S_OK )
      return;
   if( s == B2S_OOM )
      throw Exceptions::CudaBadAlloc();
   const std::string msg = std::string( where ) + ": " + b2s_status_string( s ) + " " + b2s_last_error();
   if( s == B2S_CUDA_ERROR || s == B2S_TIMEOUT )
      throw Exceptions::CudaRuntimeError( msg );
   throw std::logic_error( msg );
}
inline void
check_cuda( cudaError_t e )
{
   if( e == cudaErrorMemoryAllocation )
      throw Exceptions::CudaBadAlloc();
   if( e != cudaSuccess )
      throw Exceptions::CudaRuntimeError( cudaGetErrorString( e ) );
}
template< typename Real >
constexpr b2s_dtype
dtype_of()
{
   static_assert( std::is_same< Real, double >::value || std::is_same< Real, float >::value
                     || std::is_same< Real, bool >::value,
                  "libb2sparse supports Real = double, float or bool (binary matrices)" );
   return std::is_same< Real, double >::value ? B2S_F64 : ( std::is_same< Real, bool >::value ? B2S_BOOL : B2S_F32 );
}
}  // namespace detail

// ---------------------------------------------------------------------------
// Containers::Vector< Real, Device, Index > (Containers/Vector.h:39)
namespace Containers {

template< typename Real, typename Device = Devices::Host, typename Index = int >
class Vector
{
public:
   using RealType = Real;
   using DeviceType = Device;
   using IndexType = Index;
   static constexpr bool onDevice = std::is_same< Device, Devices::Cuda >::value;

   Vector() = default;
   explicit Vector( Index size ) { setSize( size ); }
   Vector( Index size, Real value )
   {
      setSize( size );
      setValue( value );
   }
   Vector( std::initializer_list< Real > l )
   {
      setSize( (Index) l.size() );
      std::vector< Real > h( l );
      upload( h.data() );
   }
   Vector( const Vector& o ) { *this = o; }
   Vector& operator=( const Vector& o )
   {
      if( this != &o ) {
         setSize( o.size_ );
         if( size_ > 0 ) {
            if( onDevice )
               detail::check_cuda( cudaMemcpy( data_, o.data_, bytes(), cudaMemcpyDeviceToDevice ) );
            else
               std::copy( o.host_.begin(), o.host_.end(), host_.begin() );
         }
      }
      return *this;
   }
   template< typename D2 >
   Vector& operator=( const Vector< Real, D2, Index >& o )
   {
      setSize( o.getSize() );
      std::vector< Real > h = o.toStdVector();
      upload( h.data() );
      return *this;
   }
   ~Vector() { reset(); }

   void setSize( Index n )
   {
      if( n == size_ )
         return;
      reset();
      size_ = n;
      if( n <= 0 )
         return;
      if( onDevice )
         detail::check_cuda( cudaMalloc( &data_, bytes() ) );
      else {
         host_.assign( n, Real( 0 ) );
         data_ = host_.data();
      }
   }
   template< typename V >
   void setLike( const V& v ) { setSize( v.getSize() ); }
   void reset()
   {
      if( onDevice && data_ )
         cudaFree( data_ );
      host_.clear();
      data_ = nullptr;
      size_ = 0;
   }
   Index getSize() const { return size_; }
   Real* getData() { return data_; }
   const Real* getData() const { return data_; }
   void setValue( Real v )
   {
      std::vector< Real > h( size_, v );
      upload( h.data() );
   }
   Vector& operator=( Real v )
   {
      setValue( v );
      return *this;
   }
   void setElement( Index i, Real v )
   {
      if( onDevice )
         detail::check_cuda( cudaMemcpy( data_ + i, &v, sizeof( Real ), cudaMemcpyHostToDevice ) );
      else
         host_[ i ] = v;
   }
   Real getElement( Index i ) const
   {
      if( ! onDevice )
         return host_[ i ];
      Real v;
      detail::check_cuda( cudaMemcpy( &v, data_ + i, sizeof( Real ), cudaMemcpyDeviceToHost ) );
      return v;
   }
   Real& operator[]( Index i )
   {
      static_assert( ! onDevice, "operator[] is host-only; use getElement/setElement" );
      return host_[ i ];
   }
   const Real& operator[]( Index i ) const
   {
      static_assert( ! onDevice, "operator[] is host-only; use getElement/setElement" );
      return host_[ i ];
   }
   std::vector< Real > toStdVector() const
   {
      std::vector< Real > h( size_ );
      if( size_ > 0 ) {
         if( onDevice )
            detail::check_cuda( cudaMemcpy( h.data(), data_, bytes(), cudaMemcpyDeviceToHost ) );
         else
            h = host_;
      }
      return h;
   }
   void upload( const Real* h )
   {
      if( size_ <= 0 )
         return;
      if( onDevice )
         detail::check_cuda( cudaMemcpy( data_, h, bytes(), cudaMemcpyHostToDevice ) );
      else
         std::copy( h, h + size_, host_.begin() );
   }
   const Vector& getConstView() const { return *this; }
   Vector& getView() { return *this; }

private:
   size_t bytes() const { return (size_t) size_ * sizeof( Real ); }
   Real* data_ = nullptr;
   Index size_ = 0;
   std::vector< Real > host_;
};

template< typename Real, typename Device = Devices::Host, typename Index = int >
using VectorView = Vector< Real, Device, Index >;

}  // namespace Containers

// ---------------------------------------------------------------------------
// Segment tags (Algorithms/Segments/*.h). Only their identity matters here:
// each selects a layout of libb2sparse.
namespace Algorithms {
namespace Segments {
template< typename Device, typename Index, typename Alloc = void >
struct CSRScalar
{
   static constexpr b2s_format format = B2S_CSR;
   static constexpr b2s_csr_kernel kernel = B2S_CSR_SCALAR;
};
template< typename Device, typename Index, typename Alloc = void >
struct CSRVector
{
   static constexpr b2s_format format = B2S_CSR;
   static constexpr b2s_csr_kernel kernel = B2S_CSR_VECTOR;
};
template< typename Device, typename Index, typename Alloc = void >
using CSRLight = CSRVector< Device, Index, Alloc >;
template< typename Device, typename Index, typename Alloc = void >
using CSRHybrid = CSRVector< Device, Index, Alloc >;
template< typename Device, typename Index, typename Alloc = void >
struct CSRAdaptive
{
   static constexpr b2s_format format = B2S_CSR;
   static constexpr b2s_csr_kernel kernel = B2S_CSR_ADAPTIVE;
};
template< typename Device, typename Index, typename Alloc = void >
struct CSRDefault
{
   static constexpr b2s_format format = B2S_CSR;
   static constexpr b2s_csr_kernel kernel = B2S_CSR_AUTO;
};
template< typename Device, typename Index, typename Alloc = void >
using CSR = CSRDefault< Device, Index, Alloc >;
template< typename Device, typename Index, typename Alloc = void >
struct Ellpack
{
   static constexpr b2s_format format = B2S_ELLPACK;
   static constexpr b2s_csr_kernel kernel = B2S_CSR_AUTO;
};
template< typename Device, typename Index, typename Alloc = void >
struct SlicedEllpack
{
   static constexpr b2s_format format = B2S_SLICED_ELLPACK;
   static constexpr b2s_csr_kernel kernel = B2S_CSR_AUTO;
};
template< typename Device, typename Index, typename Alloc = void >
struct ChunkedEllpack
{
   static constexpr b2s_format format = B2S_CHUNKED_ELLPACK;
   static constexpr b2s_csr_kernel kernel = B2S_CSR_AUTO;
};
template< typename Device, typename Index, typename Alloc = void >
struct BiEllpack
{
   static constexpr b2s_format format = B2S_BIELLPACK;
   static constexpr b2s_csr_kernel kernel = B2S_CSR_AUTO;
};
}  // namespace Segments
}  // namespace Algorithms

// ---------------------------------------------------------------------------
namespace Matrices {

struct GeneralMatrix
{
   static constexpr bool isSymmetric() { return false; }
};
// Matrices/MatrixType.h: a symmetric matrix stores its lower triangle; (i, j)
// with i < j is set, added and read at (j, i) (SparseMatrixView.hpp:285-289, 360-364)
struct SymmetricMatrix
{
   static constexpr bool isSymmetric() { return true; }
};

// SparseMatrix< Real, Devices::Cuda, Index, GeneralMatrix, Segments >
// (Matrices/SparseMatrix.h:40-49). Assembly follows TNL: setDimensions,
// setRowCapacities, setElement / addElement (sorted insert into the row,
// capacity-checked). The device matrix is (re)built when it is first used
// after a change.
template< typename Real,
          typename Device = Devices::Cuda,
          typename Index = int,
          typename MatrixType = GeneralMatrix,
          template< typename, typename, typename > class Segments = Algorithms::Segments::CSRDefault >
class SparseMatrix
{
   static_assert( std::is_same< Index, int >::value, "libb2sparse uses 32-bit indices" );
   using SegTag = Segments< Device, Index, void >;

public:
   using RealType = Real;
   using DeviceType = Device;
   using IndexType = Index;
   // a binary matrix computes in Index (SparseMatrixView.h:22-30)
   using ComputeRealType = typename std::conditional< std::is_same< Real, bool >::value, Index, Real >::type;
   using RowsCapacitiesType = Containers::Vector< Index, Devices::Host, Index >;

   static constexpr bool isBinary() { return std::is_same< Real, bool >::value; }

   SparseMatrix() = default;
   SparseMatrix( Index rows, Index columns ) { setDimensions( rows, columns ); }
   SparseMatrix( const SparseMatrix& o ) { *this = o; }
   SparseMatrix& operator=( const SparseMatrix& o )
   {
      rows_ = o.rows_;
      cols_ = o.cols_;
      caps_ = o.caps_;
      entries_ = o.entries_;
      dirty_ = true;
      handle_.reset();
      return *this;
   }
   // SparseMatrix::operator=( const RHSMatrix& ) (SparseMatrix.hpp:1069-1193): conversion
   // between layouts; the padded layouts drop explicit zeros exactly as TNL does.
   template< typename R2, typename D2, typename I2, typename M2, template< typename, typename, typename > class S2 >
   SparseMatrix& operator=( const SparseMatrix< R2, D2, I2, M2, S2 >& o )
   {
      rows_ = o.getRows();
      cols_ = o.getColumns();
      o.exportAssembly( caps_, entries_ );
      dirty_ = true;
      handle_.reset();
      return *this;
   }

   void setDimensions( Index rows, Index columns )
   {
      rows_ = rows;
      cols_ = columns;
      caps_.assign( rows, 0 );
      entries_.assign( rows, {} );
      dirty_ = true;
   }
   template< typename CapsVector >
   void setRowCapacities( const CapsVector& caps )
   {
      if( caps.getSize() != rows_ )
         throw std::logic_error( "Number of matrix rows does not fit with rowCapacities vector size." );
      for( Index i = 0; i < rows_; i++ )
         caps_[ i ] = caps.getElement( i );
      entries_.assign( rows_, {} );
      dirty_ = true;
   }
   void setRowCapacities( std::initializer_list< Index > caps )
   {
      RowsCapacitiesType v( caps.size() );
      Index i = 0;
      for( Index c : caps )
         v[ i++ ] = c;
      setRowCapacities( v );
   }
   // SparseMatrixView::setElement / addElement (SparseMatrixView.hpp:274-340)
   void setElement( Index row, Index column, Real value ) { addElement( row, column, value, Real( 0 ) ); }
   void addElement( Index row, Index column, Real value, Real thisElementMultiplicator = 1 )
   {
      if( MatrixType::isSymmetric() && row < column )
         std::swap( row, column );
      auto& r = entries_.at( row );
      auto it = std::lower_bound( r.begin(), r.end(), column,
                                  []( const std::pair< Index, Real >& e, Index c ) { return e.first < c; } );
      if( it != r.end() && it->first == column )
         it->second = thisElementMultiplicator * it->second + value;
      else {
         if( (Index) r.size() >= caps_[ row ] )
            throw std::logic_error( "Cannot add element - row " + std::to_string( row ) + " is completely full." );
         r.insert( it, { column, value } );
      }
      dirty_ = true;
   }
   Real getElement( Index row, Index column ) const
   {
      if( MatrixType::isSymmetric() && row < column )
         std::swap( row, column );
      for( const auto& e : entries_.at( row ) )
         if( e.first == column )
            return e.second;
      return Real( 0 );
   }
   Index getRows() const { return rows_; }
   Index getColumns() const { return cols_; }
   Index getNonzeroElementsCount() const
   {
      Index n = 0;
      for( Index r = 0; r < rows_; r++ )
         for( const auto& e : entries_[ r ] )
            if( isBinary() || e.second != Real( 0 ) )  // a binary matrix's stored elements are all ones
               n += MatrixType::isSymmetric() && e.first != r ? 2 : 1;  // both triangles of a symmetric matrix
      return n;
   }
   int64_t getStorageSize() const
   {
      b2s_matrix_info info;
      detail::check( b2s_matrix_get_info( handle(), &info ), "b2s_matrix_get_info" );
      return info.storage_size;
   }
   template< typename Vec >
   void getRowCapacities( Vec& caps ) const
   {
      caps.setSize( rows_ );
      for( Index i = 0; i < rows_; i++ )
         caps.setElement( i, caps_[ i ] );
   }

   // vectorProduct( in, out, matrixMultiplicator, outVectorMultiplicator, begin, end )
   // (Matrices/SparseMatrix.h:1078-1085)
   template< typename InVector, typename OutVector >
   void vectorProduct( const InVector& in,
                       OutVector& out,
                       ComputeRealType matrixMultiplicator = 1.0,
                       ComputeRealType outVectorMultiplicator = 0.0,
                       Index begin = 0,
                       Index end = 0 ) const
   {
      if( in.getSize() != cols_ )
         throw std::logic_error( "Matrix columns do not fit with input vector." );
      if( out.getSize() != rows_ )
         throw std::logic_error( "Matrix rows do not fit with output vector." );
      static_assert( std::is_same< typename InVector::RealType, typename OutVector::RealType >::value,
                     "in and out vectors of one value type" );
      constexpr bool dev = std::is_same< typename OutVector::DeviceType, Devices::Cuda >::value;
      // a binary matrix takes double or float vectors; a real one its own type
      detail::check( b2s_spmv_ex( handle(), in.getData(), out.getData(), detail::dtype_of< typename InVector::RealType >(),
                                  (double) matrixMultiplicator, (double) outVectorMultiplicator, begin, end,
                                  dev ? B2S_DEVICE : B2S_HOST, nullptr ),
                     "vectorProduct" );
      if( dev )
         detail::check_cuda( cudaStreamSynchronize( nullptr ) );
   }

   b2s_matrix handle() const
   {
      if( dirty_ || ! handle_ ) {
         // the assembled rows go to the device as triplets with the row
         // capacities: setRowCapacities + setElement there (explicit zeros
         // kept, unused slots of the padded layouts left as padding)
         std::vector< int32_t > ri, ci;
         std::vector< double > val;
         for( Index r = 0; r < rows_; r++ )
            for( const auto& e : entries_[ r ] ) {
               ri.push_back( r );
               ci.push_back( e.first );
               val.push_back( (double) e.second );
            }
         b2s_matrix_opts opts;
         b2s_matrix_opts_default( &opts );
         opts.csr_kernel = SegTag::kernel;
         opts.symmetric = MatrixType::isSymmetric() ? 1 : 0;
         b2s_matrix m = nullptr;
         detail::check( b2s_matrix_from_coo( SegTag::format, detail::dtype_of< Real >(), rows_, cols_, (int64_t) ri.size(),
                                             ri.data(), ci.data(), val.data(), B2S_F64, B2S_HOST, B2S_DUP_SET,
                                             caps_.data(), &opts, nullptr, &m ),
                        "b2s_matrix_from_coo" );
         handle_.reset( m, []( b2s_matrix p ) { b2s_matrix_destroy( p ); } );
         dirty_ = false;
      }
      return handle_.get();
   }

   // SparseMatrix::save / load( fileName ) (Matrices/SparseMatrix.hpp:1264-1290): TNL's binary file
   void save( const std::string& fileName ) const
   {
      detail::check( b2s_matrix_save( handle(), fileName.c_str() ), "b2s_matrix_save" );
   }
   void load( const std::string& fileName )
   {
      b2s_matrix m = nullptr;
      detail::check( b2s_matrix_load( fileName.c_str(), nullptr, nullptr, &m ), "b2s_matrix_load" );
      std::shared_ptr< b2s_matrix_t > loaded( m, []( b2s_matrix p ) { b2s_matrix_destroy( p ); } );
      b2s_matrix_info info;
      detail::check( b2s_matrix_get_info( m, &info ), "b2s_matrix_get_info" );
      if( info.format != SegTag::format || info.dtype != detail::dtype_of< Real >() )
         throw std::runtime_error( "the file holds another matrix type" );
      // the rows as CSR (no padding), kept as this matrix's assembled entries
      b2s_matrix csr = m;
      std::shared_ptr< b2s_matrix_t > conv;
      if( info.format != B2S_CSR ) {
         detail::check( b2s_matrix_convert( m, B2S_CSR, (b2s_dtype) info.dtype, nullptr, nullptr, &csr ), "b2s_matrix_convert" );
         conv.reset( csr, []( b2s_matrix p ) { b2s_matrix_destroy( p ); } );
      }
      int64_t n = 0;
      detail::check( b2s_matrix_export( csr, "offsets", nullptr, 0, &n ), "export" );
      std::vector< int64_t > off( (size_t) n );
      detail::check( b2s_matrix_export( csr, "offsets", off.data(), n, &n ), "export" );
      detail::check( b2s_matrix_export( csr, "columnIndexes", nullptr, 0, &n ), "export" );
      std::vector< int32_t > col( (size_t) std::max< int64_t >( n, 1 ) );
      std::vector< Real > val( (size_t) std::max< int64_t >( n, 1 ) );
      detail::check( b2s_matrix_export( csr, "columnIndexes", col.data(), n, &n ), "export" );
      detail::check( b2s_matrix_export( csr, "values", val.data(), n, &n ), "export" );
      rows_ = info.rows;
      cols_ = info.cols;
      caps_.assign( rows_, 0 );
      entries_.assign( rows_, {} );
      for( Index r = 0; r < rows_; r++ ) {
         caps_[ r ] = (Index) ( off[ r + 1 ] - off[ r ] );
         for( int64_t k = off[ r ]; k < off[ r + 1 ]; k++ )
            entries_[ r ].emplace_back( col[ k ], val[ k ] );
      }
      handle_ = loaded;  // the loaded layout itself serves the products
      dirty_ = false;
   }

   void exportAssembly( std::vector< Index >& caps, std::vector< std::vector< std::pair< Index, Real > > >& e ) const
   {
      caps = caps_;
      e = entries_;
   }

private:
   Index rows_ = 0, cols_ = 0;
   std::vector< Index > caps_;
   std::vector< std::vector< std::pair< Index, Real > > > entries_;
   mutable bool dirty_ = true;
   mutable std::shared_ptr< b2s_matrix_t > handle_;
};

// MatrixReader< Matrix >::readMtx (Matrices/MatrixReader.hpp:21-359): the
// file is parsed by the library with TNL's checks and messages, then
// assembled through setRowCapacities + setElement.
template< typename Matrix, typename Device = typename Matrix::DeviceType >
class MatrixReader
{
public:
   static void readMtx( const std::string& fileName, Matrix& matrix, bool verbose = false )
   {
      (void) verbose;
      b2s_mtx* f = nullptr;
      const b2s_status st = b2s_mtx_read( fileName.c_str(), &f );
      if( st != B2S_OK )
         throw std::runtime_error( b2s_last_error() );
      std::unique_ptr< b2s_mtx, void ( * )( b2s_mtx* ) > guard( f, b2s_mtx_free );
      using Index = typename Matrix::IndexType;
      using Real = typename Matrix::RealType;
      matrix.setDimensions( f->rows, f->cols );
      typename Matrix::RowsCapacitiesType caps( f->rows );
      for( Index i = 0; i < f->rows; i++ )
         caps[ i ] = 0;
      for( int64_t k = 0; k < f->count; k++ )
         caps[ f->row_indexes[ k ] ]++;
      matrix.setRowCapacities( caps );
      for( int64_t k = 0; k < f->count; k++ )
         matrix.setElement( f->row_indexes[ k ], f->column_indexes[ k ], (Real) f->values[ k ] );
   }
};

// MatrixWriter< Matrix >::writeMtx (Matrices/MatrixWriter.hpp:103-128)
template< typename Matrix, typename Device = typename Matrix::DeviceType >
class MatrixWriter
{
public:
   static void writeMtx( const std::string& fileName, const Matrix& matrix, bool verbose = false )
   {
      (void) verbose;
      detail::check( b2s_matrix_write_mtx( matrix.handle(), fileName.c_str() ), "b2s_matrix_write_mtx" );
   }
};

// MultidiagonalMatrix< Real, Devices::Cuda, Index > (Matrices/MultidiagonalMatrix.h:27-60):
// the diagonals' offsets (column - row) are fixed by setDimensions and kept
// ascending; setElement / addElement outside them throw as in TNL. Elements
// are staged on the host and the device matrix (format B2S_MULTIDIAGONAL:
// values only, ColumnMajor) is (re)built when it is first used after a change.
template< typename Real = double, typename Device = Devices::Cuda, typename Index = int >
class MultidiagonalMatrix
{
public:
   using RealType = Real;
   using DeviceType = Device;
   using IndexType = Index;

   MultidiagonalMatrix() = default;
   template< typename Offsets >
   MultidiagonalMatrix( Index rows, Index columns, const Offsets& diagonalsOffsets )
   {
      setDimensions( rows, columns, diagonalsOffsets );
   }
   MultidiagonalMatrix( Index rows, Index columns, std::initializer_list< Index > diagonalsOffsets )
   {
      setDimensions( rows, columns, std::vector< Index >( diagonalsOffsets ) );
   }

   template< typename Offsets >
   void setDimensions( Index rows, Index columns, const Offsets& diagonalsOffsets )
   {
      if( rows < 0 || columns < 0 )
         throw std::logic_error( "negative matrix dimensions" );
      rows_ = rows;
      cols_ = columns;
      offsets_.clear();
      for( Index k = 0; k < (Index) diagonalsOffsets.getSize(); k++ )
         offsets_.push_back( (int32_t) diagonalsOffsets[ k ] );
      std::sort( offsets_.begin(), offsets_.end() );
      if( std::adjacent_find( offsets_.begin(), offsets_.end() ) != offsets_.end() )
         throw std::logic_error( "repeated diagonal offset" );
      values_.assign( (size_t) rows_ * offsets_.size(), Real( 0 ) );
      dirty_ = true;
   }
   void setDimensions( Index rows, Index columns, const std::vector< Index >& diagonalsOffsets )
   {
      struct View
      {
         const std::vector< Index >& v;
         Index getSize() const { return (Index) v.size(); }
         Index operator[]( Index k ) const { return v[ k ]; }
      };
      setDimensions( rows, columns, View{ diagonalsOffsets } );
   }

   Index getRows() const { return rows_; }
   Index getColumns() const { return cols_; }
   Index getDiagonalsCount() const { return (Index) offsets_.size(); }
   const std::vector< int32_t >& getDiagonalsOffsets() const { return offsets_; }
   Index getNonzeroElementsCount() const
   {
      Index n = 0;
      for( Index r = 0; r < rows_; r++ )
         for( size_t d = 0; d < offsets_.size(); d++ )
            n += inRange( r, d ) && values_[ (size_t) r * offsets_.size() + d ] != Real( 0 );
      return n;
   }

   void setElement( Index row, Index column, const Real& value )
   {
      values_[ slot( row, column ) ] = value;
      dirty_ = true;
   }
   void addElement( Index row, Index column, const Real& value, const Real& thisElementMultiplicator = 1.0 )
   {
      Real& v = values_[ slot( row, column ) ];
      v = thisElementMultiplicator * v + value;
      dirty_ = true;
   }
   Real getElement( Index row, Index column ) const
   {
      if( row < 0 || row >= rows_ || column < 0 || column >= cols_ )
         throw std::logic_error( "element outside the matrix" );
      const auto it = std::lower_bound( offsets_.begin(), offsets_.end(), (int32_t) ( column - row ) );
      if( it == offsets_.end() || *it != column - row )
         return 0;
      return values_[ (size_t) row * offsets_.size() + ( it - offsets_.begin() ) ];
   }

   // vectorProduct (MultidiagonalMatrixView.hpp:488-528)
   template< typename InVector, typename OutVector >
   void vectorProduct( const InVector& in,
                       OutVector& out,
                       Real matrixMultiplicator = 1.0,
                       Real outVectorMultiplicator = 0.0,
                       Index begin = 0,
                       Index end = 0 ) const
   {
      if( in.getSize() != cols_ )
         throw std::logic_error( "Matrix columns do not fit with input vector." );
      if( out.getSize() != rows_ )
         throw std::logic_error( "Matrix rows do not fit with output vector." );
      constexpr bool dev = std::is_same< typename OutVector::DeviceType, Devices::Cuda >::value;
      detail::check( b2s_spmv_ex( handle(), in.getData(), out.getData(), detail::dtype_of< typename InVector::RealType >(),
                                  (double) matrixMultiplicator, (double) outVectorMultiplicator, begin, end,
                                  dev ? B2S_DEVICE : B2S_HOST, nullptr ),
                     "vectorProduct" );
      if( dev )
         detail::check_cuda( cudaStreamSynchronize( nullptr ) );
   }

   b2s_matrix handle() const
   {
      if( dirty_ || ! handle_ ) {
         // every in-range slot as an element (zeros included): the pattern
         // then names exactly these diagonals
         const size_t nd = offsets_.size();
         std::vector< int32_t > off( (size_t) rows_ + 1, 0 ), col;
         std::vector< double > val;
         for( Index r = 0; r < rows_; r++ ) {
            for( size_t d = 0; d < nd; d++ )
               if( inRange( r, d ) ) {
                  col.push_back( r + offsets_[ d ] );
                  val.push_back( (double) values_[ (size_t) r * nd + d ] );
               }
            off[ r + 1 ] = (int32_t) col.size();
         }
         b2s_matrix m = nullptr;
         detail::check( b2s_matrix_create( B2S_MULTIDIAGONAL, detail::dtype_of< Real >(), rows_, cols_,
                                           (int64_t) col.size(), off.data(), col.data(), val.data(), B2S_F64, B2S_HOST,
                                           nullptr, nullptr, &m ),
                        "b2s_matrix_create" );
         handle_.reset( m, []( b2s_matrix p ) { b2s_matrix_destroy( p ); } );
         dirty_ = false;
      }
      return handle_.get();
   }

private:
   bool inRange( Index r, size_t d ) const
   {
      const int64_t c = (int64_t) r + offsets_[ d ];
      return c >= 0 && c < cols_;
   }
   size_t slot( Index row, Index column ) const
   {
      if( row < 0 || row >= rows_ || column < 0 || column >= cols_ )
         throw std::logic_error( "element outside the matrix" );
      const auto it = std::lower_bound( offsets_.begin(), offsets_.end(), (int32_t) ( column - row ) );
      if( it == offsets_.end() || *it != column - row )
         throw std::logic_error( "the element is not on a diagonal of the matrix" );
      return (size_t) row * offsets_.size() + ( it - offsets_.begin() );
   }

   Index rows_ = 0, cols_ = 0;
   std::vector< int32_t > offsets_;
   std::vector< Real > values_;
   mutable bool dirty_ = true;
   mutable std::shared_ptr< b2s_matrix_t > handle_;
};

}  // namespace Matrices

// ---------------------------------------------------------------------------
namespace Config {
// Config::ParameterContainer (Config/ParameterContainer.h): named parameters.
class ParameterContainer
{
public:
   template< typename T >
   void addParameter( const std::string& name, const T& value )
   {
      values_[ name ] = to_string( value );
   }
   template< typename T >
   void setParameter( const std::string& name, const T& value )
   {
      addParameter( name, value );
   }
   bool checkParameter( const std::string& name ) const { return values_.count( name ) > 0; }
   const std::string& raw( const std::string& name ) const { return values_.at( name ); }

private:
   static std::string to_string( const std::string& v ) { return v; }
   static std::string to_string( const char* v ) { return v; }
   static std::string to_string( bool v ) { return v ? "1" : "0"; }
   template< typename T >
   static std::string to_string( const T& v )
   {
      return std::to_string( v );
   }
   std::map< std::string, std::string > values_;
};
}  // namespace Config

// ---------------------------------------------------------------------------
namespace Solvers {
namespace Linear {

namespace Preconditioners {
// Preconditioners::Diagonal< Matrix > (Solvers/Linear/Preconditioners/Diagonal.h:28)
template< typename Matrix >
class Diagonal
{
public:
   static constexpr b2s_precond_kind kind = B2S_PRECOND_JACOBI;
   template< typename MatrixPointer >
   void update( const MatrixPointer& )
   {}
};
// Preconditioners::ILU0< Matrix > (Solvers/Linear/Preconditioners/ILU0.h:60): the
// factorization runs on the device when the solver is created
template< typename Matrix >
class ILU0
{
public:
   static constexpr b2s_precond_kind kind = B2S_PRECOND_ILU0;
   template< typename MatrixPointer >
   void update( const MatrixPointer& )
   {}
};
// Preconditioners::ILUT< Matrix > (Solvers/Linear/Preconditioners/ILUT.h): TNL's
// host factorization with "ilut-p" / "ilut-threshold" from the solver's setup(),
// applied on the device (TNL's own Devices::Cuda ILUT throws)
template< typename Matrix >
class ILUT
{
public:
   static constexpr b2s_precond_kind kind = B2S_PRECOND_ILUT;
   template< typename MatrixPointer >
   void update( const MatrixPointer& )
   {}
};
}  // namespace Preconditioners

template< typename Matrix, b2s_solver_kind Kind >
class LinearSolverBase
{
public:
   using RealType = typename Matrix::RealType;
   using IndexType = typename Matrix::IndexType;
   using MatrixPointer = std::shared_ptr< const Matrix >;

   LinearSolverBase()
   {
      b2s_solve_opts_default( &opts_ );
      opts_.solver = Kind;
   }
   ~LinearSolverBase() { reset(); }

   // LinearSolver::setMatrix / setPreconditioner (Solvers/Linear/LinearSolver.h:121-132)
   void setMatrix( const MatrixPointer& m )
   {
      matrix_ = m;
      reset();
   }
   template< typename P >
   void setPreconditioner( const std::shared_ptr< P >& p )
   {
      opts_.preconditioner = p ? P::kind : B2S_PRECOND_NONE;
      reset();
   }
   // IterativeSolver setters (Solvers/IterativeSolver.h)
   void setConvergenceResidue( RealType r ) { opts_.convergence_residue = r, reset(); }
   void setDivergenceResidue( RealType r ) { opts_.divergence_residue = r, reset(); }
   void setMaxIterations( IndexType n ) { opts_.max_iterations = n, reset(); }
   void setMinIterations( IndexType n ) { opts_.min_iterations = n, reset(); }
   IndexType getIterations() const { return (IndexType) report_.iterations; }
   RealType getResidue() const { return (RealType) report_.residue; }
   const b2s_solve_report& getReport() const { return report_; }
   // Mixed precision: FP32 inner solves inside FP64 iterative refinement.
   void setMixedPrecision( bool on, double innerTolerance = 1e-4 )
   {
      opts_.precision = on ? B2S_PRECISION_MIXED : B2S_PRECISION_PLAIN;
      opts_.inner_tolerance = innerTolerance;
      reset();
   }

   // setup( ParameterContainer ) with TNL's keys
   bool setup( const Config::ParameterContainer& p, const std::string& prefix = "" )
   {
      auto num = [ & ]( const char* k, auto& field )
      {
         const std::string key = prefix + k;
         if( p.checkParameter( key ) )
            field = ( std::remove_reference_t< decltype( field ) > ) std::stod( p.raw( key ) );
      };
      num( "convergence-residue", opts_.convergence_residue );
      num( "divergence-residue", opts_.divergence_residue );
      num( "max-iterations", opts_.max_iterations );
      num( "min-iterations", opts_.min_iterations );
      num( "gmres-restarting-min", opts_.gmres_restarting_min );
      num( "gmres-restarting-max", opts_.gmres_restarting_max );
      num( "gmres-restarting-step-min", opts_.gmres_restarting_step_min );
      num( "gmres-restarting-step-max", opts_.gmres_restarting_step_max );
      num( "bicgstab-exact-residue", opts_.bicgstab_exact_residue );
      num( "bicgstab-ell", opts_.bicgstab_ell );
      num( "jacobi-omega", opts_.omega );
      num( "sor-omega", opts_.omega );
      num( "residue-period", opts_.residue_period );
      num( "ilut-p", opts_.ilut_p );
      num( "ilut-threshold", opts_.ilut_threshold );
      if( p.checkParameter( prefix + "gmres-variant" ) ) {
         const std::string v = p.raw( prefix + "gmres-variant" );
         if( v == "CGS" )
            opts_.gmres_variant = B2S_GMRES_CGS;
         else if( v == "CGSR" )
            opts_.gmres_variant = B2S_GMRES_CGSR;
         else if( v == "MGS" )
            opts_.gmres_variant = B2S_GMRES_MGS;
         else if( v == "MGSR" )
            opts_.gmres_variant = B2S_GMRES_MGSR;
         else if( v == "CWY" )
            opts_.gmres_variant = B2S_GMRES_CWY;
         else
            return false;
      }
      reset();
      return true;
   }

   // bool solve( ConstVectorViewType b, VectorViewType x ) (LinearSolver.h:155-156)
   template< typename VecB, typename VecX >
   bool solve( const VecB& b, VecX& x )
   {
      if( ! matrix_ )
         throw std::logic_error( "No matrix was set. Call setMatrix() before solve()." );
      if( ! solver_ ) {
         b2s_solver s = nullptr;
         detail::check( b2s_solver_create( matrix_->handle(), &opts_, &s ), "b2s_solver_create" );
         solver_ = s;
      }
      constexpr bool dev = std::is_same< typename VecX::DeviceType, Devices::Cuda >::value;
      const b2s_status st = b2s_solve( solver_, b.getData(), x.getData(), dev ? B2S_DEVICE : B2S_HOST, nullptr, &report_ );
      if( st == B2S_OK )
         return true;
      if( st == B2S_NOT_CONVERGED || st == B2S_NAN || st == B2S_DIVERGED || st == B2S_BREAKDOWN )
         return false;
      detail::check( st, "solve" );
      return false;
   }

protected:
   void reset()
   {
      if( solver_ )
         b2s_solver_destroy( solver_ );
      solver_ = nullptr;
   }
   b2s_solve_opts opts_;
   b2s_solve_report report_{};
   MatrixPointer matrix_;
   b2s_solver solver_ = nullptr;
};

template< typename Matrix >
class CG : public LinearSolverBase< Matrix, B2S_CG >
{};
template< typename Matrix >
class BICGStab : public LinearSolverBase< Matrix, B2S_BICGSTAB >
{};
template< typename Matrix >
class GMRES : public LinearSolverBase< Matrix, B2S_GMRES >
{};
// Solvers::Linear::TFQMR (Solvers/Linear/TFQMR.h)
template< typename Matrix >
class TFQMR : public LinearSolverBase< Matrix, B2S_TFQMR >
{};
// Solvers::Linear::BICGStabL (Solvers/Linear/BICGStabL.h); ell from "bicgstab-ell"
template< typename Matrix >
class BICGStabL : public LinearSolverBase< Matrix, B2S_BICGSTABL >
{};

// the relaxation parameter and the residue period of Jacobi.h:83-110 / SOR.h:82-110
template< typename Matrix, b2s_solver_kind Kind >
class StationarySolver : public LinearSolverBase< Matrix, Kind >
{
public:
   using typename LinearSolverBase< Matrix, Kind >::RealType;
   using typename LinearSolverBase< Matrix, Kind >::IndexType;
   void setOmega( RealType omega ) { this->opts_.omega = omega, this->reset(); }
   RealType getOmega() const { return (RealType) this->opts_.omega; }
   void setResiduePeriod( IndexType period ) { this->opts_.residue_period = period, this->reset(); }
   IndexType getResiduePerid() const { return this->opts_.residue_period; }
};
// Solvers::Linear::Jacobi (Solvers/Linear/Jacobi.h)
template< typename Matrix >
class Jacobi : public StationarySolver< Matrix, B2S_JACOBI >
{};
// Solvers::Linear::SOR (Solvers/Linear/SOR.h): the sequential sweep of TNL's host solver
template< typename Matrix >
class SOR : public StationarySolver< Matrix, B2S_SOR >
{};

}  // namespace Linear
}  // namespace Solvers
}  // namespace TNL
