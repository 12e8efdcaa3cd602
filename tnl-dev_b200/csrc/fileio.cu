// TNL's binary matrix files: SparseMatrix::save / load (Matrices/SparseMatrix.hpp:1233-1290,
// Matrices/Matrix.hpp:127-145, Object.hpp, File.hpp, and each segments type's save / load:
// Segments/CSR.hpp:231-244, Ellpack.hpp:233-249, SlicedEllpack.hpp:278-300,
// ChunkedEllpack.hpp:377-407, BiEllpack.hpp:409-431).
//
// An object starts with the magic "TNLMN" and its serialization type (int32
// length + characters). A sparse matrix is such a header, rows and columns
// (int32), the values and the columnIndexes as arrays (each an object header,
// an int32 element count and the raw elements), then its segments' fields:
//   CSR             offsets
//   Ellpack         segmentSize, size, alignedSize
//   SlicedEllpack   size, alignedSize, segmentsCount, sliceOffsets, sliceSegmentSizes
//   ChunkedEllpack  size, storageSize, chunksInSlice, desiredChunkSize, rowToChunkMapping,
//                   chunksToSegmentsMapping, rowToSliceMapping, rowPointers, slices, numberOfSlices
//                   (the order TNL's save produces; TNL's own load expects the two
//                   mappings and rowPointers in another order and so does not read
//                   its files back — here they are read as written)
//   BiEllpack       size, storageSize, virtualRows, rowPermArray, groupPointers
// Files are written as TNL writes them for Devices::Host CSR and for the
// ColumnMajor organisation of the padded layouts (the one TNL uses on the
// GPU and this library keeps); the type names carry neither the organisation
// nor SlicedEllpack's slice size, as in TNL.
#include "b2s_internal.cuh"

#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

using namespace b2s;

namespace b2s {

static const char kMagic[] = "TNLMN";

static std::string
real_name( int dtype )
{
   return dtype == B2S_F64 ? "double" : "float";
}

static std::string
segments_name( int format )
{
   switch( format ) {
      case B2S_CSR:
         return "CSR< [any_device], int, TNL::Algorithms::Segments::CSRScalarKernel<int, TNL::Devices::Host> >";
      case B2S_ELLPACK:
         return "Ellpack< [any_device], int >";
      case B2S_SLICED_ELLPACK:
         return "SlicedEllpack< [any_device], int >";
      case B2S_CHUNKED_ELLPACK:
         return "ChunkedEllpack< [any_device], int >";
      default:
         return "BiEllpack< [any_device], int >";
   }
}

static std::string
matrix_type( int format, int dtype )
{
   return "Matrices::SparseMatrix< " + real_name( dtype ) + ", " + segments_name( format ) +
          ", [any_device], int, General, [any_allocator], [any_allocator] >";
}

static std::string
array_type( const std::string& elem )
{
   return "Containers::Array< " + elem + ", [any_device], int, [any_allocator] >";
}

static const char kSliceInfo[] = "TNL::Algorithms::Segments::detail::ChunkedEllpackSliceInfo<int>";

// ---------------------------------------------------------------------------
struct Writer
{
   std::string buf;
   void raw( const void* p, size_t n ) { buf.append( static_cast< const char* >( p ), n ); }
   void i32( int32_t v ) { raw( &v, 4 ); }
   void header( const std::string& type )
   {
      raw( kMagic, 5 );
      i32( (int32_t) type.size() );
      raw( type.data(), type.size() );
   }
   void array( const std::string& elem, const void* data, int64_t n, size_t es )
   {
      header( array_type( elem ) );
      i32( (int32_t) n );
      raw( data, (size_t) n * es );
   }
   void array_i32( const std::vector< int32_t >& v ) { array( "int", v.data(), (int64_t) v.size(), 4 ); }
};

// one exported index array / scalar of `m`, as int32
static b2s_status
get_i32( b2s_matrix m, const char* name, std::vector< int32_t >& out )
{
   int64_t n = 0;
   B2S_TRY( b2s_matrix_export( m, name, nullptr, 0, &n ) );
   std::vector< int64_t > t( (size_t) std::max< int64_t >( n, 1 ) );
   B2S_TRY( b2s_matrix_export( m, name, t.data(), n, &n ) );
   out.resize( (size_t) n );
   for( int64_t k = 0; k < n; k++ )
      out[ k ] = (int32_t) t[ k ];
   return B2S_OK;
}

static b2s_status
get_scalar( b2s_matrix m, const char* name, int32_t& v )
{
   std::vector< int32_t > t;
   B2S_TRY( get_i32( m, name, t ) );
   v = t.empty() ? 0 : t[ 0 ];
   return B2S_OK;
}

// ---------------------------------------------------------------------------
struct Reader
{
   std::vector< unsigned char > data;
   size_t pos = 0;
   std::string error;
   bool take( void* dst, size_t n )
   {
      if( pos + n > data.size() ) {
         error = "file ends too early";
         return false;
      }
      std::memcpy( dst, data.data() + pos, n );
      pos += n;
      return true;
   }
   bool i32( int32_t& v ) { return take( &v, 4 ); }
   bool header( std::string& type )
   {
      char mn[ 5 ];
      if( ! take( mn, 5 ) )
         return false;
      if( std::memcmp( mn, kMagic, 5 ) != 0 ) {
         error = "wrong magic number - file is not in a TNL-compatible format.";
         return false;
      }
      int32_t len = 0;
      if( ! i32( len ) )
         return false;
      if( len < 0 || pos + (size_t) len > data.size() ) {
         error = "bad object type length";
         return false;
      }
      type.assign( reinterpret_cast< const char* >( data.data() + pos ), (size_t) len );
      pos += (size_t) len;
      return true;
   }
   // an array of `elem`: its elements as raw bytes
   bool array( const std::string& elem, size_t es, std::vector< unsigned char >& out, int64_t& n )
   {
      std::string type;
      if( ! header( type ) )
         return false;
      if( type != array_type( elem ) ) {
         error = "expected " + array_type( elem ) + ", found " + type;
         return false;
      }
      int32_t cnt = 0;
      if( ! i32( cnt ) )
         return false;
      if( cnt < 0 ) {
         error = "negative array size";
         return false;
      }
      n = cnt;
      out.resize( (size_t) cnt * es );
      return take( out.data(), out.size() );
   }
   bool array_i32( std::vector< int32_t >& v )
   {
      std::vector< unsigned char > raw;
      int64_t n = 0;
      if( ! array( "int", 4, raw, n ) )
         return false;
      v.resize( (size_t) n );
      if( n )
         std::memcpy( v.data(), raw.data(), raw.size() );
      return true;
   }
};

static bool
starts_with( const std::string& s, const std::string& p )
{
   return s.compare( 0, p.size(), p ) == 0;
}

}  // namespace b2s

extern "C" {

b2s_status
b2s_matrix_save( b2s_matrix m, const char* path )
{
   clear_error();
   B2S_NO_BINARY( m, "saving" );
   B2S_CHECK_ARG( m && path, "NULL argument" );
   if( m->symmetric ) {
      set_error( "SparseMatrix::save is not provided for SymmetricMatrix (lower-triangle) storage" );
      return B2S_UNSUPPORTED;
   }
   if( m->format == B2S_MULTIDIAGONAL ) {
      set_error( "binary files are provided for the sparse layouts (convert the Multidiagonal matrix first)" );
      return B2S_UNSUPPORTED;
   }
   Writer w;
   w.header( matrix_type( m->format, m->dtype ) );
   w.i32( m->rows );
   w.i32( m->cols );
   // values and columnIndexes in TNL's storage size (BiEllpack: WarpSize x the addressed part)
   int64_t n = 0;
   B2S_TRY( b2s_matrix_export( m, "values", nullptr, 0, &n ) );
   const size_t es = m->dtype == B2S_F64 ? 8 : 4;
   std::vector< unsigned char > vals( (size_t) std::max< int64_t >( n, 1 ) * es );
   B2S_TRY( b2s_matrix_export( m, "values", vals.data(), n, &n ) );
   w.array( real_name( m->dtype ), vals.data(), n, es );
   std::vector< int32_t > cols( (size_t) std::max< int64_t >( n, 1 ) );
   B2S_TRY( b2s_matrix_export( m, "columnIndexes", cols.data(), n, &n ) );
   cols.resize( (size_t) n );
   w.array_i32( cols );
   switch( m->format ) {
      case B2S_CSR: {
         std::vector< int32_t > off;
         B2S_TRY( get_i32( m, "offsets", off ) );
         w.array_i32( off );
         break;
      }
      case B2S_ELLPACK: {
         int32_t a, b, c;
         B2S_TRY( get_scalar( m, "segmentSize", a ) );
         B2S_TRY( get_scalar( m, "size", b ) );
         B2S_TRY( get_scalar( m, "alignedSize", c ) );
         w.i32( a );
         w.i32( b );
         w.i32( c );
         break;
      }
      case B2S_SLICED_ELLPACK: {
         int32_t size, aligned;
         std::vector< int32_t > so, ss;
         B2S_TRY( get_scalar( m, "size", size ) );
         B2S_TRY( get_scalar( m, "alignedSize", aligned ) );
         B2S_TRY( get_i32( m, "sliceOffsets", so ) );
         B2S_TRY( get_i32( m, "sliceSegmentSizes", ss ) );
         w.i32( size );
         w.i32( aligned );
         w.i32( m->rows );  // segmentsCount
         w.array_i32( so );
         w.array_i32( ss );
         break;
      }
      case B2S_CHUNKED_ELLPACK: {
         int32_t storage, nsl;
         std::vector< int32_t > r2c, r2s, rp, c2s, sl;
         B2S_TRY( get_scalar( m, "storageSize", storage ) );
         B2S_TRY( get_scalar( m, "numberOfSlices", nsl ) );
         B2S_TRY( get_i32( m, "rowToChunkMapping", r2c ) );
         B2S_TRY( get_i32( m, "rowToSliceMapping", r2s ) );
         B2S_TRY( get_i32( m, "rowPointers", rp ) );
         B2S_TRY( get_i32( m, "chunksToSegmentsMapping", c2s ) );
         B2S_TRY( get_i32( m, "slices", sl ) );
         w.i32( m->rows );
         w.i32( storage );
         w.i32( kChunksInSlice );
         w.i32( kDesiredChunkSize );
         w.array_i32( r2c );
         w.array_i32( c2s );
         w.array_i32( r2s );
         w.array_i32( rp );
         // TNL sizes the slice container by rows; the entries past numberOfSlices are unused (zero here)
         sl.resize( (size_t) std::max( m->rows, nsl ) * 4, 0 );
         w.array( kSliceInfo, sl.data(), (int64_t) sl.size() / 4, 16 );
         w.i32( nsl );
         break;
      }
      case B2S_BIELLPACK: {
         int32_t storage, vr;
         std::vector< int32_t > perm, gp;
         B2S_TRY( get_scalar( m, "storageSize", storage ) );
         B2S_TRY( get_scalar( m, "virtualRows", vr ) );
         B2S_TRY( get_i32( m, "rowPermArray", perm ) );
         B2S_TRY( get_i32( m, "groupPointers", gp ) );
         w.i32( m->rows );
         w.i32( storage );
         w.i32( vr );
         w.array_i32( perm );
         w.array_i32( gp );
         break;
      }
   }
   FILE* f = std::fopen( path, "wb" );
   if( ! f ) {
      set_error( "cannot open %s for writing", path );
      return B2S_IO_ERROR;
   }
   const bool ok = std::fwrite( w.buf.data(), 1, w.buf.size(), f ) == w.buf.size();
   if( ( std::fclose( f ) != 0 ) || ! ok ) {
      set_error( "write to %s failed", path );
      return B2S_IO_ERROR;
   }
   return B2S_OK;
}

b2s_status
b2s_matrix_load( const char* path, const b2s_matrix_opts* opts, b2s_stream stream, b2s_matrix* out )
{
   clear_error();
   B2S_CHECK_ARG( path && out, "NULL argument" );
   *out = nullptr;
   b2s_matrix_opts o;
   b2s_matrix_opts_default( &o );
   if( opts )
      o = *opts;
   Reader r;
   {
      FILE* f = std::fopen( path, "rb" );
      if( ! f ) {
         set_error( "cannot open %s", path );
         return B2S_IO_ERROR;
      }
      unsigned char tmp[ 1 << 16 ];
      size_t got;
      while( ( got = std::fread( tmp, 1, sizeof( tmp ), f ) ) > 0 )
         r.data.insert( r.data.end(), tmp, tmp + got );
      std::fclose( f );
   }
   auto fail = [ & ]() -> b2s_status
   {
      set_error( "%s: %s", path, r.error.c_str() );
      return B2S_INVALID_ARG;
   };
   std::string type;
   if( ! r.header( type ) )
      return fail();
   // Matrices::SparseMatrix< Real, Segments< ... >, [any_device], int, General, ... >
   int dtype = -1, format = -1;
   for( int dt : { (int) B2S_F64, (int) B2S_F32 } )
      for( int fm : { (int) B2S_CSR, (int) B2S_ELLPACK, (int) B2S_SLICED_ELLPACK, (int) B2S_CHUNKED_ELLPACK,
                      (int) B2S_BIELLPACK } ) {
         const std::string t = matrix_type( fm, dt );
         const bool match = fm == B2S_CSR
                               // any CSR kernel (the Cuda build of TNL names a Cuda kernel)
                               ? starts_with( type, "Matrices::SparseMatrix< " + real_name( dt ) + ", CSR< [any_device], int" ) &&
                                    type.find( "[any_device], int, General," ) != std::string::npos
                               : type == t;
         if( match ) {
            dtype = dt;
            format = fm;
         }
      }
   if( format < 0 ) {
      r.error = "not a sparse matrix of double/float values, int indexes and a known segments type: " + type;
      return fail();
   }
   LayoutArrays L;
   L.format = format;
   L.dtype = dtype;
   if( ! r.i32( L.rows ) || ! r.i32( L.cols ) )
      return fail();
   const size_t es = dtype == B2S_F64 ? 8 : 4;
   int64_t nv = 0, nc = 0;
   std::vector< unsigned char > craw;
   if( ! r.array( real_name( dtype ), es, L.values, nv ) || ! r.array( "int", 4, craw, nc ) )
      return fail();
   if( nv != nc ) {
      r.error = "values and columnIndexes differ in length";
      return fail();
   }
   L.columns.resize( (size_t) nc );
   if( nc )
      std::memcpy( L.columns.data(), craw.data(), craw.size() );
   L.storage = nv;
   cudaStream_t s = as_stream( stream );
   b2s_status st = B2S_OK;
   switch( format ) {
      case B2S_CSR: {
         std::vector< int32_t > off;
         if( ! r.array_i32( off ) )
            return fail();
         if( (int64_t) off.size() != (int64_t) L.rows + 1 || off[ 0 ] != 0 || off.back() != nc ) {
            r.error = "CSR offsets do not match the arrays";
            return fail();
         }
         // rows keep their elements; slots left unused by setRowCapacities (column -1) are dropped
         std::vector< int32_t > noff( off.size(), 0 ), ncol;
         std::vector< unsigned char > nval;
         for( int32_t i = 0; i < L.rows; i++ ) {
            if( off[ i + 1 ] < off[ i ] ) {
               r.error = "CSR offsets decrease";
               return fail();
            }
            for( int32_t k = off[ i ]; k < off[ i + 1 ]; k++ )
               if( L.columns[ k ] != -1 ) {
                  ncol.push_back( L.columns[ k ] );
                  nval.insert( nval.end(), L.values.begin() + (size_t) k * es, L.values.begin() + (size_t) ( k + 1 ) * es );
               }
            noff[ i + 1 ] = (int32_t) ncol.size();
         }
         return b2s_matrix_create( B2S_CSR, (b2s_dtype) dtype, L.rows, L.cols, (int64_t) ncol.size(), noff.data(),
                                   ncol.data(), nval.data(), (b2s_dtype) dtype, B2S_HOST, &o, stream, out );
      }
      case B2S_ELLPACK: {
         int32_t size = 0;
         if( ! r.i32( L.segmentSize ) || ! r.i32( size ) || ! r.i32( L.alignedSize ) )
            return fail();
         if( size != L.rows ) {
            r.error = "Ellpack size differs from the rows";
            return fail();
         }
         break;
      }
      case B2S_SLICED_ELLPACK: {
         int32_t size = 0, aligned = 0, count = 0;
         if( ! r.i32( size ) || ! r.i32( aligned ) || ! r.i32( count ) || ! r.array_i32( L.sliceOffsets ) ||
             ! r.array_i32( L.sliceSegmentSizes ) )
            return fail();
         if( count != L.rows || aligned != nv ) {
            r.error = "SlicedEllpack sizes differ from the arrays";
            return fail();
         }
         L.size = size;
         L.slice_size = o.slice_size ? o.slice_size : kSliceSize;
         break;
      }
      case B2S_CHUNKED_ELLPACK: {
         int32_t size = 0, storage = 0, cis = 0, dcs = 0;
         if( ! r.i32( size ) || ! r.i32( storage ) || ! r.i32( cis ) || ! r.i32( dcs ) )
            return fail();
         if( size != L.rows || cis != kChunksInSlice ) {
            r.error = "ChunkedEllpack sizes";
            return fail();
         }
         std::vector< unsigned char > sraw;
         int64_t ns = 0;
         if( ! r.array_i32( L.rowToChunk ) || ! r.array_i32( L.chunksToSeg ) || ! r.array_i32( L.rowToSlice ) ||
             ! r.array_i32( L.rowPointers ) || ! r.array( kSliceInfo, 16, sraw, ns ) || ! r.i32( L.numberOfSlices ) )
            return fail();
         L.slices.resize( (size_t) ns );
         if( ns )
            std::memcpy( L.slices.data(), sraw.data(), sraw.size() );
         L.storage = storage;
         break;
      }
      case B2S_BIELLPACK: {
         int32_t size = 0, storage = 0;
         if( ! r.i32( size ) || ! r.i32( storage ) || ! r.i32( L.virtualRows ) || ! r.array_i32( L.rowPerm ) ||
             ! r.array_i32( L.groupPointers ) )
            return fail();
         if( size != L.rows || storage != nv ) {
            r.error = "BiEllpack sizes";
            return fail();
         }
         break;
      }
   }
   st = matrix_from_layout( L, o, s, out );
   return st;
}

}  // extern "C"
