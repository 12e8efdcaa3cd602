/*
 * TEST INFRASTRUCTURE ONLY — the checker, never the product.
 *
 * Plain-C restatement of TNL's sparse path: the segment-layout builders, the
 * zero-dropping format conversion, the per-row SpMV reductions in the order
 * TNL's Devices::Host code uses, and the CG / BiCGStab / GMRES iterations.
 * Each function names the reference file:line it restates (paths are relative
 * to the TNL source tree, src/TNL/...).
 */
#include "b2s_oracle.h"

#include <math.h>
#include <float.h>
#include <limits.h>
#include <stdlib.h>
#include <string.h>

#define PADDING_INDEX ( -1 ) /* Matrices/SparseMatrix.hpp:1315 getPaddingIndex() */
#define SLICE_SIZE 32        /* Segments/SlicedEllpack.h default SliceSize */
#define WARP 32              /* Segments/BiEllpack.h default WarpSize */
#define LOG_WARP 5
#define GROUPS ( LOG_WARP + 1 )
#define CHUNKS_IN_SLICE 256  /* Segments/ChunkedEllpack.h:182 */
#define DESIRED_CHUNK 16

#define MAX_META 12

typedef struct
{
   char name[ 32 ];
   long long n;
   long long* v;
} meta_t;

struct b2so_matrix
{
   int format, org, real, rows, cols;
   long long storage;
   double* values;
   int* columns;
   /* layout metadata (only the family in use is filled) */
   int* offsets;                           /* CSR */
   int segmentSize, alignedSize;           /* Ellpack */
   int nslices, slice;                     /* SlicedEllpack (slice = SliceSize) */
   int *sliceOffsets, *sliceSegmentSizes;  /* SlicedEllpack */
   int numberOfSlices;                     /* ChunkedEllpack */
   int *rowToChunk, *rowToSlice, *chunksToSeg, *rowPointers, *cslices; /* cslices: 4 per slice */
   int virtualRows;                        /* BiEllpack */
   int *rowPerm, *groupPointers;
   int nmeta;
   meta_t meta[ MAX_META ];
};

static void
put_meta_i( b2so_matrix* m, const char* name, const int* v, long long n )
{
   meta_t* t = &m->meta[ m->nmeta++ ];
   strncpy( t->name, name, sizeof( t->name ) - 1 );
   t->n = n;
   t->v = (long long*) malloc( sizeof( long long ) * ( n > 0 ? n : 1 ) );
   for( long long i = 0; i < n; i++ )
      t->v[ i ] = v[ i ];
}

static void
put_meta_s( b2so_matrix* m, const char* name, long long s )
{
   meta_t* t = &m->meta[ m->nmeta++ ];
   strncpy( t->name, name, sizeof( t->name ) - 1 );
   t->n = 1;
   t->v = (long long*) malloc( sizeof( long long ) );
   t->v[ 0 ] = s;
}

static int
round_up_div( int a, int b )
{
   /* TNL::roundUpDivision (Math.h) */
   return a / b + ( a % b != 0 );
}

/* ---------------------------------------------------------------------------
 * Ellpack — Segments/Ellpack.hpp:69-80 (setSegmentsSizes), EllpackView.hpp:246-253
 * (getGlobalIndex): segment size = max capacity; ColumnMajor pads the row
 * count to a multiple of 32 and strides by it. */
static void
build_ellpack( b2so_matrix* m, const int* caps )
{
   int mx = 0;
   for( int i = 0; i < m->rows; i++ )
      if( caps[ i ] > mx )
         mx = caps[ i ];
   m->segmentSize = mx;
   m->alignedSize = m->org == 1 ? m->rows : round_up_div( m->rows, 32 ) * 32;
   m->storage = (long long) m->alignedSize * m->segmentSize;
   put_meta_s( m, "segmentSize", m->segmentSize );
   put_meta_s( m, "size", m->rows );
   put_meta_s( m, "alignedSize", m->alignedSize );
}

static long long
gidx_ellpack( const b2so_matrix* m, int row, int local )
{
   if( m->org == 1 )
      return (long long) row * m->segmentSize + local;
   return row + (long long) m->alignedSize * local;
}

/* ---------------------------------------------------------------------------
 * SlicedEllpack — SlicedEllpack.hpp:64-101: per slice of 32 rows the width is
 * the largest capacity in the slice, slice offsets = exclusive scan of
 * 32*width; SlicedEllpackView.hpp:108-132 gives the element position. */
static void
build_sliced( b2so_matrix* m, const int* caps )
{
   const int S = m->slice;
   const int ns = round_up_div( m->rows, S );
   m->nslices = ns;
   m->sliceOffsets = (int*) calloc( ns + 1, sizeof( int ) );
   m->sliceSegmentSizes = (int*) calloc( ns > 0 ? ns : 1, sizeof( int ) );
   long long sum = 0;
   for( int s = 0; s < ns; s++ ) {
      int w = INT_MIN;
      for( int k = 0; k < S; k++ ) {
         const int r = s * S + k;
         const int c = r < m->rows ? caps[ r ] : 0;
         if( c > w )
            w = c;
      }
      m->sliceSegmentSizes[ s ] = w;
      m->sliceOffsets[ s ] = w * S;
   }
   /* exclusive scan (Algorithms/scan.h inplaceExclusiveScan) */
   int run = 0;
   for( int s = 0; s <= ns; s++ ) {
      const int v = m->sliceOffsets[ s ];
      m->sliceOffsets[ s ] = run;
      run += v;
   }
   for( int i = 0; i < m->rows; i++ )
      sum += caps[ i ];
   m->alignedSize = m->sliceOffsets[ ns ];
   m->storage = m->alignedSize;
   put_meta_i( m, "sliceOffsets", m->sliceOffsets, ns + 1 );
   put_meta_i( m, "sliceSegmentSizes", m->sliceSegmentSizes, ns );
   put_meta_s( m, "size", sum );
   put_meta_s( m, "alignedSize", m->alignedSize );
}

static long long
gidx_sliced( const b2so_matrix* m, int row, int local )
{
   const int s = row / m->slice, i = row % m->slice;
   if( m->org == 1 )
      return (long long) m->sliceOffsets[ s ] + (long long) i * m->sliceSegmentSizes[ s ] + local;
   return (long long) m->sliceOffsets[ s ] + i + (long long) m->slice * local;
}

/* ---------------------------------------------------------------------------
 * ChunkedEllpack — ChunkedEllpack.hpp:80-110 (resolveSliceSizes: greedy slices
 * of about 256*16 elements and at most 256 rows), :113-183 (setSlice: one chunk
 * per row plus a share of the free chunks proportional to the row length,
 * truncated; leftovers go round-robin to the longest rows; chunk size = max
 * ceil(len/chunks)), :186-222 (setSegmentsSizes: row pointers by inclusive
 * scan, chunk -> row map); getGlobalIndex in detail/ChunkedEllpack.h:110-135. */
static void
build_chunked( b2so_matrix* m, const int* caps )
{
   const int n = m->rows;
   int* sl = (int*) malloc( sizeof( int ) * 4 * ( n > 0 ? n : 1 ) ); /* size, chunkSize, firstSegment, pointer */
   m->rowToChunk = (int*) calloc( n > 0 ? n : 1, sizeof( int ) );
   m->rowToSlice = (int*) calloc( n > 0 ? n : 1, sizeof( int ) );
   m->rowPointers = (int*) calloc( n + 1, sizeof( int ) );
   const int desired = CHUNKS_IN_SLICE * DESIRED_CHUNK;

   /* resolveSliceSizes */
   int seg = 0, sliceSize = 0, alloc = 0, ns = 0;
   while( seg < n ) {
      alloc += caps[ seg ];
      sliceSize++;
      seg++;
      if( alloc < desired && seg < n && sliceSize < CHUNKS_IN_SLICE )
         continue;
      sl[ 4 * ns + 0 ] = sliceSize;
      sl[ 4 * ns + 2 ] = seg - sliceSize;
      sl[ 4 * ns + 3 ] = alloc; /* temporary: elements in the slice */
      sliceSize = 0;
      ns++;
      alloc = 0;
   }

   /* setSlice for every slice */
   int storage = 0;
   for( int s = 0; s < ns; s++ ) {
      const int size = sl[ 4 * s + 0 ], begin = sl[ 4 * s + 2 ], allocated = sl[ 4 * s + 3 ];
      const int end = begin + size;
      int freeChunks = CHUNKS_IN_SLICE - size;
      for( int i = begin; i < end; i++ )
         m->rowToChunk[ i ] = 1;
      int totalAdded = 0;
      int maxLen = caps[ begin ];
      for( int i = begin; i < end; i++ ) {
         double ratio = 0.0;
         if( allocated != 0 )
            ratio = (double) caps[ i ] / (double) allocated;
         const int added = (int) ( (double) freeChunks * ratio );
         totalAdded += added;
         m->rowToChunk[ i ] += added;
         if( maxLen < caps[ i ] )
            maxLen = caps[ i ];
      }
      freeChunks -= totalAdded;
      while( freeChunks )
         for( int i = begin; i < end && freeChunks; i++ )
            if( caps[ i ] == maxLen ) {
               m->rowToChunk[ i ]++;
               freeChunks--;
            }
      int maxChunk = 0;
      for( int i = begin; i < end; i++ ) {
         const int c = round_up_div( caps[ i ], m->rowToChunk[ i ] );
         if( c > maxChunk )
            maxChunk = c;
      }
      sl[ 4 * s + 1 ] = maxChunk;
      sl[ 4 * s + 3 ] = storage;
      storage += CHUNKS_IN_SLICE * maxChunk;
      for( int i = begin; i < end; i++ ) {
         m->rowToSlice[ i ] = s;
         m->rowPointers[ i + 1 ] = maxChunk * m->rowToChunk[ i ];
      }
      for( int j = begin + 1; j < end; j++ )
         m->rowToChunk[ j ] += m->rowToChunk[ j - 1 ];
   }
   /* inclusive scan of rowPointers (element 0 is 0) */
   for( int i = 1; i <= n; i++ )
      m->rowPointers[ i ] += m->rowPointers[ i - 1 ];

   const long long chunks = (long long) ns * CHUNKS_IN_SLICE;
   m->chunksToSeg = (int*) calloc( chunks > 0 ? chunks : 1, sizeof( int ) );
   long long chunkIdx = 0;
   for( int r = 0; r < n; r++ ) {
      const int s = m->rowToSlice[ r ];
      const int first = ( r != sl[ 4 * s + 2 ] ) ? m->rowToChunk[ r - 1 ] : 0;
      const int cnt = m->rowToChunk[ r ] - first;
      for( int i = 0; i < cnt; i++ )
         m->chunksToSeg[ chunkIdx++ ] = r;
   }
   m->numberOfSlices = ns;
   m->cslices = sl;
   m->storage = storage;
   put_meta_s( m, "numberOfSlices", ns );
   put_meta_s( m, "storageSize", storage );
   put_meta_i( m, "rowToChunkMapping", m->rowToChunk, n );
   put_meta_i( m, "rowToSliceMapping", m->rowToSlice, n );
   put_meta_i( m, "chunksToSegmentsMapping", m->chunksToSeg, chunks );
   put_meta_i( m, "rowPointers", m->rowPointers, n + 1 );
   put_meta_i( m, "slices", sl, 4LL * ns );
}

static long long
gidx_chunked( const b2so_matrix* m, int row, int local )
{
   const int s = m->rowToSlice[ row ];
   const int first = ( row != m->cslices[ 4 * s + 2 ] ) ? m->rowToChunk[ row - 1 ] : 0;
   const long long ptr = m->cslices[ 4 * s + 3 ];
   const int cs = m->cslices[ 4 * s + 1 ];
   if( m->org == 1 )
      return ptr + (long long) first * cs + local;
   return ptr + (long long) ( local % cs ) * CHUNKS_IN_SLICE + first + local / cs;
}

/* ---------------------------------------------------------------------------
 * BiEllpack — BiEllpack.hpp:74-131 (performRowBubbleSort): inside each strip of
 * 32 rows the rows are ordered by non-increasing capacity with ties kept in
 * row order (the reference's cocktail sort swaps only strictly out-of-order
 * neighbours, so it is stable); rowPermArray[row] = strip*32 + rank.
 * BiEllpack.hpp:134-170 (computeColumnSizes): group g of a strip has height
 * 32>>g and width len(rank 2^(4-g)-1) - len(rank 2^(5-g)-1); the last strip
 * skips groups it cannot fill; group 5 stays empty. groupPointers is an
 * exclusive scan of group sizes; storage = 32 * total (BiEllpack.hpp:261).
 * Element positions: detail/BiEllpack.h:150-180 (getGlobalIndex). */
static void
build_biell( b2so_matrix* m, const int* caps )
{
   const int n = m->rows;
   m->virtualRows = ( n % WARP ) ? n + WARP - ( n % WARP ) : n;
   const int strips = m->virtualRows / WARP;
   m->rowPerm = (int*) calloc( n > 0 ? n : 1, sizeof( int ) );
   m->groupPointers = (int*) calloc( (size_t) strips * GROUPS + 1, sizeof( int ) );
   int order[ WARP ];
   for( int st = 0; st < strips; st++ ) {
      const int begin = st * WARP;
      const int end = ( begin + WARP < n ) ? begin + WARP : n;
      const int cnt = end - begin;
      /* stable insertion sort of the strip's rows by non-increasing capacity */
      for( int i = 0; i < cnt; i++ ) {
         int j = i;
         while( j > 0 && caps[ begin + order[ j - 1 ] ] < caps[ begin + i ] ) {
            order[ j ] = order[ j - 1 ];
            j--;
         }
         order[ j ] = i;
      }
      for( int rank = 0; rank < cnt; rank++ )
         m->rowPerm[ begin + order[ rank ] ] = begin + rank;

      const int gb = st * GROUPS;
      int empty = 0;
      if( st == strips - 1 ) {
         while( cnt <= ( 1 << ( LOG_WARP - 1 - empty ) ) - 1 )
            empty++;
         for( int g = 0; g < empty; g++ )
            m->groupPointers[ gb + g ] = 0;
      }
      int allocated = 0;
      for( int g = empty; g < LOG_WARP; g++ ) {
         const int rank = ( 1 << ( LOG_WARP - 1 - g ) ) - 1;
         const int len = caps[ begin + order[ rank ] ];
         const int width = len - allocated;
         const int height = 1 << ( LOG_WARP - g );
         allocated = len;
         m->groupPointers[ gb + g ] = width * height;
      }
   }
   int run = 0;
   const int ng = strips * GROUPS + 1;
   for( int i = 0; i < ng; i++ ) {
      const int v = m->groupPointers[ i ];
      m->groupPointers[ i ] = run;
      run += v;
   }
   m->storage = (long long) WARP * m->groupPointers[ strips * GROUPS ];
   put_meta_s( m, "virtualRows", m->virtualRows );
   put_meta_s( m, "storageSize", m->storage );
   put_meta_i( m, "rowPermArray", m->rowPerm, n );
   put_meta_i( m, "groupPointers", m->groupPointers, ng );
}

static int
bi_active_groups( int rank_in_strip )
{
   /* detail/BiEllpack.h:48-64 getActiveGroupsCountDirect */
   int bisection = 1;
   for( int i = 0; i < GROUPS; i++ ) {
      if( rank_in_strip < bisection )
         return GROUPS - i;
      bisection *= 2;
   }
   return -1;
}

static long long
gidx_biell( const b2so_matrix* m, int row, int local )
{
   const int strip = row / WARP;
   const int gidx = strip * GROUPS;
   const int p = m->rowPerm[ row ] - strip * WARP;
   const int groups = bi_active_groups( p );
   long long g = m->groupPointers[ gidx ];
   int h = WARP;
   for( int k = 0; k < groups; k++ ) {
      const int size = m->groupPointers[ gidx + k + 1 ] - m->groupPointers[ gidx + k ];
      if( size ) {
         const int w = size / h;
         if( local >= w ) {
            local -= w;
            g += size;
         }
         else
            return m->org == 1 ? g + (long long) p * w + local : g + p + (long long) local * h;
      }
      h /= 2;
   }
   return -1;
}

/* ---------------------------------------------------------------------------
 * Generic segment access */
static long long
gidx( const b2so_matrix* m, int row, int local )
{
   switch( m->format ) {
      case 0:
         return (long long) m->offsets[ row ] + local;
      case 1:
         return gidx_ellpack( m, row, local );
      case 2:
         return gidx_sliced( m, row, local );
      case 3:
         return gidx_chunked( m, row, local );
      case 4:
         return gidx_biell( m, row, local );
   }
   return -1;
}

static int
segment_size( const b2so_matrix* m, int row )
{
   switch( m->format ) {
      case 0:
         return m->offsets[ row + 1 ] - m->offsets[ row ];
      case 1:
         return m->segmentSize;
      case 2:
         return m->sliceSegmentSizes[ row / m->slice ];
      case 3: {
         /* detail/ChunkedEllpack.h:78-92 getSegmentSizeDirect */
         const int s = m->rowToSlice[ row ];
         const int first = ( row != m->cslices[ 4 * s + 2 ] ) ? m->rowToChunk[ row - 1 ] : 0;
         return ( m->rowToChunk[ row ] - first ) * m->cslices[ 4 * s + 1 ];
      }
      case 4: {
         /* detail/BiEllpack.h:92-108 getSegmentSizeDirect */
         const int strip = row / WARP;
         const int groups = bi_active_groups( m->rowPerm[ row ] - strip * WARP );
         int h = WARP, sz = 0;
         for( int g = 0; g < groups; g++ ) {
            const int gs = m->groupPointers[ strip * GROUPS + g + 1 ] - m->groupPointers[ strip * GROUPS + g ];
            sz += gs / h;
            h /= 2;
         }
         return sz;
      }
   }
   return 0;
}

b2so_matrix*
b2so_create( int format, int org, int real, int rows, int cols, const int* offsets, const int* columns, const double* values )
{
   if( rows < 0 || cols < 0 || format < 0 || format > 7 )
      return NULL;
   b2so_matrix* m = (b2so_matrix*) calloc( 1, sizeof( b2so_matrix ) );
   /* formats 5, 6, 7: SlicedEllpack< ..., SliceSize = 8, 16, 64 > */
   m->slice = SLICE_SIZE;
   if( format >= 5 ) {
      m->slice = format == 5 ? 8 : ( format == 6 ? 16 : 64 );
      format = 2;
   }
   m->format = format;
   m->org = org;
   m->real = real;
   m->rows = rows;
   m->cols = cols;
   int* caps = (int*) malloc( sizeof( int ) * ( rows > 0 ? rows : 1 ) );
   for( int i = 0; i < rows; i++ )
      caps[ i ] = offsets[ i + 1 ] - offsets[ i ];
   const long long nnz = offsets[ rows ];

   if( format == 0 ) {
      /* CSR kept exactly as assembled */
      m->offsets = (int*) malloc( sizeof( int ) * ( rows + 1 ) );
      memcpy( m->offsets, offsets, sizeof( int ) * ( rows + 1 ) );
      m->storage = nnz;
      m->values = (double*) malloc( sizeof( double ) * ( nnz > 0 ? nnz : 1 ) );
      m->columns = (int*) malloc( sizeof( int ) * ( nnz > 0 ? nnz : 1 ) );
      for( long long k = 0; k < nnz; k++ ) {
         m->values[ k ] = real ? (double) (float) values[ k ] : values[ k ];
         m->columns[ k ] = columns[ k ];
      }
      put_meta_i( m, "offsets", m->offsets, rows + 1 );
      free( caps );
      return m;
   }

   switch( format ) {
      case 1:
         build_ellpack( m, caps );
         break;
      case 2:
         build_sliced( m, caps );
         break;
      case 3:
         build_chunked( m, caps );
         break;
      case 4:
         build_biell( m, caps );
         break;
   }
   /* SparseMatrix::setRowCapacities (SparseMatrix.hpp:284-304): values 0,
    * columns = padding index; then operator= (SparseMatrix.hpp:1093-1110):
    * nonzero elements of each row go to consecutive local slots. */
   const long long st = m->storage;
   m->values = (double*) calloc( st > 0 ? st : 1, sizeof( double ) );
   m->columns = (int*) malloc( sizeof( int ) * ( st > 0 ? st : 1 ) );
   for( long long k = 0; k < st; k++ )
      m->columns[ k ] = PADDING_INDEX;
   for( int r = 0; r < rows; r++ ) {
      int local = 0;
      for( int k = offsets[ r ]; k < offsets[ r + 1 ]; k++ ) {
         const double v = real ? (double) (float) values[ k ] : values[ k ];
         if( v != 0.0 && columns[ k ] != PADDING_INDEX ) {
            const long long g = gidx( m, r, local++ );
            m->columns[ g ] = columns[ k ];
            m->values[ g ] = v;
         }
      }
   }
   free( caps );
   return m;
}

/* SparseMatrixView::addElement( row, column, value, multiplicator )
 * (Matrices/SparseMatrixView.hpp:272-340): the row is scanned in local order;
 * an equal column is merged (multiplicator * old + value), otherwise the
 * element goes to the first padding slot or is inserted before the first
 * larger column with the tail shifted by one slot. Returns -1 when the row
 * is full. Arithmetic in the matrix's Real (float when m->real). */
static int
add_element( b2so_matrix* m, int row, int column, double value, double mult )
{
   const int rowSize = segment_size( m, row );
   int col = PADDING_INDEX;
   int i;
   long long g = -1;
   for( i = 0; i < rowSize; i++ ) {
      g = gidx( m, row, i );
      col = m->columns[ g ];
      if( col == column ) {
         if( m->real ) {
            const float r = (float) mult * (float) m->values[ g ] + (float) value;
            m->values[ g ] = r;
         }
         else
            m->values[ g ] = mult * m->values[ g ] + value;
         return 0;
      }
      if( col == PADDING_INDEX || col > column )
         break;
   }
   if( i == rowSize )
      return -1;
   if( col != PADDING_INDEX ) {
      for( int j = rowSize - 1; j > i; j-- ) {
         const long long g1 = gidx( m, row, j ), g2 = gidx( m, row, j - 1 );
         m->columns[ g1 ] = m->columns[ g2 ];
         m->values[ g1 ] = m->values[ g2 ];
      }
   }
   m->columns[ g ] = column;
   m->values[ g ] = m->real ? (double) (float) value : value;
   return 0;
}

b2so_matrix*
b2so_from_coo( int format, int org, int real, int rows, int cols, long long n, const int* ri, const int* ci,
               const double* v, int add, const int* row_caps )
{
   if( rows < 0 || cols < 0 || format < 0 || format > 7 || n < 0 )
      return NULL;
   for( long long k = 0; k < n; k++ )
      if( ri[ k ] < 0 || ri[ k ] >= rows || ci[ k ] < 0 || ci[ k ] >= cols )
         return NULL;
   /* SparseMatrix::setRowCapacities( counts ) (SparseMatrix.hpp:284-304) */
   int* caps = (int*) calloc( rows > 0 ? rows : 1, sizeof( int ) );
   for( long long k = 0; k < n; k++ )
      caps[ ri[ k ] ]++;
   if( row_caps )
      for( int i = 0; i < rows; i++ )
         caps[ i ] = row_caps[ i ];
   b2so_matrix* m = (b2so_matrix*) calloc( 1, sizeof( b2so_matrix ) );
   m->slice = SLICE_SIZE;
   if( format >= 5 ) {
      m->slice = format == 5 ? 8 : ( format == 6 ? 16 : 64 );
      format = 2;
   }
   m->format = format;
   m->org = org;
   m->real = real;
   m->rows = rows;
   m->cols = cols;
   switch( format ) {
      case 0: {
         /* CSR offsets: exclusive scan of the capacities (Segments/detail/CSR.h:25-35) */
         m->offsets = (int*) malloc( sizeof( int ) * ( rows + 1 ) );
         long long acc = 0;
         for( int i = 0; i < rows; i++ ) {
            m->offsets[ i ] = (int) acc;
            acc += caps[ i ];
         }
         m->offsets[ rows ] = (int) acc;
         m->storage = acc;
         put_meta_i( m, "offsets", m->offsets, rows + 1 );
         break;
      }
      case 1:
         build_ellpack( m, caps );
         break;
      case 2:
         build_sliced( m, caps );
         break;
      case 3:
         build_chunked( m, caps );
         break;
      case 4:
         build_biell( m, caps );
         break;
   }
   free( caps );
   const long long st = m->storage;
   m->values = (double*) calloc( st > 0 ? st : 1, sizeof( double ) );
   m->columns = (int*) malloc( sizeof( int ) * ( st > 0 ? st : 1 ) );
   for( long long k = 0; k < st; k++ )
      m->columns[ k ] = PADDING_INDEX;
   /* setElement = addElement( row, column, value, 0 ) (SparseMatrixView.hpp:256-263) */
   for( long long k = 0; k < n; k++ )
      if( add_element( m, ri[ k ], ci[ k ], v[ k ], add ? 1.0 : 0.0 ) != 0 ) {
         b2so_destroy( m );
         return NULL;
      }
   return m;
}

void
b2so_destroy( b2so_matrix* m )
{
   if( ! m )
      return;
   free( m->values );
   free( m->columns );
   free( m->offsets );
   free( m->sliceOffsets );
   free( m->sliceSegmentSizes );
   free( m->rowToChunk );
   free( m->rowToSlice );
   free( m->chunksToSeg );
   free( m->rowPointers );
   free( m->cslices );
   free( m->rowPerm );
   free( m->groupPointers );
   for( int i = 0; i < m->nmeta; i++ )
      free( m->meta[ i ].v );
   free( m );
}

long long
b2so_storage_size( const b2so_matrix* m )
{
   return m->storage;
}

void
b2so_export_values( const b2so_matrix* m, double* out )
{
   memcpy( out, m->values, sizeof( double ) * m->storage );
}

void
b2so_export_columns( const b2so_matrix* m, int* out )
{
   memcpy( out, m->columns, sizeof( int ) * m->storage );
}

int
b2so_meta_count( const b2so_matrix* m )
{
   return m->nmeta;
}

const char*
b2so_meta_name( const b2so_matrix* m, int i )
{
   return m->meta[ i ].name;
}

long long
b2so_meta_size( const b2so_matrix* m, int i )
{
   return m->meta[ i ].n;
}

void
b2so_meta_get( const b2so_matrix* m, int i, long long* out )
{
   memcpy( out, m->meta[ i ].v, sizeof( long long ) * m->meta[ i ].n );
}

/* ---------------------------------------------------------------------------
 * SpMV — Matrices/SparseMatrixView.hpp:390-490: for each row, sum of
 * value*x[column] over the row's local slots in order, starting from 0 and
 * stopping at the first padding slot; then the keeper selected by alpha/beta.
 * Row loops as in CSRScalarKernel.hpp:32-57 (Host), EllpackView.hpp:357-372,
 * SlicedEllpackView.hpp:237-284, ChunkedEllpackView.hpp:275-316,
 * BiEllpackView.hpp:244-297. */
void
b2so_spmv( const b2so_matrix* m, const double* x, double* y, double alpha, double beta, int begin, int end )
{
   if( end == 0 )
      end = m->rows;
   for( int r = begin; r < end; r++ ) {
      const int len = segment_size( m, r );
      double sd = 0.0;
      float sf = 0.0f;
      for( int l = 0; l < len; l++ ) {
         const long long g = gidx( m, r, l );
         const int c = m->columns[ g ];
         if( m->format != 0 && c == PADDING_INDEX )
            break;
         if( m->real ) {
            const float p = (float) m->values[ g ] * (float) x[ c ];
            sf = sf + p;
         }
         else {
            const double p = m->values[ g ] * x[ c ];
            sd = sd + p;
         }
      }
      const double s = m->real ? (double) sf : sd;
      if( beta == 0.0 )
         y[ r ] = ( alpha == 1.0 ) ? s : alpha * s;
      else
         y[ r ] = ( alpha == 1.0 ) ? beta * y[ r ] + s : beta * y[ r ] + alpha * s;
   }
}

/* ---------------------------------------------------------------------------
 * Krylov solvers (FP64, CSR). Vector kernels follow the expression order of
 * the reference statements; sums are sequential. */
typedef struct
{
   int n;
   const int* off;
   const int* col;
   const double* val;
   const double* diag; /* Jacobi: NULL when unpreconditioned */
} sys_t;

static void
matvec( const sys_t* s, const double* x, double* y )
{
   for( int r = 0; r < s->n; r++ ) {
      double a = 0.0;
      for( int k = s->off[ r ]; k < s->off[ r + 1 ]; k++ ) {
         const double p = s->val[ k ] * x[ s->col[ k ] ];
         a = a + p;
      }
      y[ r ] = a;
   }
}

static double
dot( int n, const double* a, const double* b )
{
   double s = 0.0;
   for( int i = 0; i < n; i++ ) {
      const double p = a[ i ] * b[ i ];
      s = s + p;
   }
   return s;
}

static double
nrm2( int n, const double* a )
{
   return sqrt( dot( n, a, a ) );
}

static void
precond( const sys_t* s, const double* b, double* x )
{
   /* Preconditioners/Diagonal.hpp:43-47: x = b / diagonal */
   for( int i = 0; i < s->n; i++ )
      x[ i ] = b[ i ] / s->diag[ i ];
}

typedef struct
{
   long long it, maxit;
   double res, tol;
} ctl_t;

/* IterativeSolver.hpp:98-118 nextIteration / checkNextIteration (minIterations
 * 0, divergence residue = DBL_MAX) */
static int
check_next( const ctl_t* c )
{
   if( isnan( c->res ) || c->it > c->maxit || c->res > DBL_MAX || c->res < c->tol )
      return 0;
   return 1;
}

static int
next_iteration( ctl_t* c )
{
   const int r = check_next( c );
   c->it++;
   return r;
}

/* IterativeSolver.hpp:121-146 checkConvergence */
static int
check_convergence( const ctl_t* c )
{
   if( isnan( c->res ) )
      return 0;
   if( c->res > DBL_MAX && c->it > 0 )
      return 0;
   if( c->it >= c->maxit )
      return 0;
   if( c->res > c->tol )
      return 0;
   return 1;
}

/* Solvers/Linear/CG.hpp:11-104 */
static int
solve_cg( const sys_t* s, const double* b, double* x, ctl_t* c )
{
   const int n = s->n;
   double *r = malloc( sizeof( double ) * n ), *p = malloc( sizeof( double ) * n ), *Ap = malloc( sizeof( double ) * n ),
          *z = malloc( sizeof( double ) * n );
   double normb;
   if( s->diag ) {
      precond( s, b, r );
      normb = nrm2( n, r );
   }
   else
      normb = nrm2( n, b );
   if( normb == 0.0 )
      normb = 1.0;
   matvec( s, x, r );
   for( int i = 0; i < n; i++ )
      r[ i ] = b[ i ] - r[ i ];
   double s1, s2;
   if( s->diag ) {
      precond( s, r, z );
      memcpy( p, z, sizeof( double ) * n );
      s1 = dot( n, r, z );
   }
   else {
      memcpy( p, r, sizeof( double ) * n );
      s1 = dot( n, r, r );
   }
   c->it = 0;
   c->res = sqrt( s1 ) / normb;
   while( next_iteration( c ) ) {
      matvec( s, p, Ap );
      s2 = dot( n, Ap, p );
      if( s2 == 0.0 ) {
         c->res = 0.0;
         break;
      }
      const double alpha = s1 / s2;
      for( int i = 0; i < n; i++ )
         x[ i ] += alpha * p[ i ];
      for( int i = 0; i < n; i++ )
         r[ i ] -= alpha * Ap[ i ];
      s2 = s1;
      if( s->diag ) {
         precond( s, r, z );
         s1 = dot( n, r, z );
      }
      else
         s1 = dot( n, r, r );
      const double beta = ( s2 == 0.0 ) ? 0.0 : s1 / s2;
      const double* src = s->diag ? z : r;
      for( int i = 0; i < n; i++ )
         p[ i ] = src[ i ] + beta * p[ i ];
      c->res = sqrt( s1 ) / normb;
   }
   free( r );
   free( p );
   free( Ap );
   free( z );
   return check_convergence( c );
}

/* Solvers/Linear/BICGStab.hpp:33-145 */
static void
bicg_residue( const sys_t* s, double* r, const double* x, const double* b, double* tmp )
{
   if( s->diag ) {
      matvec( s, x, tmp );
      for( int i = 0; i < s->n; i++ )
         tmp[ i ] = b[ i ] - tmp[ i ];
      precond( s, tmp, r );
   }
   else {
      matvec( s, x, r );
      for( int i = 0; i < s->n; i++ )
         r[ i ] = b[ i ] - r[ i ];
   }
}

static void
bicg_matvec( const sys_t* s, const double* src, double* dst, double* tmp )
{
   if( s->diag ) {
      matvec( s, src, tmp );
      precond( s, tmp, dst );
   }
   else
      matvec( s, src, dst );
}

static int
solve_bicgstab( const sys_t* s, const double* b, double* x, ctl_t* c, int exact )
{
   const int n = s->n;
   double* buf = calloc( (size_t) 7 * n, sizeof( double ) );
   double *r = buf, *r_ast = buf + n, *p = buf + 2 * n, *sv = buf + 3 * n, *Ap = buf + 4 * n, *As = buf + 5 * n,
          *tmp = buf + 6 * n;
   double b_norm;
   if( s->diag ) {
      precond( s, b, tmp );
      b_norm = nrm2( n, tmp );
   }
   else
      b_norm = nrm2( n, b );
   if( b_norm == 0.0 )
      b_norm = 1.0;
   bicg_residue( s, r, x, b, tmp );
   memcpy( p, r, sizeof( double ) * n );
   memcpy( r_ast, r, sizeof( double ) * n );
   double rho = dot( n, r, r_ast ), r_ast_sqnorm = rho;
   const double eps2 = DBL_EPSILON * DBL_EPSILON;
   c->it = 0;
   c->res = sqrt( rho ) / b_norm;
   while( next_iteration( c ) ) {
      bicg_matvec( s, p, Ap, tmp );
      const double alpha = rho / dot( n, Ap, r_ast );
      for( int i = 0; i < n; i++ )
         sv[ i ] = r[ i ] - alpha * Ap[ i ];
      bicg_matvec( s, sv, As, tmp );
      const double omega = dot( n, As, sv ) / dot( n, As, As );
      for( int i = 0; i < n; i++ )
         x[ i ] += alpha * p[ i ] + omega * sv[ i ];
      for( int i = 0; i < n; i++ )
         r[ i ] = sv[ i ] - omega * As[ i ];
      const double rho_old = rho;
      rho = dot( n, r, r_ast );
      if( fabs( rho ) < eps2 * r_ast_sqnorm ) {
         bicg_residue( s, r, x, b, tmp );
         memcpy( r_ast, r, sizeof( double ) * n );
         r_ast_sqnorm = rho = dot( n, r, r_ast );
      }
      const double beta = ( rho / rho_old ) * ( alpha / omega );
      for( int i = 0; i < n; i++ )
         p[ i ] = r[ i ] + beta * p[ i ] - ( beta * omega ) * Ap[ i ];
      if( exact ) {
         bicg_residue( s, sv, x, b, tmp );
         c->res = nrm2( n, sv ) / b_norm;
      }
      else
         c->res = nrm2( n, r ) / b_norm;
   }
   free( buf );
   return check_convergence( c );
}

/* Solvers/Linear/GMRES.hpp:72-178 (restart loop with Baker-Jessup-Kolev
 * adaptivity), :182-346 (CGS/CGSR/MGS/MGSR Arnoldi), :641-665 (update:
 * back substitution and x += V y), :722-763 (Givens rotations). */
static void
gen_rot( double dx, double dy, double* cs, double* sn )
{
   if( dy == 0.0 ) {
      *cs = 1.0;
      *sn = 0.0;
   }
   else if( fabs( dy ) > fabs( dx ) ) {
      const double t = dx / dy;
      *sn = 1.0 / sqrt( 1.0 + t * t );
      *cs = t * *sn;
   }
   else {
      const double t = dy / dx;
      *cs = 1.0 / sqrt( 1.0 + t * t );
      *sn = t * *cs;
   }
}

static void
app_rot( double* dx, double* dy, double cs, double sn )
{
   const double t = cs * *dx + sn * *dy;
   *dy = cs * *dy - sn * *dx;
   *dx = t;
}

static int
solve_gmres( const sys_t* s, const double* b, double* x, ctl_t* c, int variant, int rmin, int rmax )
{
   const int n = s->n;
   if( rmin <= 0 || rmax <= 0 || rmin > rmax )
      return 0;
   const int step_min = 3, step_max = 3;
   const int M = rmax;
   double* V = malloc( sizeof( double ) * (size_t) n * ( M + 1 ) );
   double *r = malloc( sizeof( double ) * n ), *w = malloc( sizeof( double ) * n ), *tmp = malloc( sizeof( double ) * n );
   double* H = malloc( sizeof( double ) * ( M + 1 ) * M );
   double *sv = malloc( sizeof( double ) * ( M + 1 ) ), *cs = malloc( sizeof( double ) * ( M + 1 ) ),
          *sn = malloc( sizeof( double ) * ( M + 1 ) ), *y = malloc( sizeof( double ) * ( M + 1 ) ),
          *Hl = malloc( sizeof( double ) * ( M + 1 ) );
   double normb;
   if( s->diag ) {
      precond( s, b, tmp );
      normb = nrm2( n, tmp );
   }
   else
      normb = nrm2( n, b );
   if( normb == 0.0 )
      normb = 1.0;
   bicg_residue( s, r, x, b, tmp );
   double beta = nrm2( n, r );
   c->it = 0;
   c->res = beta / normb;
   double beta_ratio = 1;
   int restart_cycles = 0, m = rmax;
   int result = -1;
   while( check_next( c ) ) {
      if( rmax > rmin && restart_cycles > 0 ) {
         if( beta_ratio > 0.99 )
            m = rmax;
         else if( beta_ratio >= 0.175 ) {
            const int step = step_min + (int) ( (float) ( step_max - step_min ) / ( rmax - rmin ) * ( m - rmin ) );
            if( m - step >= rmin )
               m -= step;
            else
               m = rmax;
         }
      }
      /* Arnoldi */
      for( int i = 0; i < n; i++ )
         V[ i ] = ( 1.0 / beta ) * r[ i ];
      for( int i = 0; i < ( M + 1 ) * M; i++ )
         H[ i ] = 0.0;
      for( int i = 0; i <= M; i++ )
         sv[ i ] = 0.0;
      sv[ 0 ] = beta;
      int o_steps = m;
      for( int i = 0; i < m && next_iteration( c ); i++ ) {
         const double* vi = V + (size_t) i * n;
         bicg_matvec( s, vi, w, tmp );
         for( int k = 0; k <= i; k++ )
            H[ k + i * ( m + 1 ) ] = 0.0;
         if( variant == 0 || variant == 1 ) {
            const int reps = variant == 1 ? 2 : 1;
            for( int l = 0; l < reps; l++ ) {
               for( int k = 0; k <= i; k++ )
                  Hl[ k ] = dot( n, V + (size_t) k * n, w );
               for( int k = 0; k <= i; k++ )
                  H[ k + i * ( m + 1 ) ] += Hl[ k ];
               for( int j = 0; j < n; j++ ) {
                  double acc = 0.0;
                  for( int k = 0; k <= i; k++ )
                     acc += V[ (size_t) k * n + j ] * Hl[ k ];
                  w[ j ] = -1.0 * acc + 1.0 * w[ j ];
               }
            }
         }
         else {
            const int reps = variant == 3 ? 2 : 1;
            for( int l = 0; l < reps; l++ )
               for( int k = 0; k <= i; k++ ) {
                  const double* vk = V + (size_t) k * n;
                  const double hki = dot( n, w, vk );
                  H[ k + i * ( m + 1 ) ] += hki;
                  for( int j = 0; j < n; j++ )
                     w[ j ] = w[ j ] - hki * vk[ j ];
               }
         }
         const double normw = nrm2( n, w );
         H[ i + 1 + i * ( m + 1 ) ] = normw;
         double* vn = V + (size_t) ( i + 1 ) * n;
         for( int j = 0; j < n; j++ )
            vn[ j ] = ( 1.0 / normw ) * w[ j ];
         /* apply_givens_rotations */
         for( int k = 0; k < i; k++ )
            app_rot( &H[ k + i * ( m + 1 ) ], &H[ k + 1 + i * ( m + 1 ) ], cs[ k ], sn[ k ] );
         if( H[ i + 1 + i * ( m + 1 ) ] != 0.0 ) {
            gen_rot( H[ i + i * ( m + 1 ) ], H[ i + 1 + i * ( m + 1 ) ], &cs[ i ], &sn[ i ] );
            app_rot( &H[ i + i * ( m + 1 ) ], &H[ i + 1 + i * ( m + 1 ) ], cs[ i ], sn[ i ] );
            app_rot( &sv[ i ], &sv[ i + 1 ], cs[ i ], sn[ i ] );
         }
         c->res = fabs( sv[ i + 1 ] ) / normb;
         if( ! check_next( c ) ) {
            o_steps = i;
            break;
         }
      }
      /* o_steps < m: loop left by the check (i) or by nextIteration failing */
      {
         int k = ( o_steps < m ) ? o_steps : m - 1;
         /* when nextIteration() stopped the loop before step i ran, the
          * reference returns m from the orthogonalization (the for-condition
          * fails) and updates with m - 1 columns */
         for( int i = 0; i <= m; i++ )
            y[ i ] = sv[ i ];
         for( int i = k; i >= 0; i-- ) {
            if( H[ i + i * ( m + 1 ) ] == 0 ) {
               result = 0;
               goto done;
            }
            y[ i ] /= H[ i + i * ( m + 1 ) ];
            for( int j = i - 1; j >= 0; j-- )
               y[ j ] -= H[ j + i * ( m + 1 ) ] * y[ i ];
         }
         for( int j = 0; j < n; j++ ) {
            double acc = 0.0;
            for( int i = 0; i <= k; i++ )
               acc += V[ (size_t) i * n + j ] * y[ i ];
            x[ j ] = 1.0 * acc + 1.0 * x[ j ];
         }
      }
      if( o_steps < m ) {
         result = check_convergence( c );
         goto done;
      }
      bicg_residue( s, r, x, b, tmp );
      const double beta_old = beta;
      beta = nrm2( n, r );
      c->res = beta / normb;
      ++restart_cycles;
      beta_ratio = beta / beta_old;
   }
   result = check_convergence( c );
done:
   free( V );
   free( r );
   free( w );
   free( tmp );
   free( H );
   free( sv );
   free( cs );
   free( sn );
   free( y );
   free( Hl );
   return result;
}

/* Solvers/Linear/TFQMR.hpp:18-114. Iteration m (counted from 1 after
 * nextIteration) computes alpha in odd iterations and Au = M^-1 A u in even
 * ones; the residue estimate is tau sqrt(m + 1) / ||M^-1 b||. */
static int
solve_tfqmr( const sys_t* s, const double* b, double* x, ctl_t* c )
{
   const int n = s->n;
   double* buf = calloc( (size_t) 9 * ( n > 0 ? n : 1 ), sizeof( double ) );
   double *d = buf, *r = buf + n, *w = buf + 2 * n, *u = buf + 3 * n, *v = buf + 4 * n, *r_ast = buf + 5 * n,
          *Au = buf + 6 * n, *tmp = buf + 7 * n;
   double b_norm;
   if( s->diag ) {
      precond( s, b, tmp );
      b_norm = nrm2( n, tmp );
   }
   else
      b_norm = nrm2( n, b );
   bicg_residue( s, r, x, b, tmp );
   memcpy( w, r, sizeof( double ) * n );
   memcpy( u, r, sizeof( double ) * n );
   bicg_matvec( s, u, Au, tmp );
   memcpy( v, Au, sizeof( double ) * n );
   double tau = nrm2( n, r ), theta = 0.0, eta = 0.0, alpha = 0.0;
   memcpy( r_ast, r, sizeof( double ) * n );
   double rho = dot( n, r_ast, r );
   if( b_norm == 0.0 )
      b_norm = 1.0;
   c->it = 0;
   c->res = tau / b_norm;
   while( next_iteration( c ) ) {
      const long long iter = c->it;
      if( iter % 2 == 1 )
         alpha = rho / dot( n, v, r_ast );
      else
         bicg_matvec( s, u, Au, tmp );
      const double coef = theta * theta * eta / alpha;
      for( int i = 0; i < n; i++ ) {
         w[ i ] -= alpha * Au[ i ];
         d[ i ] = u[ i ] + coef * d[ i ];
      }
      theta = nrm2( n, w ) / tau;
      const double cc = 1.0 / sqrt( 1.0 + theta * theta );
      tau = tau * theta * cc;
      eta = cc * cc * alpha;
      for( int i = 0; i < n; i++ )
         x[ i ] += eta * d[ i ];
      c->res = tau * sqrt( (double) ( iter + 1 ) ) / b_norm;
      if( iter > 0 && c->res < c->tol )
         break;
      if( iter % 2 == 0 ) {
         const double rho_new = dot( n, w, r_ast );
         const double beta = rho_new / rho;
         rho = rho_new;
         for( int i = 0; i < n; i++ ) {
            u[ i ] = w[ i ] + beta * u[ i ];
            v[ i ] = beta * Au[ i ] + ( beta * beta ) * v[ i ];
         }
         bicg_matvec( s, u, Au, tmp );
         for( int i = 0; i < n; i++ )
            v[ i ] += Au[ i ];
      }
      else
         for( int i = 0; i < n; i++ )
            u[ i ] -= alpha * v[ i ];
   }
   free( buf );
   return check_convergence( c );
}

/* Solvers/Linear/BICGStabL.hpp:42-250: ell Bi-CG steps on the columns R_0..R_ell,
 * U_0..U_ell, then MGS of R_1..R_ell, the small triangular solves for g_0, g_2
 * and the updates of x, r_0, u_0. */
static int
solve_bicgstabl( const sys_t* s, const double* b, double* x, ctl_t* c, int ell, int exact )
{
   const int n = s->n;
   const size_t nn = (size_t) ( n > 0 ? n : 1 );
   double* R = calloc( ( ell + 1 ) * nn, sizeof( double ) );
   double* U = calloc( ( ell + 1 ) * nn, sizeof( double ) );
   double *r_ast = calloc( nn, sizeof( double ) ), *tmp = calloc( nn, sizeof( double ) ),
          *res = calloc( nn, sizeof( double ) );
   double* T = calloc( (size_t) ell * ell, sizeof( double ) );
   double *sigma = calloc( ell + 1, sizeof( double ) ), *g0 = calloc( ell + 1, sizeof( double ) ),
          *g1 = calloc( ell + 1, sizeof( double ) ), *g2 = calloc( ell + 1, sizeof( double ) );
   double b_norm;
   if( s->diag ) {
      precond( s, b, tmp );
      b_norm = nrm2( n, tmp );
   }
   else
      b_norm = nrm2( n, b );
   if( b_norm == 0.0 )
      b_norm = 1.0;
   bicg_residue( s, R, x, b, tmp );
   sigma[ 0 ] = nrm2( n, R );
   int ok = 0;
   if( isnan( sigma[ 0 ] ) ) {
      c->res = sigma[ 0 ];
      goto out;
   }
   for( int i = 0; i < n; i++ )
      r_ast[ i ] = R[ i ] / sigma[ 0 ];
   double rho_0 = 1.0, alpha = 0.0, omega = 1.0;
   c->it = 0;
   c->res = sigma[ 0 ] / b_norm;
   while( check_next( c ) ) {
      rho_0 = -omega * rho_0;
      for( int j = 0; j < ell; j++ ) {
         c->it++;
         const double rho_1 = dot( n, r_ast, R + (size_t) j * nn );
         const double beta = alpha * rho_1 / rho_0;
         rho_0 = rho_1;
         for( int q = 0; q <= j; q++ )
            for( int i = 0; i < n; i++ )
               U[ q * nn + i ] = R[ q * nn + i ] - beta * U[ q * nn + i ];
         bicg_matvec( s, U + (size_t) j * nn, U + (size_t) ( j + 1 ) * nn, tmp );
         const double gamma = dot( n, r_ast, U + (size_t) ( j + 1 ) * nn );
         alpha = rho_0 / gamma;
         for( int q = 0; q <= j; q++ )
            for( int i = 0; i < n; i++ )
               R[ q * nn + i ] -= alpha * U[ ( q + 1 ) * nn + i ];
         bicg_matvec( s, R + (size_t) j * nn, R + (size_t) ( j + 1 ) * nn, tmp );
         for( int i = 0; i < n; i++ )
            x[ i ] += alpha * U[ i ];
      }
      for( int j = 1; j <= ell; j++ ) {
         double* rj = R + (size_t) j * nn;
         for( int i = 1; i < j; i++ ) {
            const int ij = ( i - 1 ) + ( j - 1 ) * ell;
            T[ ij ] = dot( n, R + (size_t) i * nn, rj ) / sigma[ i ];
            for( int k = 0; k < n; k++ )
               rj[ k ] -= T[ ij ] * R[ i * nn + k ];
         }
         sigma[ j ] = dot( n, rj, rj );
         g1[ j ] = dot( n, R, rj ) / sigma[ j ];
      }
      omega = g1[ ell ];
      for( int j = ell; j >= 1; j-- ) {
         g0[ j ] = g1[ j ];
         for( int i = j + 1; i <= ell; i++ )
            g0[ j ] -= T[ ( j - 1 ) + ( i - 1 ) * ell ] * g0[ i ];
      }
      for( int j = 1; j < ell; j++ ) {
         g2[ j ] = g0[ j + 1 ];
         for( int i = j + 1; i < ell; i++ )
            g2[ j ] += T[ ( j - 1 ) + ( i - 1 ) * ell ] * g0[ i + 1 ];
      }
      g2[ 0 ] = g0[ 1 ];
      for( int i = 0; i < n; i++ ) {
         double ax = 0.0, ar = 0.0, au = 0.0;
         for( int k = 0; k < ell; k++ ) {
            ax += R[ k * nn + i ] * g2[ k ];
            ar += R[ ( k + 1 ) * nn + i ] * -g1[ k + 1 ];
            au += U[ ( k + 1 ) * nn + i ] * -g0[ k + 1 ];
         }
         x[ i ] = ax + x[ i ];
         R[ i ] = ar + R[ i ];
         U[ i ] = au + U[ i ];
      }
      if( exact ) {
         bicg_residue( s, res, x, b, tmp );
         sigma[ 0 ] = nrm2( n, res );
      }
      else
         sigma[ 0 ] = nrm2( n, R );
      c->res = sigma[ 0 ] / b_norm;
   }
   ok = check_convergence( c );
out:
   free( R );
   free( U );
   free( r_ast );
   free( tmp );
   free( res );
   free( T );
   free( sigma );
   free( g0 );
   free( g1 );
   free( g2 );
   return ok;
}

int
b2so_solve( int solver, int precond_kind, int rows, const int* offsets, const int* columns, const double* values,
            const double* b, double* x, double rtol, long long maxit, int gmres_variant, int restart_min, int restart_max,
            int exact_residue, int ell, long long* iters, double* residue )
{
   sys_t s = { rows, offsets, columns, values, NULL };
   double* diag = NULL;
   if( precond_kind ) {
      /* Preconditioners/Diagonal.hpp:20-40: diag[i] = A(i,i) (0 if absent) */
      diag = (double*) calloc( rows > 0 ? rows : 1, sizeof( double ) );
      for( int r = 0; r < rows; r++ )
         for( int k = offsets[ r ]; k < offsets[ r + 1 ]; k++ )
            if( columns[ k ] == r ) {
               diag[ r ] = values[ k ];
               break;
            }
      s.diag = diag;
   }
   ctl_t c = { 0, maxit, 0.0, rtol };
   int ok;
   if( solver == 0 )
      ok = solve_cg( &s, b, x, &c );
   else if( solver == 1 )
      ok = solve_bicgstab( &s, b, x, &c, exact_residue );
   else if( solver == 2 )
      ok = solve_gmres( &s, b, x, &c, gmres_variant, restart_min, restart_max );
   else if( solver == 3 )
      ok = solve_tfqmr( &s, b, x, &c );
   else
      ok = solve_bicgstabl( &s, b, x, &c, ell > 0 ? ell : 1, exact_residue );
   *iters = c.it;
   *residue = c.res;
   free( diag );
   return ok;
}

/* SymmetricMatrix product (Matrices/SparseMatrixView.hpp:413-476): the CSR
 * arrays hold the lower triangle; y *= beta (unless beta is 1), then every row i
 * of [begin, end) adds alpha v x_i to y_j for its elements (i, j, v) with j < i,
 * and alpha times its row sum of v x_j to y_i (rows in order). */
void
b2so_spmv_symmetric( int rows, const int* off, const int* col, const double* val, const double* x, double* y,
                     double alpha, double beta, int begin, int end )
{
   if( end == 0 )
      end = rows;
   if( beta != 1.0 )
      for( int i = 0; i < rows; i++ )
         y[ i ] = beta * y[ i ];
   for( int r = begin; r < end; r++ ) {
      double s = 0.0;
      for( int k = off[ r ]; k < off[ r + 1 ]; k++ ) {
         const int j = col[ k ];
         if( j < r )
            y[ j ] += alpha * val[ k ] * x[ r ];
         const double p = val[ k ] * x[ j ];
         s = s + p;
      }
      y[ r ] += alpha * s;
   }
}

/* ------------------------------------------------------------------------
 * Permutations — Matrices/MatrixPermutationApplier.h and
 * Matrices/SparseOperations_impl.h, restated for CSR matrices.
 */

/* permuteMatrixRows (MatrixPermutationApplier.h:17-62): row i of the result is
 * row perm[i], its slots copied in order (for CSR the capacity of a row is its
 * length). */
int
b2so_permute_rows( b2so_matrix* m, const int* perm )
{
   if( m->format != 0 )
      return -1;
   const int n = m->rows;
   int* off = (int*) malloc( sizeof( int ) * ( n + 1 ) );
   off[ 0 ] = 0;
   for( int i = 0; i < n; i++ )
      off[ i + 1 ] = off[ i ] + ( m->offsets[ perm[ i ] + 1 ] - m->offsets[ perm[ i ] ] );
   const long long st = off[ n ];
   double* val = (double*) malloc( sizeof( double ) * ( st > 0 ? st : 1 ) );
   int* col = (int*) malloc( sizeof( int ) * ( st > 0 ? st : 1 ) );
   for( int i = 0; i < n; i++ ) {
      const int b = m->offsets[ perm[ i ] ], len = m->offsets[ perm[ i ] + 1 ] - b;
      for( int k = 0; k < len; k++ ) {
         val[ off[ i ] + k ] = m->values[ b + k ];
         col[ off[ i ] + k ] = m->columns[ b + k ];
      }
   }
   free( m->values );
   free( m->columns );
   memcpy( m->offsets, off, sizeof( int ) * ( n + 1 ) );
   free( off );
   m->values = val;
   m->columns = col;
   /* refresh the exported "offsets" array */
   for( int i = 0; i < m->nmeta; i++ )
      if( strcmp( m->meta[ i ].name, "offsets" ) == 0 )
         for( int r = 0; r <= n; r++ )
            m->meta[ i ].v[ r ] = m->offsets[ r ];
   return 0;
}

/* permuteMatrixColumns (MatrixPermutationApplier.h:64-90): every stored column
 * c becomes iperm[c]; a row stops at its first padding slot; the slots keep
 * their order (rows are not re-sorted). Any layout. */
int
b2so_permute_columns( b2so_matrix* m, const int* iperm )
{
   for( int r = 0; r < m->rows; r++ ) {
      const int len = segment_size( m, r );
      for( int k = 0; k < len; k++ ) {
         const long long g = gidx( m, r, k );
         if( m->columns[ g ] == PADDING_INDEX )
            break;
         m->columns[ g ] = iperm[ m->columns[ g ] ];
      }
   }
   return 0;
}

/* reorderSparseMatrix (SparseOperations_impl.h:253-312): a new CSR matrix whose
 * row i is row perm[i] with columns mapped by iperm and sorted ascending. */
b2so_matrix*
b2so_reorder( int rows, int cols, const int* offsets, const int* columns, const double* values, const int* perm,
              const int* iperm )
{
   int* off = (int*) malloc( sizeof( int ) * ( rows + 1 ) );
   off[ 0 ] = 0;
   for( int i = 0; i < rows; i++ )
      off[ i + 1 ] = off[ i ] + ( offsets[ perm[ i ] + 1 ] - offsets[ perm[ i ] ] );
   const long long st = off[ rows ];
   int* col = (int*) malloc( sizeof( int ) * ( st > 0 ? st : 1 ) );
   double* val = (double*) malloc( sizeof( double ) * ( st > 0 ? st : 1 ) );
   for( int i = 0; i < rows; i++ ) {
      const int b = offsets[ perm[ i ] ], len = offsets[ perm[ i ] + 1 ] - b;
      int* c = col + off[ i ];
      double* v = val + off[ i ];
      for( int k = 0; k < len; k++ ) {
         c[ k ] = iperm[ columns[ b + k ] ];
         v[ k ] = values[ b + k ];
      }
      /* insertion sort by column (distinct columns: the same order as std::sort) */
      for( int k = 1; k < len; k++ ) {
         const int ck = c[ k ];
         const double vk = v[ k ];
         int j = k - 1;
         while( j >= 0 && c[ j ] > ck ) {
            c[ j + 1 ] = c[ j ];
            v[ j + 1 ] = v[ j ];
            j--;
         }
         c[ j + 1 ] = ck;
         v[ j + 1 ] = vk;
      }
   }
   b2so_matrix* m = b2so_create( 0, 0, 0, rows, cols, off, col, val );
   free( off );
   free( col );
   free( val );
   return m;
}

/* ILU(0) of a CSR matrix with rows sorted by column and a stored diagonal,
 * then x = U^-1 L^-1 b (Solvers/Linear/Preconditioners/ILU0.hpp:23-144,
 * Utils/TriangularSolve.h:24-110). The factors live in A's pattern: L (unit
 * diagonal) strictly below, U on and above the diagonal. Row i, for each
 * L entry k in increasing order: L_ik /= U_kk, then every later entry j of
 * the row takes -= L_ik * U_kj (0 when U has no (k, j)). `fused` bit 0 / 3:
 * the updates of the row's U part / L part as fused multiply-adds, bit 1 / 2:
 * the forward / backward sums, bit 4: the sums grouped as described below.
 * The reference build (g++ -O3 -march=x86-64-v3) contracts the updates in
 * both precisions, leaves the FP64 sums uncontracted and vectorizes the FP32
 * sums by four.
 * Returns -1 when a diagonal entry is missing. */
static double
ilu_msub( double a, double l, double u, int fused, int real )
{
   if( real ) {
      const float r = fused ? fmaf( -(float) l, (float) u, (float) a ) : (float) a - (float) l * (float) u;
      return r;
   }
   return fused ? fma( -l, u, a ) : a - l * u;
}

int
b2so_ilu0_apply( int real, int fused, int rows, const int* off, const int* col, const double* val, const double* b,
                 double* x )
{
   const long long nnz = off[ rows ];
   double* lu = (double*) malloc( sizeof( double ) * ( nnz > 0 ? nnz : 1 ) );
   int* dg = (int*) malloc( sizeof( int ) * ( rows > 0 ? rows : 1 ) );
   for( long long k = 0; k < nnz; k++ )
      lu[ k ] = real ? (double) (float) val[ k ] : val[ k ];
   for( int i = 0; i < rows; i++ ) {
      dg[ i ] = -1;
      for( int k = off[ i ]; k < off[ i + 1 ]; k++ )
         if( col[ k ] == i )
            dg[ i ] = k;
      if( dg[ i ] < 0 ) {
         free( lu );
         free( dg );
         return -1;
      }
   }
   for( int i = 0; i < rows; i++ ) {
      for( int ck = off[ i ]; ck < dg[ i ]; ck++ ) {
         const int k = col[ ck ];
         const double lik = real ? (double) ( (float) lu[ ck ] / (float) lu[ dg[ k ] ] ) : lu[ ck ] / lu[ dg[ k ] ];
         lu[ ck ] = lik;
         for( int cj = ck + 1; cj < off[ i + 1 ]; cj++ ) {
            double u = 0.0;
            for( int q = dg[ k ]; q < off[ k + 1 ]; q++ )
               if( col[ q ] == col[ cj ] )
                  u = lu[ q ];
            /* the L part and the U part of the row are separate loops in TNL */
            const int f = cj < dg[ i ] ? ( fused >> 3 ) & 1 : fused & 1;
            lu[ cj ] = ilu_msub( lu[ cj ], lik, u, f, real );
         }
      }
   }
   /* L y = b (unit lower), then U x = y. With bit 4 the terms of a row go in
    * groups of four with separately rounded products and the remaining
    * (count mod 4) terms as fused multiply-adds — the reference build's
    * vectorized FP32 loop and its scalar epilogue. */
   for( int i = 0; i < rows; i++ ) {
      double t = real ? (double) (float) b[ i ] : b[ i ];
      const int m = dg[ i ] - off[ i ], nv = m / 4 * 4;
      for( int k = off[ i ]; k < dg[ i ]; k++ ) {
         const int f = ( fused & 16 ) ? ( k - off[ i ] >= nv ) : ( fused >> 1 ) & 1;
         t = ilu_msub( t, lu[ k ], x[ col[ k ] ], f, real );
      }
      x[ i ] = t;
   }
   for( int i = rows - 1; i >= 0; i-- ) {
      double t = x[ i ];
      const int m = off[ i + 1 ] - dg[ i ] - 1, nv = m / 4 * 4;
      for( int k = dg[ i ] + 1; k < off[ i + 1 ]; k++ ) {
         const int f = ( fused & 16 ) ? ( k - dg[ i ] - 1 >= nv ) : ( fused >> 2 ) & 1;
         t = ilu_msub( t, lu[ k ], x[ col[ k ] ], f, real );
      }
      x[ i ] = real ? (double) ( (float) t / (float) lu[ dg[ i ] ] ) : t / lu[ dg[ i ] ];
   }
   free( lu );
   free( dg );
   return 0;
}
