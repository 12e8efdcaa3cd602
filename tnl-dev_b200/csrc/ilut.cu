// ILUT( p, tau ): Preconditioners::ILUT (Solvers/Linear/Preconditioners/ILUT.hpp:33-289).
//
// TNL provides ILUT on Devices::Host only (its Devices::Cuda specialization,
// ILUT.h:156-179, throws "Not implemented"). Here the factorization is TNL's
// host algorithm, run on the host once per update (it is sequential in the
// rows and keeps a sorted set and heaps per row), and the factors are applied
// on the device by the ILU(0) dependency kernels (ilu.cuh).
//
// The factorization, row by row (Saad, Iterative Methods for Sparse Linear
// Systems, 2nd ed., sec. 10.4, with TNL's own choices kept for parity):
//  * row i of A (its stored elements in row order) goes into a dense work row
//    w; tau_i = tau * ||A_i||_2;
//  * for the nonzero columns k < i of w in increasing order, fill-in included:
//    w_k = w_k / A_kk (A's diagonal element), dropped when |w_k| < tau_i; a kept
//    w_k takes w_k U_kj off w_j for every stored entry of U's row k — its
//    diagonal j = k included, so the L_ik that is stored is w_k - w_k U_kk;
//  * the entries of w with |w_j| >= tau_i, in increasing column order, form an
//    L list (j < i) and a U list (j >= i), each made a max-heap by magnitude
//    (std::make_heap); entries are popped while the count taken is below both
//    the row's capacity in that factor (A's entries of that part + p) and the
//    heap's remaining size, which keeps at most ceil(size / 2) of them;
//  * the kept entries are stored sorted by column.
// The heaps use the standard library's make_heap / pop_heap on the same
// sequences as the reference, so ties in magnitude resolve the same way.
//
// Arithmetic as the reference build (g++ -O3 -march=x86-64-v3) evaluates it:
// the updates w_j - w_k U_kj and the row norm's squares are fused
// multiply-adds (std::fma); the substitutions subtract rounded products in
// stored order and divide by the first stored U entry of the row.
//
// The factors are stored row by row as [L entries | U entries] in the ILU(0)
// structure, the U part starting at diag[i]. A row whose U list came out empty
// gets an explicit zero there: TNL divides by the (zero) value of the row's
// first, unused U slot.
#include "ilu.cuh"

#include <algorithm>
#include <cmath>
#include <set>
#include <utility>
#include <vector>

namespace b2s {

namespace {

template< typename Real >
struct Candidate
{
   int32_t column;
   Real value;
   Real magnitude;
};

// the rows of A in storage order (a padded layout's rows without padding),
// values in Real, on the host
template< typename Real >
b2s_status
host_rows( const b2s_matrix_t* A, std::vector< int32_t >& off, std::vector< int32_t >& col, std::vector< Real >& val,
           cudaStream_t s )
{
   const int32_t n = A->rows;
   DevBuf doff, dcol, dval;
   int64_t nnz = A->nnz;
   const int32_t* po = nullptr;
   const int32_t* pc = nullptr;
   const void* pv = nullptr;
   if( A->format == B2S_CSR ) {
      po = A->offsets.as< int32_t >();
      pc = A->columns.as< int32_t >();
      pv = A->values.p;
   }
   else {
      B2S_TRY( layout_to_csr( A, false, doff, dcol, dval, nnz, s ) );
      po = doff.as< int32_t >();
      pc = dcol.as< int32_t >();
      pv = dval.p;
   }
   off.assign( (size_t) n + 1, 0 );
   col.assign( (size_t) std::max< int64_t >( nnz, 1 ), 0 );
   val.assign( (size_t) std::max< int64_t >( nnz, 1 ), Real( 0 ) );
   if( n > 0 )
      B2S_TRY( copy_d2h( off.data(), po, off.size() * sizeof( int32_t ), s ) );
   if( nnz > 0 ) {
      B2S_TRY( copy_d2h( col.data(), pc, (size_t) nnz * sizeof( int32_t ), s ) );
      if( A->dtype == B2S_F64 ) {
         std::vector< double > v( (size_t) nnz );
         B2S_TRY( copy_d2h( v.data(), pv, (size_t) nnz * sizeof( double ), s ) );
         for( int64_t k = 0; k < nnz; k++ )
            val[ k ] = (Real) v[ k ];
      }
      else {
         std::vector< float > v( (size_t) nnz );
         B2S_TRY( copy_d2h( v.data(), pv, (size_t) nnz * sizeof( float ), s ) );
         for( int64_t k = 0; k < nnz; k++ )
            val[ k ] = (Real) v[ k ];
      }
   }
   return B2S_OK;
}

}  // namespace

template< typename Real >
b2s_status
ilut_factorize( const b2s_matrix_t* A, int32_t p, double tau_d, IluFactors< Real >& F, cudaStream_t s )
{
   if( A->rows != A->cols ) {
      set_error( "ILUT needs a square matrix" );
      return B2S_INVALID_ARG;
   }
   if( p < 0 ) {
      set_error( "ILUT: p must not be negative" );
      return B2S_INVALID_ARG;
   }
   const int32_t n = A->rows;
   const Real tau = (Real) tau_d;
   std::vector< int32_t > off, col;
   std::vector< Real > val;
   B2S_TRY( host_rows< Real >( A, off, col, val, s ) );

   // A_kk as getElement( k, k ) reads it: the first element of row k in column k, else 0
   std::vector< Real > adiag( (size_t) std::max( n, 1 ), Real( 0 ) );
   std::vector< int32_t > lcap( (size_t) std::max( n, 1 ) ), ucap( (size_t) std::max( n, 1 ) );
   for( int32_t i = 0; i < n; i++ ) {
      int32_t nl = 0, nu = 0;
      bool seen = false;
      for( int32_t k = off[ i ]; k < off[ i + 1 ]; k++ ) {
         const int32_t j = col[ k ];
         if( j == i && ! seen ) {
            adiag[ i ] = val[ k ];
            seen = true;
         }
         if( j < i )
            nl++;
         else if( j < n )
            nu++;
      }
      lcap[ i ] = nl + p;
      ucap[ i ] = nu + p;
   }

   // U's rows as they are produced (the k loop reads them), and the output
   std::vector< std::vector< std::pair< int32_t, Real > > > urows( (size_t) n );
   std::vector< int32_t > foff( (size_t) n + 1, 0 ), fdiag( (size_t) std::max( n, 1 ) );
   std::vector< int32_t > fcol;
   std::vector< Real > fval;
   std::vector< Real > w( (size_t) std::max( n, 1 ), Real( 0 ) );
   std::set< int32_t > nz;
   std::vector< Candidate< Real > > heap_l, heap_u, keep_l, keep_u;
   auto by_magnitude = []( const Candidate< Real >& a, const Candidate< Real >& b ) { return a.magnitude < b.magnitude; };
   auto by_column = []( const Candidate< Real >& a, const Candidate< Real >& b ) { return a.column < b.column; };
   auto extract = [ & ]( std::vector< Candidate< Real > >& heap, int32_t cap, std::vector< Candidate< Real > >& out )
   {
      std::make_heap( heap.begin(), heap.end(), by_magnitude );
      for( int32_t c = 0; c < cap && c < (int32_t) heap.size(); c++ ) {
         std::pop_heap( heap.begin(), heap.end(), by_magnitude );
         out.push_back( heap.back() );
         heap.pop_back();
      }
      std::sort( out.begin(), out.end(), by_column );
   };

   for( int32_t i = 0; i < n; i++ ) {
      Real norm = 0;
      nz.clear();
      for( int32_t k = off[ i ]; k < off[ i + 1 ]; k++ ) {
         const int32_t j = col[ k ];
         w[ j ] = val[ k ];
         norm = std::fma( w[ j ], w[ j ], norm );
         nz.insert( j );
      }
      const Real tau_i = tau * std::sqrt( norm );
      for( auto it = nz.begin(); it != nz.end() && *it < i; ++it ) {
         const int32_t k = *it;
         Real wk = w[ k ] / adiag[ k ];
         if( std::abs( wk ) < tau_i )
            wk = 0;
         w[ k ] = wk;
         if( wk != Real( 0 ) )
            for( const auto& e : urows[ k ] ) {
               w[ e.first ] = std::fma( -wk, e.second, w[ e.first ] );
               nz.insert( e.first );  // columns >= k: visited later (or k itself, present)
            }
      }
      for( const int32_t j : nz ) {
         const Real m = std::abs( w[ j ] );
         if( m < tau_i )
            continue;
         ( j < i ? heap_l : heap_u ).push_back( Candidate< Real >{ j, w[ j ], m } );
      }
      extract( heap_l, lcap[ i ], keep_l );
      extract( heap_u, ucap[ i ], keep_u );
      for( const auto& e : keep_l ) {
         fcol.push_back( e.column );
         fval.push_back( e.value );
      }
      fdiag[ i ] = (int32_t) fcol.size();
      if( keep_u.empty() ) {
         fcol.push_back( i );
         fval.push_back( Real( 0 ) );
      }
      for( const auto& e : keep_u ) {
         fcol.push_back( e.column );
         fval.push_back( e.value );
         urows[ i ].emplace_back( e.column, e.value );
      }
      if( fcol.size() > (size_t) INT32_MAX ) {
         set_error( "ILUT: more than 2^31 - 1 factor entries" );
         return B2S_INDEX_OVERFLOW;
      }
      foff[ i + 1 ] = (int32_t) fcol.size();
      for( const int32_t j : nz )
         w[ j ] = 0;
      heap_l.clear();
      heap_u.clear();
      keep_l.clear();
      keep_u.clear();
   }

   // the factors on the device in the ILU(0) structure
   F.n = n;
   const size_t nf = std::max< size_t >( fcol.size(), 1 );
   B2S_TRY( F.off_own.alloc( ( (size_t) n + 1 ) * sizeof( int32_t ) ) );
   B2S_TRY( F.col_own.alloc( nf * sizeof( int32_t ) ) );
   B2S_TRY( F.lu.alloc( nf * sizeof( Real ) ) );
   B2S_TRY( F.diag.alloc( (size_t) std::max( n, 1 ) * sizeof( int32_t ) ) );
   B2S_TRY( F.flags.alloc( (size_t) std::max( n, 1 ) * sizeof( int32_t ) ) );
   B2S_TRY( F.state.alloc( sizeof( IluState ) ) );
   B2S_TRY_CUDA( cudaMemsetAsync( F.flags.p, 0, (size_t) std::max( n, 1 ) * sizeof( int32_t ), s ) );
   B2S_TRY_CUDA( cudaMemsetAsync( F.state.p, 0, sizeof( IluState ), s ) );
   B2S_TRY( copy_h2d( F.off_own.p, foff.data(), foff.size() * sizeof( int32_t ), s ) );
   if( ! fcol.empty() ) {
      B2S_TRY( copy_h2d( F.col_own.p, fcol.data(), fcol.size() * sizeof( int32_t ), s ) );
      B2S_TRY( copy_h2d( F.lu.p, fval.data(), fval.size() * sizeof( Real ), s ) );
   }
   if( n > 0 )
      B2S_TRY( copy_h2d( F.diag.p, fdiag.data(), (size_t) n * sizeof( int32_t ), s ) );
   F.off = F.off_own.template as< int32_t >();
   F.col = F.col_own.template as< int32_t >();
   F.plain_sum = true;
   if( n == 0 )
      return B2S_OK;
   B2S_TRY( ilu_levels( F, foff, fcol, fdiag, s ) );
   B2S_TRY_CUDA( cudaStreamSynchronize( s ) );
   return B2S_OK;
}

template b2s_status ilut_factorize< double >( const b2s_matrix_t*, int32_t, double, IluFactors< double >&, cudaStream_t );
template b2s_status ilut_factorize< float >( const b2s_matrix_t*, int32_t, double, IluFactors< float >&, cudaStream_t );

}  // namespace b2s
