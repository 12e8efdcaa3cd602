// Drop-in check of the TNL-shaped C++ interface (tnl-dev_b200/include/TNL/b2s_tnl.h):
// the matrices of TNL's SparseMatrixVectorProductTest
// (src/UnitTests/Matrices/SparseMatrixVectorProductTest.hpp) assembled through
// setRowCapacities / setElement, multiplied with vectorProduct on the GPU, for
// every segment type and Real in {double, float, bool}; then CG, BiCGStab, GMRES, TFQMR and BiCGStab(ell)
// through setMatrix / setup / solve. Exit status 0 = all checks passed.
#include <TNL/b2s_tnl.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <functional>
#include <memory>

using namespace TNL;
namespace Seg = TNL::Algorithms::Segments;

static int failures = 0;

#define EXPECT( cond, ... )                          \
   do {                                              \
      if( ! ( cond ) ) {                             \
         failures++;                                 \
         std::printf( "FAIL %s:%d ", __FILE__, __LINE__ ); \
         std::printf( __VA_ARGS__ );                 \
         std::printf( "\n" );                        \
      }                                              \
   } while( 0 )

template< typename Matrix >
static void
product_check( const char* name, Matrix& m, typename Matrix::RealType xval, const std::vector< double >& expected )
{
   using Real = typename Matrix::RealType;
   Containers::Vector< Real, Devices::Cuda, int > in( m.getColumns(), xval ), out( m.getRows(), Real( 0 ) );
   m.vectorProduct( in, out );
   const auto y = out.toStdVector();
   for( size_t i = 0; i < expected.size(); i++ )
      EXPECT( (double) y[ i ] == expected[ i ], "%s row %zu: %g != %g", name, i, (double) y[ i ], expected[ i ] );
}

// Rows given as lists of (column, value); capacities = row lengths (+ extra slack).
template< typename Matrix >
static void
assemble( Matrix& m, int rows, int cols, const std::vector< std::vector< std::pair< int, double > > >& e, int slack = 0 )
{
   m.setDimensions( rows, cols );
   typename Matrix::RowsCapacitiesType caps( rows );
   for( int r = 0; r < rows; r++ )
      caps[ r ] = (int) e[ r ].size() + slack;
   m.setRowCapacities( caps );
   for( int r = 0; r < rows; r++ )
      for( auto& p : e[ r ] )
         m.setElement( r, p.first, ( typename Matrix::RealType ) p.second );
}

template< typename Real, template< typename, typename, typename > class S >
static void
run_products()
{
   using M = Matrices::SparseMatrix< Real, Devices::Cuda, int, Matrices::GeneralMatrix, S >;
   {
      M m;
      assemble( m, 4, 4, { { { 0, 1 } }, { { 1, 2 }, { 3, 3 } }, { { 1, 4 } }, { { 2, 5 } } } );
      product_check( "small1", m, 2, { 2, 10, 8, 10 } );
   }
   {
      M m;
      assemble( m, 4, 4, { { { 0, 1 }, { 1, 2 }, { 2, 3 } }, { { 3, 4 } }, { { 0, 5 }, { 1, 6 }, { 2, 7 } }, { { 1, 8 } } } );
      product_check( "small2", m, 2, { 12, 8, 36, 16 } );
   }
   {
      M m;
      assemble( m, 4, 4,
                { { { 0, 1 }, { 1, 2 }, { 2, 3 } },
                  { { 1, 4 }, { 2, 5 }, { 3, 6 } },
                  { { 0, 7 }, { 1, 8 }, { 2, 9 } },
                  { { 1, 10 }, { 2, 11 }, { 3, 12 } } },
                1 );  // one unused slot per row: padding in every layout but CSR
      product_check( "small3", m, 2, { 12, 30, 48, 66 } );
   }
   {
      // 8x8 with row lengths 4,4,5,4,4,4,5,5 and consecutive values
      const int starts[ 8 ] = { 0, 1, 0, 1, 2, 3, 0, 0 }, lens[ 8 ] = { 4, 4, 5, 4, 4, 4, 5, 5 };
      std::vector< std::vector< std::pair< int, double > > > e( 8 );
      int v = 1;
      for( int r = 0; r < 8; r++ ) {
         if( r == 0 ) {
            for( int c : { 0, 1, 2, 5 } )
               e[ 0 ].push_back( { c, v++ } );
            continue;
         }
         for( int c = starts[ r ]; c < starts[ r ] + lens[ r ]; c++ )
            e[ r ].push_back( { c, v++ } );
      }
      M m;
      assemble( m, 8, 8, e );
      product_check( "medium1", m, 2, { 20, 52, 110, 124, 156, 188, 280, 330 } );
   }
   {
      const int size = 1051;
      std::vector< std::vector< std::pair< int, double > > > diag( size ), tri( size );
      std::vector< double > ed( size ), et( size );
      for( int i = 0; i < size; i++ ) {
         diag[ i ].push_back( { i, i + 1.0 } );
         for( int j = 0; j <= i; j++ )
            tri[ i ].push_back( { j, j + 1.0 } );
         ed[ i ] = i + 1;
         et[ i ] = ( i + 1.0 ) * ( i + 2.0 ) / 2.0;
      }
      M m1, m2;
      assemble( m1, size, size, diag );
      product_check( "large_diagonal", m1, 1, ed );
      assemble( m2, size, size, tri );
      product_check( "large_triangular", m2, 1, et );
   }
   for( int columns : { 64, 65, 128, 129, 256, 257, 512, 513, 1024, 1025, 2048, 2049, 3000 } ) {
      std::vector< std::vector< std::pair< int, double > > > e( 33 );
      std::vector< double > ex( 33 );
      for( int r = 0; r < 33; r++ ) {
         for( int c = 0; c < columns; c++ )
            e[ r ].push_back( { c, (double) ( c + r ) } );
         ex[ r ] = (double) columns * ( columns - 1 ) / 2.0 + (double) columns * r;
      }
      M m;
      assemble( m, 33, columns, e );
      product_check( "long_rows", m, 1, ex );
   }
}

template< template< typename > class Solver, template< typename > class Pre = Solvers::Linear::Preconditioners::ILU0 >
static void
run_solver( const char* name, bool nonsymmetric, const char* variant, int ell = 1, bool ilu = false )
{
   using M = Matrices::SparseMatrix< double, Devices::Cuda, int >;
   const int nx = 40, n = nx * nx;
   auto A = std::make_shared< M >( n, n );
   typename M::RowsCapacitiesType caps( n );
   for( int i = 0; i < n; i++ )
      caps[ i ] = 5;
   A->setRowCapacities( caps );
   for( int j = 0; j < nx; j++ )
      for( int i = 0; i < nx; i++ ) {
         const int r = i + nx * j;
         A->setElement( r, r, 4.0 + ( nonsymmetric ? 0.5 : 0.0 ) );
         if( i > 0 )
            A->setElement( r, r - 1, nonsymmetric ? -1.5 : -1.0 );
         if( i < nx - 1 )
            A->setElement( r, r + 1, nonsymmetric ? -0.5 : -1.0 );
         if( j > 0 )
            A->setElement( r, r - nx, -1.0 );
         if( j < nx - 1 )
            A->setElement( r, r + nx, -1.0 );
      }
   Containers::Vector< double, Devices::Cuda, int > ones( n, 1.0 ), b( n ), x( n, 0.0 );
   A->vectorProduct( ones, b );
   Solver< M > solver;
   Config::ParameterContainer params;
   params.addParameter< std::string >( "gmres-variant", variant );
   params.addParameter< int >( "gmres-restarting-min", 30 );
   params.addParameter< int >( "gmres-restarting-max", 30 );
   params.addParameter< int >( "bicgstab-ell", ell );
   EXPECT( solver.setup( params ), "%s setup", name );
   solver.setMatrix( A );
   if( ilu ) {
      auto pre = std::make_shared< Pre< M > >();
      pre->update( A );
      solver.setPreconditioner( pre );
   }
   solver.setConvergenceResidue( 1e-10 );
   const bool ok = solver.solve( b, x );
   EXPECT( ok, "%s did not converge (%d iterations, residue %g)", name, solver.getIterations(), solver.getResidue() );
   const auto h = x.toStdVector();
   double err = 0;
   for( double v : h )
      err = std::max( err, std::fabs( v - 1.0 ) );
   EXPECT( err < 1e-7, "%s error %g", name, err );
   std::printf( "%s: %d iterations, residue %.3e, max error %.3e\n", name, solver.getIterations(), solver.getResidue(),
                err );
}

// SparseMatrix< double, Cuda, int, SymmetricMatrix, S >: a 2D Laplacian given by
// elements on both sides of the diagonal (stored once, in the lower triangle),
// its product against the full matrix computed on the host, and a CG solve
template< template< typename, typename, typename > class S >
static void
run_symmetric( const char* label )
{
   using M = Matrices::SparseMatrix< double, Devices::Cuda, int, Matrices::SymmetricMatrix, S >;
   const int nx = 30, n = nx * nx;
   auto A = std::make_shared< M >( n, n );
   typename M::RowsCapacitiesType caps( n );
   for( int i = 0; i < n; i++ )
      caps[ i ] = 3;  // the diagonal and the two lower neighbours
   A->setRowCapacities( caps );
   std::vector< std::vector< std::pair< int, double > > > full( n );
   for( int j = 0; j < nx; j++ )
      for( int i = 0; i < nx; i++ ) {
         const int r = i + nx * j;
         full[ r ].push_back( { r, 4.0 } );
         A->setElement( r, r, 4.0 );
         const int nb[ 4 ] = { i > 0 ? r - 1 : -1, i < nx - 1 ? r + 1 : -1, j > 0 ? r - nx : -1, j < nx - 1 ? r + nx : -1 };
         for( int c : nb )
            if( c >= 0 ) {
               full[ r ].push_back( { c, -1.0 } );
               A->setElement( r, c, -1.0 );  // the upper ones land on the stored lower element
            }
      }
   EXPECT( A->getElement( 0, 1 ) == -1.0 && A->getElement( 1, 0 ) == -1.0, "symmetric getElement" );
   std::vector< double > xs( n ), want( n, 0.0 );
   for( int i = 0; i < n; i++ )
      xs[ i ] = std::sin( 0.1 * i );
   for( int r = 0; r < n; r++ )
      for( const auto& e : full[ r ] )
         want[ r ] += e.second * xs[ e.first ];
   Containers::Vector< double, Devices::Cuda, int > x( n ), y( n, 0.0 );
   for( int i = 0; i < n; i++ )
      x.setElement( i, xs[ i ] );
   A->vectorProduct( x, y );
   const auto h = y.toStdVector();
   double err = 0;
   for( int i = 0; i < n; i++ )
      err = std::max( err, std::fabs( h[ i ] - want[ i ] ) );
   EXPECT( err < 1e-12, "symmetric product error %g", err );
   Containers::Vector< double, Devices::Cuda, int > b( n ), xx( n, 0.0 );
   Containers::Vector< double, Devices::Cuda, int > ones( n, 1.0 );
   A->vectorProduct( ones, b );
   Solvers::Linear::CG< M > cg;
   cg.setMatrix( A );
   cg.setConvergenceResidue( 1e-10 );
   EXPECT( cg.solve( b, xx ), "symmetric CG" );
   double e2 = 0;
   for( double v : xx.toStdVector() )
      e2 = std::max( e2, std::fabs( v - 1.0 ) );
   EXPECT( e2 < 1e-7, "symmetric CG error %g", e2 );
   std::printf( "SymmetricMatrix (%s): product error %.3e, CG %d iterations, error %.3e\n", label, err,
                cg.getIterations(), e2 );
}

// MultidiagonalMatrix< double, Cuda, int >: a 2D Laplacian on its five
// diagonals (boundary slots left zero), the product against the host and a CG
// solve; elements off the diagonals are refused
static void
run_multidiagonal()
{
   using M = Matrices::MultidiagonalMatrix< double, Devices::Cuda, int >;
   const int nx = 30, n = nx * nx;
   auto A = std::make_shared< M >( n, n, std::initializer_list< int >{ 1, -nx, 0, nx, -1 } );
   EXPECT( A->getDiagonalsCount() == 5 && A->getDiagonalsOffsets()[ 0 ] == -nx, "diagonal offsets" );
   std::vector< double > xs( n ), want( n, 0.0 );
   for( int i = 0; i < n; i++ )
      xs[ i ] = std::cos( 0.05 * i );
   for( int j = 0; j < nx; j++ )
      for( int i = 0; i < nx; i++ ) {
         const int r = i + nx * j;
         A->setElement( r, r, 4.0 );
         want[ r ] += 4.0 * xs[ r ];
         const int nb[ 4 ] = { i > 0 ? r - 1 : -1, i < nx - 1 ? r + 1 : -1, j > 0 ? r - nx : -1, j < nx - 1 ? r + nx : -1 };
         for( int c : nb )
            if( c >= 0 ) {
               A->setElement( r, c, -1.0 );
               want[ r ] -= xs[ c ];
            }
      }
   EXPECT( A->getElement( 1, 0 ) == -1.0 && A->getElement( nx, nx - 1 ) == 0.0, "multidiagonal getElement" );
   bool threw = false;
   try {
      A->setElement( 0, 2, 1.0 );
   }
   catch( const std::logic_error& ) {
      threw = true;
   }
   EXPECT( threw, "an element off the diagonals was accepted" );
   Containers::Vector< double, Devices::Cuda, int > x( n ), y( n, 0.0 );
   for( int i = 0; i < n; i++ )
      x.setElement( i, xs[ i ] );
   A->vectorProduct( x, y );
   const auto h = y.toStdVector();
   double err = 0;
   for( int i = 0; i < n; i++ )
      err = std::max( err, std::fabs( h[ i ] - want[ i ] ) );
   EXPECT( err < 1e-12, "multidiagonal product error %g", err );
   Containers::Vector< double, Devices::Cuda, int > b( n ), xx( n, 0.0 ), ones( n, 1.0 );
   A->vectorProduct( ones, b );
   Solvers::Linear::CG< M > cg;
   cg.setMatrix( A );
   cg.setConvergenceResidue( 1e-10 );
   EXPECT( cg.solve( b, xx ), "multidiagonal CG" );
   double e2 = 0;
   for( double v : xx.toStdVector() )
      e2 = std::max( e2, std::fabs( v - 1.0 ) );
   EXPECT( e2 < 1e-7, "multidiagonal CG error %g", e2 );
   std::printf( "MultidiagonalMatrix: product error %.3e, CG %d iterations, error %.3e\n", err, cg.getIterations(), e2 );
}

int
main()
{
   run_products< double, Seg::CSRDefault >();
   run_products< double, Seg::CSRScalar >();
   run_products< double, Seg::CSRVector >();
   run_products< double, Seg::Ellpack >();
   run_products< double, Seg::SlicedEllpack >();
   run_products< double, Seg::ChunkedEllpack >();
   run_products< double, Seg::BiEllpack >();
   run_products< float, Seg::CSRDefault >();
   run_products< float, Seg::SlicedEllpack >();
   run_products< float, Seg::BiEllpack >();
   run_solver< Solvers::Linear::CG >( "CG", false, "MGSR" );
   run_solver< Solvers::Linear::BICGStab >( "BICGStab", true, "MGSR" );
   run_solver< Solvers::Linear::GMRES >( "GMRES(MGSR)", true, "MGSR" );
   run_solver< Solvers::Linear::GMRES >( "GMRES(CGSR)", true, "CGSR" );
   run_solver< Solvers::Linear::TFQMR >( "TFQMR", true, "MGSR" );
   run_solver< Solvers::Linear::BICGStabL >( "BICGStab(2)", true, "MGSR", 2 );
   run_solver< Solvers::Linear::BICGStabL >( "BICGStab(4)+ILU0", true, "MGSR", 4, true );
   run_solver< Solvers::Linear::TFQMR >( "TFQMR+ILU0", true, "MGSR", 1, true );
   run_solver< Solvers::Linear::BICGStab, Solvers::Linear::Preconditioners::ILUT >( "BICGStab+ILUT", true, "MGSR", 1,
                                                                                   true );
   run_solver< Solvers::Linear::Jacobi >( "Jacobi", true, "MGSR" );
   run_solver< Solvers::Linear::SOR >( "SOR", true, "MGSR" );
   run_multidiagonal();
   run_symmetric< Seg::CSRDefault >( "CSR" );
   run_symmetric< Seg::Ellpack >( "Ellpack" );
   run_symmetric< Seg::SlicedEllpack >( "SlicedEllpack" );
   run_symmetric< Seg::ChunkedEllpack >( "ChunkedEllpack" );
   run_symmetric< Seg::BiEllpack >( "BiEllpack" );
   {
      // setElement beyond the row capacity throws std::logic_error, as in TNL
      Matrices::SparseMatrix< double, Devices::Cuda, int > m( 2, 2 );
      m.setRowCapacities( { 1, 1 } );
      m.setElement( 0, 0, 1.0 );
      bool threw = false;
      try {
         m.setElement( 0, 1, 2.0 );
      }
      catch( const std::logic_error& ) {
         threw = true;
      }
      EXPECT( threw, "capacity overflow did not throw" );
   }
   {
      // MatrixReader::readMtx / MatrixWriter::writeMtx round trip (symmetric
      // file, a duplicate, an explicit zero, comments)
      const std::string dir = std::getenv( "TMPDIR" ) ? std::getenv( "TMPDIR" ) : "/tmp";
      const std::string in = dir + "/b2s_tnl_api_in.mtx", out = dir + "/b2s_tnl_api_out.mtx";
      {
         std::ofstream f( in );
         f << "%%MatrixMarket matrix coordinate real symmetric\n% test\n4 4 6\n1 1 4\n2 1 -1\n2 2 4\n"
              "3 2 -1\n3 3 0\n4 4 2\n4 4 4\n";
      }
      using E = Matrices::SparseMatrix< double, Devices::Cuda, int, Matrices::GeneralMatrix, Seg::Ellpack >;
      E a;
      Matrices::MatrixReader< E >::readMtx( in, a );
      EXPECT( a.getRows() == 4 && a.getColumns() == 4, "readMtx dimensions" );
      EXPECT( a.getElement( 0, 1 ) == -1.0 && a.getElement( 1, 0 ) == -1.0, "symmetric expansion" );
      EXPECT( a.getElement( 3, 3 ) == 4.0, "the last duplicate wins" );
      product_check( "readMtx", a, 1, { 3, 2, -1, 4 } );
      Matrices::MatrixWriter< E >::writeMtx( out, a );
      Matrices::SparseMatrix< double, Devices::Cuda, int > b;
      Matrices::MatrixReader< decltype( b ) >::readMtx( out, b );
      product_check( "writeMtx round trip", b, 1, { 3, 2, -1, 4 } );
      bool threw = false;
      try {
         Matrices::MatrixReader< E >::readMtx( dir + "/b2s_tnl_api_absent.mtx", a );
      }
      catch( const std::runtime_error& ) {
         threw = true;
      }
      EXPECT( threw, "a missing file did not throw" );
      // SparseMatrix::save / load: TNL's binary file
      const std::string bin = dir + "/b2s_tnl_api.tnl";
      a.save( bin );
      E c;
      c.load( bin );
      EXPECT( c.getRows() == 4 && c.getElement( 3, 3 ) == 4.0, "load" );
      product_check( "save/load round trip", c, 1, { 3, 2, -1, 4 } );
   }
   // binary matrices: SparseMatrix< bool, ... > (Matrices/SparseMatrix.h:23-26); the
   // product computes in Index, so x = 2.9 counts 2 per stored element
   {
      const std::vector< std::vector< std::pair< int, double > > > e = {
         { { 0, 1 }, { 2, 1 } }, { { 1, 1 } }, {}, { { 0, 1 }, { 1, 1 }, { 2, 1 }, { 3, 1 } } };
      Matrices::SparseMatrix< bool, Devices::Cuda, int, Matrices::GeneralMatrix, Seg::CSRDefault > bc;
      Matrices::SparseMatrix< bool, Devices::Cuda, int, Matrices::GeneralMatrix, Seg::SlicedEllpack > bs;
      Matrices::SparseMatrix< bool, Devices::Cuda, int, Matrices::GeneralMatrix, Seg::BiEllpack > bb;
      auto check_binary = [ & ]( auto& m, const char* name )
      {
         assemble( m, 4, 4, e, 1 );
         EXPECT( m.getNonzeroElementsCount() == 7, "%s nonzeros %d", name, (int) m.getNonzeroElementsCount() );
         Containers::Vector< double, Devices::Cuda, int > in( 4, 2.9 ), out( 4, 1.0 );
         m.vectorProduct( in, out );
         const auto y = out.toStdVector();
         const double want[] = { 4, 2, 0, 8 };
         for( int i = 0; i < 4; i++ )
            EXPECT( y[ i ] == want[ i ], "%s row %d: %g != %g", name, i, y[ i ], want[ i ] );
         Containers::Vector< float, Devices::Cuda, int > fin( 4, -1.5f ), fout( 4, 1.0f );
         m.vectorProduct( fin, fout, 3, 2 );  // 2 * y + 3 * sum of (int) -1.5 = 2 - 3 * count
         const auto fy = fout.toStdVector();
         const float fwant[] = { -4, -1, 2, -10 };
         for( int i = 0; i < 4; i++ )
            EXPECT( fy[ i ] == fwant[ i ], "%s float row %d: %g != %g", name, i, (double) fy[ i ], (double) fwant[ i ] );
      };
      check_binary( bc, "binary CSR" );
      check_binary( bs, "binary SlicedEllpack" );
      check_binary( bb, "binary BiEllpack" );
   }
   std::printf( "%s (%d failures)\n", failures ? "FAILED" : "PASSED", failures );
   return failures ? 1 : 0;
}
