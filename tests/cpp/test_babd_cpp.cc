// C++ drop-in check of the dispatch wrapper alglin::BABD<double> (cyclic
// reduction branch): the system of src_tests/test7-BorderedCR.cc built
// through babd.cr(), solved with each CR choice (LU, QR, QRP panels) through
// factorize_system / solve_system, checked against the manufactured solution;
// the sparse pattern forwards; DIAZ is refused with an exception.
#define ALGLIN_B200_AS_ALGLIN
#include "alglin_b200/BABD.hh"

#include <cmath>
#include <cstdio>
#include <random>
#include <vector>

static std::mt19937 gen( 3 );
static double rnd( double a, double b ) { return a + ( b - a ) * double( gen() ) / double( gen.max() ); }

int main( int argc, char ** argv ) {
  using Choice = alglin::BABD<double>::BABD_Choice;
  int nblock = argc > 1 ? std::atoi( argv[1] ) : 2000;
  int const n = 8, qx = 2, qr = 2, nx = 1, nr = 1;
  alglin::BABD<double> babd( Choice::CYCLIC_REDUCTION_LU, 4 );
  alglin::BorderedCR<double> & CR = babd.cr();
  CR.allocate( nblock, n, qr, qx, nr, nx );
  CR.fill_zero();
  double const diag = 1.01 * n;
  for ( int i = 0; i < n + qr; ++i ) {
    for ( int j = 0; j < 2 * n + qx + nx; ++j ) CR.H( i, j ) = rnd( -1, 0 );
    CR.H( i, i + n ) += diag;
  }
  for ( int k = 0; k < nblock; ++k ) {
    for ( int i = 0; i < n; ++i ) {
      for ( int j = 0; j < n; ++j ) { CR.D( k, i, j ) = rnd( -1, 0 ); CR.E( k, i, j ) = rnd( -1, 0 ); }
      CR.D( k, i, i ) += diag;
    }
    for ( int i = 0; i < n; ++i ) {
      for ( int j = 0; j < nx; ++j ) CR.B( k, i, j ) = rnd( -0.1, 0.1 );
      for ( int j = 0; j < nr; ++j ) CR.C( k, j, i ) = rnd( -0.1, 0.1 );
    }
  }
  for ( int i = 0; i < nr; ++i ) {
    for ( int j = 0; j < nx; ++j ) CR.F( i, j ) = rnd( -0.1, 0.1 );
    for ( int j = 0; j < qx; ++j ) CR.Cq( i, j ) = rnd( -0.1, 0.1 );
    CR.F( i, i ) += diag;
  }
  for ( int i = 0; i < n; ++i )
    for ( int j = 0; j < nr; ++j ) CR.C( nblock, j, i ) = 1;

  int const N = babd.ncols();
  if ( babd.nrows() != N ) { std::printf( "not square\n" ); return 1; }
  std::vector<double> x( N ), xref( N ), rhs( N );
  for ( int i = 0; i < N; ++i ) xref[i] = 1 + ( i % 100 );
  CR.Mv( xref.data(), rhs.data() );

  for ( Choice c : { Choice::CYCLIC_REDUCTION_LU, Choice::CYCLIC_REDUCTION_QR, Choice::CYCLIC_REDUCTION_QRP } ) {
    babd.selectSolver( c );
    if ( babd.selected_solver() != c || babd.using_diaz() || !babd.using_cyclic_reduction() ) return 1;
    if ( !babd.factorize_system() ) {
      std::printf( "%s: factorize failed: %s\n", alglin::BABD<double>::Choice_to_string( c ).c_str(),
                   std::string( CR.last_error() ).c_str() );
      return 1;
    }
    x = rhs;
    if ( !babd.solve_system( x.data() ) ) { std::printf( "solve failed\n" ); return 1; }
    double err = 0;
    for ( int i = 0; i < N; ++i ) err = std::max( err, std::abs( x[i] - xref[i] ) );
    std::printf( "%s: %s, max error %.3e\n", alglin::BABD<double>::Choice_to_string( c ).c_str(),
                 babd.info().c_str(), err );
    if ( !( err < 1e-8 ) ) return 1;
  }
  int const nnz = babd.sparse_nnz();
  std::vector<int> I( nnz ), J( nnz );
  std::vector<double> V( nnz );
  babd.sparse_pattern( I.data(), J.data() );
  babd.sparse_values( V.data() );
  // the sparse matrix times xref is the right-hand side
  std::vector<double> y( N, 0.0 );
  for ( int e = 0; e < nnz; ++e ) y[I[e]] += V[e] * xref[J[e]];
  double serr = 0;
  for ( int i = 0; i < N; ++i ) serr = std::max( serr, std::abs( y[i] - rhs[i] ) );
  if ( !( serr < 1e-9 ) ) { std::printf( "sparse product error %g\n", serr ); return 1; }
  try {
    babd.selectSolver( Choice::DIAZ );
    std::printf( "DIAZ accepted\n" );
    return 1;
  } catch ( std::runtime_error const & e ) {
    std::printf( "DIAZ refused: %s", e.what() );
  }
  std::printf( "BABD drop-in ok\n" );
  return 0;
}
