// C++ drop-in check: the checks of the reference's src_tests/test7-BorderedCR.cc
// (manufactured solution x_i = 1 + (i % 100) on a diagonally dominant system,
// single and two right-hand sides, residual) written against
// alglin::BorderedCR<double> and compiled with ALGLIN_B200_AS_ALGLIN, so the
// reference-style code runs on the GPU path unchanged.
#define ALGLIN_B200_AS_ALGLIN
#include "alglin_b200/BorderedCR.hh"

#include <cmath>
#include <cstdio>
#include <random>
#include <vector>

static std::mt19937 gen( 2 );
static double rnd( double a, double b ) { return a + ( b - a ) * double( gen() ) / double( gen.max() ); }

int main( int argc, char ** argv ) {
  int nblock = argc > 1 ? std::atoi( argv[1] ) : 10000;
  int const n = 8, qx = 4, qr = 4, nx = 1, nr = 1;
  // the reference's own construction (test7-BorderedCR.cc:114-116)
  Utils::ThreadPool1         TP( 4 );
  alglin::BorderedCR<double> BCR( &TP );
  alglin::BorderedCR<double> SAVED( &TP );
  BCR.allocate( nblock, n, qr, qx, nr, nx );
  BCR.fill_zero();
  double const diag = 1.01 * n;
  for ( int i = 0; i < n + qr; ++i ) {
    for ( int j = 0; j < 2 * n + qx + nx; ++j ) BCR.H( i, j ) = rnd( -1, 0 );
    BCR.H( i, i + n ) += diag;
  }
  for ( int k = 0; k < nblock; ++k ) {
    for ( int i = 0; i < n; ++i ) {
      for ( int j = 0; j < n; ++j ) { BCR.D( k, i, j ) = rnd( -1, 0 ); BCR.E( k, i, j ) = rnd( -1, 0 ); }
      BCR.D( k, i, i ) += diag;
    }
    for ( int i = 0; i < n; ++i ) {
      for ( int j = 0; j < nx; ++j ) BCR.B( k, i, j ) = rnd( -0.1, 0.1 );
      for ( int j = 0; j < nr; ++j ) BCR.C( k, j, i ) = rnd( -0.1, 0.1 );
    }
  }
  for ( int i = 0; i < nr; ++i ) {
    for ( int j = 0; j < nx; ++j ) BCR.F( i, j ) = rnd( -0.1, 0.1 );
    for ( int j = 0; j < qx; ++j ) BCR.Cq( i, j ) = rnd( -0.1, 0.1 );
    BCR.F( i, i ) += diag;
  }
  for ( int i = 0; i < n; ++i )
    for ( int j = 0; j < nr; ++j ) BCR.C( nblock, j, i ) = 1;

  int const N = BCR.ncols();
  std::vector<double> x( 2 * N ), xref( N ), rhs( 2 * N ), resid( N );
  for ( int i = 0; i < N; ++i ) xref[i] = x[i] = 1 + ( i % 100 );
  BCR.Mv( x.data(), rhs.data() );
  SAVED.dup( BCR );
  BCR.select_LU();
  BCR.select_last_LU();
  if ( !BCR.factorize() ) { std::printf( "factorize failed: %s\n", std::string( BCR.last_error() ).c_str() ); return 1; }
  x = rhs;
  if ( !BCR.solve( x.data() ) ) { std::printf( "solve failed\n" ); return 1; }
  double err = 0;
  for ( int i = 0; i < N; ++i ) err = std::max( err, std::abs( x[i] - xref[i] ) );
  if ( !( err < 1e-8 ) ) { std::printf( "single rhs error %g\n", err ); return 1; }
  std::copy( rhs.begin(), rhs.begin() + N, x.begin() );
  std::copy( rhs.begin(), rhs.begin() + N, x.begin() + N );
  if ( !BCR.solve( 2, x.data(), N ) ) { std::printf( "solve(2) failed\n" ); return 1; }
  for ( int c = 0; c < 2; ++c )
    for ( int i = 0; i < N; ++i ) err = std::max( err, std::abs( x[c * N + i] - xref[i] ) );
  if ( !( err < 1e-8 ) ) { std::printf( "two rhs error %g\n", err ); return 1; }
  // the same through the LinearSystemSolver base and its MatrixWrapper form
  std::copy( rhs.begin(), rhs.begin() + N, x.begin() );
  std::copy( rhs.begin(), rhs.begin() + N, x.begin() + N );
  alglin::LinearSystemSolver<double> & base = BCR;
  alglin::MatrixWrapper<double> XW( x.data(), N, 2, N );
  if ( !base.solve( XW ) ) { std::printf( "solve(MatW) failed\n" ); return 1; }
  for ( int c = 0; c < 2; ++c )
    for ( int i = 0; i < N; ++i ) err = std::max( err, std::abs( x[c * N + i] - xref[i] ) );
  if ( !( err < 1e-8 ) ) { std::printf( "solve(MatW) error %g\n", err ); return 1; }
  std::copy( rhs.begin(), rhs.begin() + N, x.begin() );
  BCR.solve( x.data() );
  for ( int i = 0; i < N; ++i ) resid[i] = -rhs[i];
  SAVED.add_Mv( x.data(), resid.data() );
  double r2 = 0;
  for ( double v : resid ) r2 += v * v;
  if ( !( std::sqrt( r2 ) < 1e-6 ) ) { std::printf( "residual %g\n", std::sqrt( r2 ) ); return 1; }
  std::printf( "%s", BCR.info().c_str() );
  if ( BCR.info().find( "treads = 4/nblk:4/" ) == std::string::npos ) {
    std::printf( "info() does not show the pool's 4 threads\n" ); return 1;
  }
  std::printf( "C++ drop-in ok: max error %.3e, residual %.3e\n", err, std::sqrt( r2 ) );
  return 0;
}
