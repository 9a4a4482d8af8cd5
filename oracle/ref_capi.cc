// C entry points around the reference alglin::BorderedCR<double>, compiled
// from the unmodified reference sources through the shim in oracle/shim.
// TEST INFRASTRUCTURE ONLY: used by the tests to pin the C oracle and by the
// benchmark's CPU-baseline / reference arm.  Never linked into the product.
#include "shim/Alglin.hh"

#include <chrono>
#include <cstring>
#include <memory>
#include <string>
#include <vector>
#include <algorithm>

namespace {
  struct RefHandle {
    std::unique_ptr<Utils::ThreadPool1>          tp;
    std::unique_ptr<alglin::BorderedCR<double>>  bcr;
    std::string                                  err;
    std::string                                  info;
  };
  int fail( RefHandle * h, std::exception const & e ) { h->err = e.what(); return 0; }
}

extern "C" {

void * ref_create( int nthreads, int npb ) {
  auto * h = new RefHandle;
  if ( nthreads > 0 ) {
    h->tp.reset( new Utils::ThreadPool1( unsigned(nthreads) ) );
    h->bcr.reset( new alglin::BorderedCR<double>( h->tp.get(), npb ) );
  } else {
    h->bcr.reset( new alglin::BorderedCR<double>( nullptr ) );
  }
  return h;
}

void ref_destroy( void * p ) { delete static_cast<RefHandle*>(p); }

int ref_allocate( void * p, int nblock, int n, int qr, int qx, int nr, int nx ) {
  auto * h = static_cast<RefHandle*>(p);
  try { h->bcr->allocate( nblock, n, qr, qx, nr, nx ); } catch ( std::exception const & e ) { return fail( h, e ); }
  return 1;
}

// whole-matrix load through the public block loaders (reference layout arrays)
int ref_load( void * p, double const * D, double const * E, double const * B, double const * C,
              double const * Cq, double const * F, double const * H ) {
  auto * h = static_cast<RefHandle*>(p);
  auto & b = *h->bcr;
  int const nb = b.number_of_blocks(), n = b.block_size(), nr = b.dim_nr(), nx = b.dim_nx();
  try {
    b.fill_zero();
    for ( int k = 0; k < nb; ++k ) {
      b.load_D( k, D + size_t(k)*n*n, n );
      b.load_E( k, E + size_t(k)*n*n, n );
      if ( nx > 0 ) b.load_B( k, B + size_t(k)*n*nx, n );
    }
    if ( nr > 0 ) {
      for ( int k = 0; k <= nb; ++k ) b.load_C( k, C + size_t(k)*nr*n, nr );
      b.load_Cq( Cq, nr );
      b.load_F( F, nr );
    }
    b.load_bottom( H, n + b.dim_qr() );
  } catch ( std::exception const & e ) { return fail( h, e ); }
  return 1;
}

int ref_select( void * p, char const * internal, char const * last, char const * last2 ) {
  auto * h = static_cast<RefHandle*>(p);
  try {
    h->bcr->select( internal );
    h->bcr->select_last( last );
    h->bcr->select_last2( last2 );
  } catch ( std::exception const & e ) { return fail( h, e ); }
  return 1;
}

void ref_set_threads( void * p, int fact, int solve ) {
  auto * h = static_cast<RefHandle*>(p);
  h->bcr->set_factorize_use_thread( fact != 0 );
  h->bcr->set_solve_use_thread( solve != 0 );
}

void ref_set_num_parallel_block( void * p, int npb ) {
  static_cast<RefHandle*>(p)->bcr->set_num_parallel_block( npb );
}

int ref_factorize( void * p ) {
  auto * h = static_cast<RefHandle*>(p);
  try { return h->bcr->factorize() ? 1 : 0; } catch ( std::exception const & e ) { return fail( h, e ); }
}

int ref_solve( void * p, double * x ) {
  auto * h = static_cast<RefHandle*>(p);
  try { return h->bcr->solve( x ) ? 1 : 0; } catch ( std::exception const & e ) { return fail( h, e ); }
}

int ref_solve_n( void * p, int nrhs, double * x, int ld ) {
  auto * h = static_cast<RefHandle*>(p);
  try { return h->bcr->solve( nrhs, x, ld ) ? 1 : 0; } catch ( std::exception const & e ) { return fail( h, e ); }
}

void ref_mv( void * p, double const * x, double * res ) { static_cast<RefHandle*>(p)->bcr->Mv( x, res ); }

int ref_dup( void * dst, void * src ) {
  auto * d = static_cast<RefHandle*>(dst);
  auto * s = static_cast<RefHandle*>(src);
  try { d->bcr->dup( *s->bcr ); } catch ( std::exception const & e ) { return fail( d, e ); }
  return 1;
}

char const * ref_last_error( void * p ) {
  auto * h = static_cast<RefHandle*>(p);
  h->err = std::string( h->bcr->last_error() ) + h->err;
  return h->err.c_str();
}

char const * ref_info( void * p ) {
  auto * h = static_cast<RefHandle*>(p);
  h->info = h->bcr->info();
  return h->info.c_str();
}

int ref_nrows( void * p ) { return static_cast<RefHandle*>(p)->bcr->nrows(); }
int ref_ncols( void * p ) { return static_cast<RefHandle*>(p)->bcr->ncols(); }

// factorize a fresh copy of `src` (dup excluded from the clock) and solve
// nrhs right-hand sides in place; returns wall seconds of factorize+solve
double ref_time_factor_solve( void * work, void * src, int nrhs, double * x, int ld, int * ok ) {
  auto * w = static_cast<RefHandle*>(work);
  auto * s = static_cast<RefHandle*>(src);
  *ok = 0;
  try {
    // dup() resets the thread pool pointer to the inline one (cc:197); keep the
    // caller's pool by copying values through the public accessors instead
    auto & a = *w->bcr; auto const & b = *s->bcr;
    int const nb = b.number_of_blocks(), n = b.block_size(), nr = b.dim_nr(), nx = b.dim_nx(), qr = b.dim_qr(), qx = b.dim_qx();
    std::memcpy( &a.D(0,0,0), &b.D(0,0,0), sizeof(double)*size_t(nb)*n*n );
    std::memcpy( &a.E(0,0,0), &b.E(0,0,0), sizeof(double)*size_t(nb)*n*n );
    if ( nx > 0 ) std::memcpy( &a.B(0,0,0), &b.B(0,0,0), sizeof(double)*size_t(nb)*n*nx );
    if ( nr > 0 ) {
      std::memcpy( &a.C(0,0,0), &b.C(0,0,0), sizeof(double)*size_t(nb+1)*nr*n );
      if ( qx > 0 ) std::memcpy( &a.Cq(0,0), &b.Cq(0,0), sizeof(double)*size_t(nr)*qx );
      if ( nx > 0 ) std::memcpy( &a.F(0,0), &b.F(0,0), sizeof(double)*size_t(nr)*nx );
    }
    std::memcpy( &a.H(0,0), &b.H(0,0), sizeof(double)*size_t(n+qr)*(2*n+qx+nx) );
    auto t0 = std::chrono::steady_clock::now();
    bool good = a.factorize();
    if ( good ) good = nrhs == 1 ? a.solve( x ) : a.solve( nrhs, x, ld );
    auto t1 = std::chrono::steady_clock::now();
    *ok = good ? 1 : 0;
    return std::chrono::duration<double>( t1 - t0 ).count();
  } catch ( std::exception const & e ) { fail( w, e ); return -1; }
}

// sparse export of the loaded matrix (hxx:1079-1097, cc:2316-2413)
int ref_sparse_nnz( void * p ) { return static_cast<RefHandle*>(p)->bcr->sparse_nnz(); }
int ref_sparse_pattern( void * p, int * I, int * J, int offs ) {
  auto * h = static_cast<RefHandle*>(p);
  try { h->bcr->sparse_pattern( I, J, offs ); } catch ( std::exception const & e ) { return fail( h, e ); }
  return 1;
}
int ref_sparse_values( void * p, double * V ) {
  auto * h = static_cast<RefHandle*>(p);
  try { h->bcr->sparse_values( V ); } catch ( std::exception const & e ) { return fail( h, e ); }
  return 1;
}

// The reference's BorderedCR<float> (explicitly instantiated at cc:2663) on
// the same system, loaded through its public loaders after rounding every
// entry to float: an unrefined FP32 factorize + solve, timed like
// ref_time_factor_solve (load excluded).  x (double, length >= max(nrows,
// ncols)) holds the right-hand side on entry and the solution on return.
double ref_f32_factor_solve( int nthreads, int npb, int nblock, int n, int qr, int qx, int nr, int nx,
                             double const * D, double const * E, double const * B, double const * C,
                             double const * Cq, double const * F, double const * H, double * x, int * ok ) {
  *ok = 0;
  try {
    std::unique_ptr<Utils::ThreadPool1> tp;
    std::unique_ptr<alglin::BorderedCR<float>> bcr;
    if ( nthreads > 0 ) {
      tp.reset( new Utils::ThreadPool1( unsigned(nthreads) ) );
      bcr.reset( new alglin::BorderedCR<float>( tp.get(), npb ) );
    } else {
      bcr.reset( new alglin::BorderedCR<float>( nullptr ) );
    }
    auto & b = *bcr;
    b.allocate( nblock, n, qr, qx, nr, nx );
    b.fill_zero();
    b.set_factorize_use_thread( nthreads > 0 );
    b.set_solve_use_thread( nthreads > 0 );
    b.select_LU();
    b.select_last_LU();
    auto cvt = []( double const * a, size_t len ) { return std::vector<float>( a, a + len ); };
    for ( int k = 0; k < nblock; ++k ) {
      b.load_D( k, cvt( D + size_t(k)*n*n, size_t(n)*n ).data(), n );
      b.load_E( k, cvt( E + size_t(k)*n*n, size_t(n)*n ).data(), n );
      if ( nx > 0 ) b.load_B( k, cvt( B + size_t(k)*n*nx, size_t(n)*nx ).data(), n );
    }
    if ( nr > 0 ) {
      for ( int k = 0; k <= nblock; ++k ) b.load_C( k, cvt( C + size_t(k)*nr*n, size_t(nr)*n ).data(), nr );
      if ( qx > 0 ) b.load_Cq( cvt( Cq, size_t(nr)*qx ).data(), nr );
      if ( nx > 0 ) b.load_F( cvt( F, size_t(nr)*nx ).data(), nr );
    }
    b.load_bottom( cvt( H, size_t(n+qr)*(2*n+qx+nx) ).data(), n + qr );
    size_t const L = size_t( std::max( b.nrows(), b.ncols() ) );
    std::vector<float> xf( x, x + L );
    auto t0 = std::chrono::steady_clock::now();
    bool good = b.factorize();
    if ( good ) good = b.solve( xf.data() );
    auto t1 = std::chrono::steady_clock::now();
    for ( size_t i = 0; i < L; ++i ) x[i] = double( xf[i] );
    *ok = good ? 1 : 0;
    return std::chrono::duration<double>( t1 - t0 ).count();
  } catch ( std::exception const & ) { return -1; }
}

} // extern "C"
