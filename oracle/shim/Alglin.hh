// Oracle build shim: stands in for the reference's umbrella header so that the
// unmodified reference files src/BABD_BorderedCR.cc and src/Alglin_Eigen.cc
// compile without the absent LapackWrapper / UtilsLite submodules.
//
// Test infrastructure only.  It provides, in our own code, the small subset of
// those submodules' interfaces that the BorderedCR path calls (the call sites
// are BABD_BorderedCR.cc:845-1044, 1281-1479 and BABD_BorderedCR.hxx:104-228):
//   Utils      : Runtime_Error, UTILS_ASSERT/ERROR macros, spin lock, Malloc,
//                ThreadPoolBase / ThreadPool0 (inline) / ThreadPool1 (threads)
//   lapack     : getrf geqrf geqp3 ormqr swaps trsm trsv gemm gemv swap
//                (unblocked restatements of the published LAPACK algorithms)
//   last block : LU LUPQ QR QRP SVD LSS LSY PINV classes
// and then includes the reference header Alglin/BABD_BorderedCR.hxx.
#pragma once
#ifndef ORACLE_SHIM_ALGLIN_HH
#define ORACLE_SHIM_ALGLIN_HH

#ifndef FMT_HEADER_ONLY
#define FMT_HEADER_ONLY 1
#endif
#include <fmt/format.h>
#include <fmt/ostream.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <functional>
#include <limits>
#include <iostream>
#include <map>
#include <mutex>
#include <stdexcept>
#include <string>
#include <string_view>
#include <thread>
#include <vector>

namespace Utils {

  class Runtime_Error : public std::runtime_error {
  public:
    explicit Runtime_Error( std::string const & m ) : std::runtime_error(m) {}
    Runtime_Error( std::string const & m, char const * file, int line )
    : std::runtime_error( fmt::format( "{}\nin file: {} line: {}\n", m, file, line ) ) {}
  };

  template <typename T> inline bool is_finite( T x ) { return std::isfinite(x); }

  class SpinLock {
    std::atomic_flag m_flag = ATOMIC_FLAG_INIT;
  public:
    void lock()   { while ( m_flag.test_and_set( std::memory_order_acquire ) ) {} }
    void unlock() { m_flag.clear( std::memory_order_release ); }
  };

  // bump allocator with the interface the reference uses (reallocate, (n),
  // must_be_empty, realloc, malloc, allocate)
  template <typename T>
  class Malloc {
    std::string    m_name;
    std::vector<T> m_buf;
    size_t         m_used{0};
  public:
    explicit Malloc( std::string const & name ) : m_name(name) {}
    void allocate( size_t n )   { if ( m_buf.size() < n ) m_buf.assign( n, T(0) ); m_used = 0; }
    void reallocate( size_t n ) { m_buf.assign( n, T(0) ); m_used = 0; }
    T * operator () ( size_t n ) {
      if ( m_used + n > m_buf.size() )
        throw Runtime_Error( fmt::format( "Malloc<{}>: out of arena", m_name ) );
      T * p = m_buf.data() + m_used; m_used += n; return p;
    }
    T * malloc( size_t n )  { allocate( n ); return (*this)( n ); }
    T * realloc( size_t n ) { allocate( n ); return (*this)( n ); }
    void must_be_empty( char const * where ) const {
      if ( m_used != m_buf.size() )
        throw Runtime_Error( fmt::format( "{}: arena not fully used ({} of {})", where, m_used, m_buf.size() ) );
    }
  };

  class ThreadPoolBase {
  public:
    virtual ~ThreadPoolBase() = default;
    virtual unsigned thread_count() const = 0;
    virtual void exec( std::function<void()> && f ) = 0;
    virtual void wait() = 0;
    template <typename Func, typename... Args>
    void run( Func && func, Args && ... args ) {
      exec( std::bind( std::forward<Func>(func), std::forward<Args>(args)... ) );
    }
  };

  // runs every task inline on the calling thread
  class ThreadPool0 : public ThreadPoolBase {
  public:
    explicit ThreadPool0( unsigned ) {}
    unsigned thread_count() const override { return 1; }
    void exec( std::function<void()> && f ) override { f(); }
    void wait() override {}
  };

  // fixed pool of worker threads with a shared FIFO queue
  class ThreadPool1 : public ThreadPoolBase {
    std::vector<std::thread>          m_workers;
    std::deque<std::function<void()>> m_queue;
    std::mutex                        m_mtx;
    std::condition_variable           m_cv, m_done;
    unsigned                          m_busy{0};
    bool                              m_stop{false};
  public:
    explicit ThreadPool1( unsigned n ) {
      if ( n < 1 ) n = 1;
      for ( unsigned i = 0; i < n; ++i )
        m_workers.emplace_back( [this]() {
          for (;;) {
            std::function<void()> task;
            {
              std::unique_lock<std::mutex> lk( m_mtx );
              m_cv.wait( lk, [this]{ return m_stop || !m_queue.empty(); } );
              if ( m_stop && m_queue.empty() ) return;
              task = std::move( m_queue.front() ); m_queue.pop_front(); ++m_busy;
            }
            task();
            {
              std::lock_guard<std::mutex> lk( m_mtx );
              --m_busy;
              if ( m_busy == 0 && m_queue.empty() ) m_done.notify_all();
            }
          }
        } );
    }
    ~ThreadPool1() override {
      { std::lock_guard<std::mutex> lk( m_mtx ); m_stop = true; }
      m_cv.notify_all();
      for ( auto & t : m_workers ) t.join();
    }
    unsigned thread_count() const override { return unsigned(m_workers.size()); }
    void exec( std::function<void()> && f ) override {
      { std::lock_guard<std::mutex> lk( m_mtx ); m_queue.emplace_back( std::move(f) ); }
      m_cv.notify_one();
    }
    void wait() override {
      std::unique_lock<std::mutex> lk( m_mtx );
      m_done.wait( lk, [this]{ return m_busy == 0 && m_queue.empty(); } );
    }
  };

} // namespace Utils

#define UTILS_SPINLOCK Utils::SpinLock
#define UTILS_ERROR(...)  throw Utils::Runtime_Error( fmt::format(__VA_ARGS__), __FILE__, __LINE__ )
#define UTILS_ERROR0(MSG) throw Utils::Runtime_Error( MSG, __FILE__, __LINE__ )
#define UTILS_ASSERT(COND, ...)  do { if ( !(COND) ) UTILS_ERROR(__VA_ARGS__); } while (0)
#define UTILS_ASSERT0(COND, MSG) do { if ( !(COND) ) UTILS_ERROR0(MSG); } while (0)

namespace lapack_wrapper {

  using integer      = int;
  using doublereal   = double;
  using ostream_type = std::ostream;

  enum class Transposition { NO = 0, YES, CONJUGATE };
  enum class ULselect      { UPPER = 0, LOWER };
  enum class SideMultiply  { LEFT = 0, RIGHT };
  enum class DiagonalType  { UNIT = 0, NON_UNIT };

  template <typename T>
  class MatrixWrapper {
  protected:
    T * m_data{nullptr};
    integer m_nr{0}, m_nc{0}, m_ld{0};
  public:
    MatrixWrapper() = default;
    MatrixWrapper( T * d, integer nr, integer nc, integer ld ) : m_data(d), m_nr(nr), m_nc(nc), m_ld(ld) {}
    void setup( T * d, integer nr, integer nc, integer ld ) { m_data = d; m_nr = nr; m_nc = nc; m_ld = ld; }
    integer nrows() const { return m_nr; }
    integer ncols() const { return m_nc; }
    integer ldim()  const { return m_ld; }
    T *       data()       { return m_data; }
    T const * data() const { return m_data; }
    T &       operator () ( integer i, integer j )       { return m_data[i + j * m_ld]; }
    T const & operator () ( integer i, integer j ) const { return m_data[i + j * m_ld]; }
  };

  template <typename T>
  class Matrix : public MatrixWrapper<T> {
    std::vector<T> m_buf;
  public:
    Matrix( integer nr, integer nc ) : m_buf( size_t(nr) * size_t(nc), T(0) ) {
      this->setup( m_buf.data(), nr, nc, nr );
    }
    void fill( T v ) { std::fill( m_buf.begin(), m_buf.end(), v ); }
  };

  template <typename T>
  class LinearSystemSolver {
  public:
    virtual ~LinearSystemSolver() = default;
    virtual bool solve( T [] ) const = 0;
    virtual bool solve( integer, T [], integer ) const = 0;
    virtual bool t_solve( T [] ) const = 0;
    virtual bool t_solve( integer, T [], integer ) const = 0;
    bool solve( MatrixWrapper<T> & M ) const { return this->solve( M.ncols(), M.data(), M.ldim() ); }
    bool t_solve( MatrixWrapper<T> & M ) const { return this->t_solve( M.ncols(), M.data(), M.ldim() ); }
    void factorize( char const * ) {}
  };

  // scalars (passed as double literals for the float instantiation) and the
  // nullptr matrices of workspace queries must not take part in deducing T
  template <typename T> struct nodeduce { using type = T; };
  template <typename T> using nd = typename nodeduce<T>::type;

  // ---------------------------------------------------------------- BLAS ---
  template <typename T>
  inline void
  swap( integer N, T * x, integer incx, T * y, integer incy ) {
    for ( integer i = 0; i < N; ++i ) std::swap( x[i*incx], y[i*incy] );
  }

  // y = alpha*op(A)*x + beta*y
  template <typename T>
  inline void
  gemv( Transposition TR, integer M, integer N, nd<T> alpha, T const * A, integer lda,
        T const * x, integer incx, nd<T> beta, T * y, integer incy ) {
    integer ny = TR == Transposition::NO ? M : N;
    for ( integer i = 0; i < ny; ++i ) y[i*incy] = beta == T(0) ? T(0) : beta * y[i*incy];
    if ( TR == Transposition::NO ) {
      for ( integer j = 0; j < N; ++j ) {
        T t = alpha * x[j*incx];
        for ( integer i = 0; i < M; ++i ) y[i*incy] += A[i + j*lda] * t;
      }
    } else {
      for ( integer j = 0; j < N; ++j ) {
        T s = 0;
        for ( integer i = 0; i < M; ++i ) s += A[i + j*lda] * x[i*incx];
        y[j*incy] += alpha * s;
      }
    }
  }

  // C = alpha*op(A)*op(B) + beta*C (NO/NO and the transposed forms)
  template <typename T>
  inline void
  gemm( Transposition TA, Transposition TB, integer M, integer N, integer K,
        nd<T> alpha, T const * A, integer lda, T const * B, integer ldb,
        nd<T> beta, T * C, integer ldc ) {
    for ( integer j = 0; j < N; ++j ) {
      for ( integer i = 0; i < M; ++i ) C[i + j*ldc] = beta == T(0) ? T(0) : beta * C[i + j*ldc];
      for ( integer l = 0; l < K; ++l ) {
        T b = TB == Transposition::NO ? B[l + j*ldb] : B[j + l*ldb];
        b *= alpha;
        if ( b == T(0) ) continue;
        for ( integer i = 0; i < M; ++i ) {
          T a = TA == Transposition::NO ? A[i + l*lda] : A[l + i*lda];
          C[i + j*ldc] += a * b;
        }
      }
    }
  }

  // triangular solve with a matrix right-hand side (LEFT/RIGHT, UPPER/LOWER, NO)
  template <typename T>
  inline void
  trsm( SideMultiply SIDE, ULselect UPLO, Transposition, DiagonalType DIAG,
        integer M, integer N, nd<T> alpha, T const * A, integer lda, T * B, integer ldb ) {
    bool unit = DIAG == DiagonalType::UNIT;
    for ( integer j = 0; j < N; ++j )
      for ( integer i = 0; i < M; ++i ) B[i + j*ldb] *= alpha;
    if ( SIDE == SideMultiply::LEFT ) {
      for ( integer c = 0; c < N; ++c ) {
        T * b = B + c*ldb;
        if ( UPLO == ULselect::LOWER ) {
          for ( integer i = 0; i < M; ++i ) {
            if ( !unit ) b[i] /= A[i + i*lda];
            for ( integer r = i+1; r < M; ++r ) b[r] -= A[r + i*lda] * b[i];
          }
        } else {
          for ( integer i = M-1; i >= 0; --i ) {
            if ( !unit ) b[i] /= A[i + i*lda];
            for ( integer r = 0; r < i; ++r ) b[r] -= A[r + i*lda] * b[i];
          }
        }
      }
    } else { // RIGHT: B <- B * op(A)^{-1}, A is N x N
      if ( UPLO == ULselect::UPPER ) {
        for ( integer i = 0; i < N; ++i ) {
          for ( integer m = 0; m < i; ++m ) {
            T a = A[m + i*lda];
            for ( integer r = 0; r < M; ++r ) B[r + i*ldb] -= B[r + m*ldb] * a;
          }
          if ( !unit ) for ( integer r = 0; r < M; ++r ) B[r + i*ldb] /= A[i + i*lda];
        }
      } else {
        for ( integer i = N-1; i >= 0; --i ) {
          for ( integer m = i+1; m < N; ++m ) {
            T a = A[m + i*lda];
            for ( integer r = 0; r < M; ++r ) B[r + i*ldb] -= B[r + m*ldb] * a;
          }
          if ( !unit ) for ( integer r = 0; r < M; ++r ) B[r + i*ldb] /= A[i + i*lda];
        }
      }
    }
  }

  template <typename T>
  inline void
  trsv( ULselect UPLO, Transposition TR, DiagonalType DIAG, integer N,
        T const * A, integer lda, T * x, integer incx ) {
    if ( incx == 1 ) { trsm( SideMultiply::LEFT, UPLO, TR, DIAG, N, 1, T(1), A, lda, x, N ); return; }
    std::vector<T> t( static_cast<size_t>(N) );
    for ( integer i = 0; i < N; ++i ) t[i] = x[i*incx];
    trsm( SideMultiply::LEFT, UPLO, TR, DIAG, N, 1, T(1), A, lda, t.data(), N );
    for ( integer i = 0; i < N; ++i ) x[i*incx] = t[i];
  }

  // -------------------------------------------------------------- LAPACK ---

  // LU with partial pivoting; ipiv is 1-based (LAPACK), INFO = first zero pivot
  template <typename T>
  inline integer
  getrf( integer M, integer N, T * A, integer lda, integer * ipiv ) {
    integer info = 0, kmax = std::min(M,N);
    for ( integer i = 0; i < kmax; ++i ) {
      integer p = i; T best = std::abs( A[i + i*lda] );
      for ( integer r = i+1; r < M; ++r ) { T v = std::abs( A[r + i*lda] ); if ( v > best ) { best = v; p = r; } }
      ipiv[i] = p + 1;
      if ( A[p + i*lda] == T(0) ) { if ( !info ) info = i+1; continue; }
      if ( p != i ) for ( integer c = 0; c < N; ++c ) std::swap( A[i + c*lda], A[p + c*lda] );
      T piv = A[i + i*lda];
      for ( integer r = i+1; r < M; ++r ) A[r + i*lda] /= piv;
      for ( integer c = i+1; c < N; ++c ) {
        T u = A[i + c*lda];
        for ( integer r = i+1; r < M; ++r ) A[r + c*lda] -= A[r + i*lda] * u;
      }
    }
    return info;
  }

  // row interchanges of rows i1..i2 (0-based, inclusive) with 1-based ipiv
  template <typename T>
  inline integer
  swaps( integer NCOL, T * A, integer lda, integer i1, integer i2, integer const * ipiv, integer inc ) {
    for ( integer i = i1; i <= i2; i += inc ) {
      integer p = ipiv[i] - 1;
      if ( p != i ) for ( integer c = 0; c < NCOL; ++c ) std::swap( A[i + c*lda], A[p + c*lda] );
    }
    return 0;
  }

  template <typename T>
  inline T
  house_make( integer m, integer i, T * A, integer lda ) {
    T alpha = A[i + i*lda], xn2 = 0;
    for ( integer r = i+1; r < m; ++r ) xn2 += A[r + i*lda] * A[r + i*lda];
    if ( xn2 == T(0) ) return T(0);
    T nrm  = std::sqrt( alpha*alpha + xn2 );
    T beta = alpha >= 0 ? -nrm : nrm;
    T tau  = (beta - alpha) / beta;
    T sc   = T(1) / (alpha - beta);
    for ( integer r = i+1; r < m; ++r ) A[r + i*lda] *= sc;
    A[i + i*lda] = beta;
    return tau;
  }

  template <typename T>
  inline void
  house_apply( integer m, integer i, T const * V, integer ldv, T tau, T * C, integer ldc, integer ncol ) {
    if ( tau == T(0) ) return;
    for ( integer c = 0; c < ncol; ++c ) {
      T w = C[i + c*ldc];
      for ( integer r = i+1; r < m; ++r ) w += V[r + i*ldv] * C[r + c*ldc];
      w *= tau;
      C[i + c*ldc] -= w;
      for ( integer r = i+1; r < m; ++r ) C[r + c*ldc] -= w * V[r + i*ldv];
    }
  }

  template <typename T>
  inline integer
  geqrf( integer M, integer N, nd<T> * A, integer lda, nd<T> * tau, T * work, integer lwork ) {
    if ( lwork < 0 ) { work[0] = T(std::max(1,N)); return 0; }
    integer kmax = std::min(M,N);
    for ( integer i = 0; i < kmax; ++i ) {
      tau[i] = house_make( M, i, A, lda );
      house_apply( M, i, A, lda, tau[i], A + (i+1)*lda, lda, N-i-1 );
    }
    return 0;
  }

  // QR with column pivoting; jpvt 1-based; entries != 0 on input are ignored
  template <typename T>
  inline integer
  geqp3( integer M, integer N, nd<T> * A, integer lda, integer * jpvt, nd<T> * tau, T * work, integer lwork ) {
    if ( lwork < 0 ) { work[0] = T(3*std::max(1,N)+1); return 0; }
    for ( integer j = 0; j < N; ++j ) jpvt[j] = j+1;
    integer kmax = std::min(M,N);
    for ( integer i = 0; i < kmax; ++i ) {
      integer p = i; T best = -1;
      for ( integer c = i; c < N; ++c ) {
        T s = 0;
        for ( integer r = i; r < M; ++r ) s += A[r + c*lda] * A[r + c*lda];
        if ( s > best ) { best = s; p = c; }
      }
      if ( p != i ) {
        for ( integer r = 0; r < M; ++r ) std::swap( A[r + i*lda], A[r + p*lda] );
        std::swap( jpvt[i], jpvt[p] );
      }
      tau[i] = house_make( M, i, A, lda );
      house_apply( M, i, A, lda, tau[i], A + (i+1)*lda, lda, N-i-1 );
    }
    return 0;
  }

  // C <- Q^T C (LEFT, YES) or Q C (LEFT, NO) with K reflectors stored in A
  template <typename T>
  inline integer
  ormqr( SideMultiply, Transposition TR, integer M, integer N, integer K,
         T const * A, integer lda, T const * tau, T * C, integer ldc, T *, integer ) {
    if ( TR != Transposition::NO ) {
      for ( integer i = 0; i < K; ++i ) house_apply( M, i, A, lda, tau[i], C, ldc, N );
    } else {
      for ( integer i = K-1; i >= 0; --i ) house_apply( M, i, A, lda, tau[i], C, ldc, N );
    }
    return 0;
  }

  // --------------------------------------------------- last-block solvers ---
  template <typename T>
  class DenseBase {
  protected:
    integer m_nr{0}, m_nc{0};
    std::vector<T> m_A;
    void load( integer NR, integer NC, T const * A, integer lda ) {
      m_nr = NR; m_nc = NC; m_A.assign( size_t(NR) * size_t(NC), T(0) );
      for ( integer j = 0; j < NC; ++j )
        for ( integer i = 0; i < NR; ++i ) m_A[i + size_t(j)*NR] = A[i + size_t(j)*lda];
    }
  public:
    virtual ~DenseBase() = default;
    virtual bool solve1( T x[] ) const = 0;
    bool solve( T x[] ) const { return solve1( x ); }
    bool solve( integer nrhs, T X[], integer ldX ) const {
      for ( integer c = 0; c < nrhs; ++c ) if ( !solve1( X + size_t(c)*ldX ) ) return false;
      return true;
    }
  };

  template <typename T>
  class LU : public DenseBase<T> {
    std::vector<integer> m_ipiv;
  public:
    bool factorize( integer NR, integer NC, T const * A, integer lda ) {
      if ( NR != NC ) return false;
      this->load( NR, NC, A, lda );
      m_ipiv.assign( size_t(NR), 0 );
      return getrf( NR, NC, this->m_A.data(), NR, m_ipiv.data() ) == 0;
    }
    bool solve1( T x[] ) const override {
      integer n = this->m_nr;
      swaps( 1, x, n, 0, n-1, m_ipiv.data(), 1 );
      trsm( SideMultiply::LEFT, ULselect::LOWER, Transposition::NO, DiagonalType::UNIT, n, 1, T(1), this->m_A.data(), n, x, n );
      trsm( SideMultiply::LEFT, ULselect::UPPER, Transposition::NO, DiagonalType::NON_UNIT, n, 1, T(1), this->m_A.data(), n, x, n );
      return true;
    }
  };

  template <typename T>
  class LUPQ : public DenseBase<T> {
    std::vector<integer> m_p, m_q;
  public:
    bool factorize( integer NR, integer NC, T const * A, integer lda ) {
      if ( NR != NC ) return false;
      this->load( NR, NC, A, lda );
      integer n = NR; T * a = this->m_A.data();
      m_p.assign( size_t(n), 0 ); m_q.assign( size_t(n), 0 );
      for ( integer i = 0; i < n; ++i ) {
        integer pr = i, pc = i; T best = -1;
        for ( integer c = i; c < n; ++c )
          for ( integer r = i; r < n; ++r ) { T v = std::abs( a[r + c*n] ); if ( v > best ) { best = v; pr = r; pc = c; } }
        m_p[i] = pr; m_q[i] = pc;
        if ( best == T(0) ) return false;
        for ( integer c = 0; c < n; ++c ) std::swap( a[i + c*n], a[pr + c*n] );
        for ( integer r = 0; r < n; ++r ) std::swap( a[r + i*n], a[r + pc*n] );
        T piv = a[i + i*n];
        for ( integer r = i+1; r < n; ++r ) a[r + i*n] /= piv;
        for ( integer c = i+1; c < n; ++c ) { T u = a[i + c*n]; for ( integer r = i+1; r < n; ++r ) a[r + c*n] -= a[r + i*n] * u; }
      }
      return true;
    }
    bool solve1( T x[] ) const override {
      integer n = this->m_nr;
      for ( integer i = 0; i < n; ++i ) std::swap( x[i], x[m_p[i]] );
      trsm( SideMultiply::LEFT, ULselect::LOWER, Transposition::NO, DiagonalType::UNIT, n, 1, T(1), this->m_A.data(), n, x, n );
      trsm( SideMultiply::LEFT, ULselect::UPPER, Transposition::NO, DiagonalType::NON_UNIT, n, 1, T(1), this->m_A.data(), n, x, n );
      for ( integer i = n-1; i >= 0; --i ) std::swap( x[i], x[m_q[i]] );
      return true;
    }
  };

  template <typename T>
  class QR : public DenseBase<T> {
  protected:
    std::vector<T>       m_tau;
    std::vector<integer> m_jpvt;
    bool                 m_pivot{false};
  public:
    bool factorize( integer NR, integer NC, T const * A, integer lda ) {
      if ( NR < NC ) return false;
      this->load( NR, NC, A, lda );
      m_tau.assign( size_t(NC), T(0) );
      T w;
      if ( m_pivot ) { m_jpvt.assign( size_t(NC), 0 ); geqp3( NR, NC, this->m_A.data(), NR, m_jpvt.data(), m_tau.data(), &w, 1 ); }
      else           geqrf( NR, NC, this->m_A.data(), NR, m_tau.data(), &w, 1 );
      for ( integer i = 0; i < NC; ++i ) if ( this->m_A[i + size_t(i)*NR] == T(0) ) return false;
      return true;
    }
    bool solve1( T x[] ) const override {
      integer m = this->m_nr, n = this->m_nc;
      T w;
      ormqr( SideMultiply::LEFT, Transposition::YES, m, 1, n, this->m_A.data(), m, m_tau.data(), x, m, &w, 1 );
      trsm( SideMultiply::LEFT, ULselect::UPPER, Transposition::NO, DiagonalType::NON_UNIT, n, 1, T(1), this->m_A.data(), m, x, n );
      if ( m_pivot ) {
        std::vector<T> t( static_cast<size_t>(n) );
        for ( integer i = 0; i < n; ++i ) t[ size_t(m_jpvt[i]-1) ] = x[i];
        for ( integer i = 0; i < n; ++i ) x[i] = t[i];
      }
      return true;
    }
  };

  template <typename T>
  class QRP : public QR<T> {
  public:
    QRP() { this->m_pivot = true; }
  };

  // minimum-norm least squares via one-sided Jacobi SVD
  template <typename T>
  class SVD : public DenseBase<T> {
  protected:
    std::vector<T> m_U, m_S, m_V;
    bool m_trans{false};
    integer m_M{0}, m_N{0};
    bool do_factorize( integer NR, integer NC, T const * A, integer lda ) {
      this->load( NR, NC, A, lda );
      m_trans = NR < NC;
      m_M = m_trans ? NC : NR; m_N = m_trans ? NR : NC;
      integer M = m_M, N = m_N;
      m_U.assign( size_t(M)*N, T(0) ); m_V.assign( size_t(N)*N, T(0) ); m_S.assign( size_t(N), T(0) );
      for ( integer i = 0; i < NR; ++i )
        for ( integer j = 0; j < NC; ++j ) {
          T v = this->m_A[i + size_t(j)*NR];
          if ( m_trans ) m_U[j + size_t(i)*M] = v; else m_U[i + size_t(j)*M] = v;
        }
      for ( integer j = 0; j < N; ++j ) m_V[j + size_t(j)*N] = T(1);
      T const eps = std::numeric_limits<T>::epsilon();
      for ( int sweep = 0; sweep < 80; ++sweep ) {
        bool rot = false;
        for ( integer p = 0; p < N-1; ++p )
          for ( integer q = p+1; q < N; ++q ) {
            T a = 0, b = 0, g = 0;
            for ( integer i = 0; i < M; ++i ) { T up = m_U[i + size_t(p)*M], uq = m_U[i + size_t(q)*M]; a += up*up; b += uq*uq; g += up*uq; }
            if ( g == T(0) || std::abs(g) <= eps * std::sqrt(a*b) ) continue;
            rot = true;
            T zeta = (b - a) / (2*g);
            T t = (zeta >= 0 ? T(1) : T(-1)) / (std::abs(zeta) + std::sqrt(1 + zeta*zeta));
            T c = 1 / std::sqrt(1 + t*t), s = c*t;
            for ( integer i = 0; i < M; ++i ) { T up = m_U[i + size_t(p)*M], uq = m_U[i + size_t(q)*M]; m_U[i + size_t(p)*M] = c*up - s*uq; m_U[i + size_t(q)*M] = s*up + c*uq; }
            for ( integer i = 0; i < N; ++i ) { T vp = m_V[i + size_t(p)*N], vq = m_V[i + size_t(q)*N]; m_V[i + size_t(p)*N] = c*vp - s*vq; m_V[i + size_t(q)*N] = s*vp + c*vq; }
          }
        if ( !rot ) break;
      }
      for ( integer j = 0; j < N; ++j ) {
        T s = 0;
        for ( integer i = 0; i < M; ++i ) s += m_U[i + size_t(j)*M] * m_U[i + size_t(j)*M];
        s = std::sqrt( s ); m_S[j] = s;
        if ( s > 0 ) for ( integer i = 0; i < M; ++i ) m_U[i + size_t(j)*M] /= s;
      }
      return true;
    }
  public:
    bool factorize( integer NR, integer NC, T const * A, integer lda ) { return do_factorize( NR, NC, A, lda ); }
    bool solve1( T x[] ) const override {
      integer M = m_M, N = m_N;
      T smax = 0; for ( T s : m_S ) smax = std::max( smax, s );
      T tol = smax * T(1e-12) * (sizeof(T) == 4 ? T(1e6) : T(1));
      std::vector<T> t( static_cast<size_t>(N), T(0) );
      if ( !m_trans ) {
        for ( integer j = 0; j < N; ++j ) if ( m_S[j] > tol ) { T s = 0; for ( integer i = 0; i < M; ++i ) s += m_U[i + size_t(j)*M] * x[i]; t[j] = s / m_S[j]; }
        for ( integer i = 0; i < N; ++i ) { T s = 0; for ( integer j = 0; j < N; ++j ) s += m_V[i + size_t(j)*N] * t[j]; x[i] = s; }
      } else {
        for ( integer j = 0; j < N; ++j ) if ( m_S[j] > tol ) { T s = 0; for ( integer i = 0; i < N; ++i ) s += m_V[i + size_t(j)*N] * x[i]; t[j] = s / m_S[j]; }
        std::vector<T> y( static_cast<size_t>(M), T(0) );
        for ( integer i = 0; i < M; ++i ) { T s = 0; for ( integer j = 0; j < N; ++j ) s += m_U[i + size_t(j)*M] * t[j]; y[i] = s; }
        for ( integer i = 0; i < M; ++i ) x[i] = y[i];
      }
      return true;
    }
  };

  template <typename T> class LSS : public SVD<T> {};
  template <typename T> class LSY : public SVD<T> {};

  template <typename T>
  class PINV : public SVD<T> {
  public:
    bool t_factorize( integer NR, integer NC, T const * A, integer lda ) { return this->do_factorize( NR, NC, A, lda ); }
    bool mult_inv( T const b[], integer incb, T x[], integer incx ) const {
      integer L = std::max( this->m_nr, this->m_nc );
      std::vector<T> t( static_cast<size_t>(L), T(0) );
      for ( integer i = 0; i < this->m_nr; ++i ) t[i] = b[i*incb];
      this->solve1( t.data() );
      for ( integer i = 0; i < this->m_nc; ++i ) x[i*incx] = t[i];
      return true;
    }
    bool t_mult_inv( T const b[], integer incb, T x[], integer incx ) const { return mult_inv( b, incb, x, incx ); }
    bool mult_inv( integer nrhs, T const B[], integer ldB, T X[], integer ldX ) const {
      for ( integer c = 0; c < nrhs; ++c ) mult_inv( B + size_t(c)*ldB, 1, X + size_t(c)*ldX, 1 );
      return true;
    }
    bool t_mult_inv( integer nrhs, T const B[], integer ldB, T X[], integer ldX ) const { return mult_inv( nrhs, B, ldB, X, ldX ); }
  };

} // namespace lapack_wrapper

namespace alglin {
  using lapack_wrapper::ostream_type;
  using integer   = lapack_wrapper::integer;
  using real_type = lapack_wrapper::doublereal;

  using lapack_wrapper::gemv;
  using lapack_wrapper::gemm;
  using lapack_wrapper::geqp3;
  using lapack_wrapper::geqrf;
  using lapack_wrapper::getrf;
  using lapack_wrapper::ormqr;
  using lapack_wrapper::swap;
  using lapack_wrapper::swaps;
  using lapack_wrapper::trsv;
  using lapack_wrapper::trsm;

  using lapack_wrapper::Matrix;
  using lapack_wrapper::MatrixWrapper;
  using lapack_wrapper::LinearSystemSolver;
  using lapack_wrapper::LU;
  using lapack_wrapper::LUPQ;
  using lapack_wrapper::QR;
  using lapack_wrapper::QRP;
  using lapack_wrapper::SVD;
  using lapack_wrapper::LSS;
  using lapack_wrapper::LSY;
  using lapack_wrapper::PINV;

  using lapack_wrapper::Transposition;
  using lapack_wrapper::DiagonalType;
  using lapack_wrapper::ULselect;
  using lapack_wrapper::SideMultiply;

  using Utils::Malloc;
  using std::string;
  using std::vector;
}

#include "Alglin/BABD_BorderedCR.hxx"

#endif
