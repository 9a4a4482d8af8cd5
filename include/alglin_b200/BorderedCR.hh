// alglin_b200::BorderedCR<double> -- header-only C++ drop-in for the
// reference class alglin::BorderedCR<double> (ebertolazzi/alglin,
// src/Alglin/BABD_BorderedCR.hxx:104-1176), implemented over the C ABI of
// libalglin_b200.so (include/alglin_b200.h).
//
// Same method names, argument orders and error behaviour as the reference:
//   * factorize() / solve() return false on a numerical failure and leave the
//     reason in last_error();
//   * bad arguments throw std::runtime_error (the reference throws
//     Utils::Runtime_Error, which derives from std::runtime_error);
//   * the element accessors B(nbl,i,j) ... H(i,j) return references into the
//     handle's host copy of the matrix.
// The constructor has the reference's signature, BorderedCR( TP, npb ) with
// TP a Utils::ThreadPoolBase* (hxx:373-384): the pool's thread count and npb
// only affect info(), because the factorization runs on the GPU.  A program
// that has the real UtilsLite pool defines ALGLIN_B200_EXTERNAL_UTILS and
// includes it first; otherwise this header supplies a minimal Utils namespace
// (ThreadPoolBase with thread_count(), ThreadPool0, ThreadPool1) so that the
// reference's `Utils::ThreadPool1 TP(n); BorderedCR<double> BCR(&TP);`
// compiles unchanged.  The class derives from LinearSystemSolver<double>, the
// base whose factorize/solve/t_solve overloads the reference class overrides
// (hxx:105, 362-364).
//
// With ALGLIN_B200_AS_ALGLIN defined, the class is also visible as
// alglin::BorderedCR so that existing code switches by changing its include.
#pragma once
#ifndef ALGLIN_B200_BORDEREDCR_HH
#define ALGLIN_B200_BORDEREDCR_HH

#include <ostream>
#include <stdexcept>
#include <string>
#include <string_view>
#include <vector>

#include "../alglin_b200.h"

#ifndef ALGLIN_B200_EXTERNAL_UTILS
// Thread-pool types of the reference's Utils library, reduced to what the
// BorderedCR constructor reads (the thread count).  Tasks never run here.
namespace Utils {
  class ThreadPoolBase {
  public:
    virtual ~ThreadPoolBase() = default;
    virtual unsigned thread_count() const = 0;
  };
  class ThreadPool0 : public ThreadPoolBase {
  public:
    explicit ThreadPool0( unsigned = 1 ) {}
    unsigned thread_count() const override { return 1; }
  };
  class ThreadPool1 : public ThreadPoolBase {
    unsigned m_n;
  public:
    explicit ThreadPool1( unsigned n ) : m_n( n < 1 ? 1 : n ) {}
    unsigned thread_count() const override { return m_n; }
  };
}
#endif

namespace alglin_b200 {

  using integer = int;

  // column-major view with a leading dimension (the reference's MatrixWrapper)
  template <typename T>
  class MatrixWrapper {
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

  // Base of the reference's BorderedCR (LapackWrapper's LinearSystemSolver,
  // which the reference does not vendor): the factorize/solve/t_solve virtuals
  // and the MatrixWrapper forms of solve/t_solve (used by the reference tests,
  // test18:1018).
  template <typename t_Value>
  class LinearSystemSolver {
  public:
    using real_type = t_Value;
    virtual ~LinearSystemSolver() = default;
    virtual bool factorize() = 0;
    virtual bool solve( t_Value x[] ) const = 0;
    virtual bool solve( integer nrhs, t_Value rhs[], integer ldRhs ) const = 0;
    virtual bool t_solve( t_Value x[] ) const = 0;
    virtual bool t_solve( integer nrhs, t_Value rhs[], integer ldRhs ) const = 0;
    bool solve( MatrixWrapper<t_Value> & M ) const { return this->solve( M.ncols(), M.data(), M.ldim() ); }
    bool t_solve( MatrixWrapper<t_Value> & M ) const { return this->t_solve( M.ncols(), M.data(), M.ldim() ); }
  };

  template <typename t_Value> class BorderedCR;

  template <>
  class BorderedCR<double> : public LinearSystemSolver<double> {
  public:
    using real_type = double;
    using MatW      = MatrixWrapper<double>;

    enum class BORDERED_Choice      : integer { LU = 0, QR = 1, QRP = 2 };
    enum class BORDERED_LAST_Choice : integer { LU = 0, LUPQ, QR, QRP, SVD, LSS, LSY, PINV };
    enum class BORDERED_LAST_Choice2: integer { NONE = 0, SVD, LSS, LSY, PINV };

  private:
    bcr_handle m_h{nullptr};

    void chk( int rc ) const {
      if ( rc == BCR_OK ) return;
      throw std::runtime_error( bcr_last_error( m_h ) );
    }
    bool ok_or_false( int rc ) const {
      if ( rc == BCR_OK ) return true;
      if ( rc == BCR_NUMERICAL ) return false;
      throw std::runtime_error( bcr_last_error( m_h ) );
    }
    static void chk_dims( MatW const & M, integer r, integer c, char const * what ) {
      if ( M.nrows() != r || M.ncols() != c )
        throw std::runtime_error( std::string("BorderedCR::") + what + " bad dimension" );
    }

  public:
    BorderedCR( BorderedCR const & ) = delete;
    BorderedCR const & operator = ( BorderedCR const & ) = delete;

    using LinearSystemSolver<double>::solve;
    using LinearSystemSolver<double>::t_solve;

    // BorderedCR( Utils::ThreadPoolBase * TP, integer num_parallel_block = 0 )
    // (hxx:373-384): with a pool, npb = its thread count, or the smaller of
    // the two when npb > 0; without one (TP == nullptr), a single block
    explicit BorderedCR( Utils::ThreadPoolBase * TP, integer num_parallel_block = 0 ) {
      integer const nth = TP != nullptr ? integer( TP->thread_count() ) : 0;
      if ( bcr_create( &m_h, nth, nth > 0 ? num_parallel_block : 0 ) != BCR_OK )
        throw std::runtime_error( "alglin_b200: bcr_create failed" );
    }
    // the same from a thread count (no pool object needed)
    explicit BorderedCR( integer num_threads = 0, integer num_parallel_block = 0 ) {
      if ( bcr_create( &m_h, num_threads, num_parallel_block ) != BCR_OK )
        throw std::runtime_error( "alglin_b200: bcr_create failed" );
    }
    ~BorderedCR() override { bcr_destroy( m_h ); }

    bcr_handle handle() const { return m_h; }

    void allocate( integer nblock, integer n, integer qr, integer qx, integer nr, integer nx )
    { chk( bcr_allocate( m_h, nblock, n, qr, qx, nr, nx ) ); }
    void dup( BorderedCR const & M ) { chk( bcr_dup( m_h, M.m_h ) ); }

    // ---------------------------------------------------------- selection
    void select( std::string_view s )       { chk( bcr_select( m_h, std::string(s).c_str() ) ); }
    void select_LU()  { select( "LU" ); }
    void select_QR()  { select( "QR" ); }
    void select_QRP() { select( "QRP" ); }
    void select_last( std::string_view s )  { chk( bcr_select_last( m_h, std::string(s).c_str() ) ); }
    void select_last_LU()   { select_last( "LU" ); }
    void select_last_LUPQ() { select_last( "LUPQ" ); }
    void select_last_QR()   { select_last( "QR" ); }
    void select_last_QRP()  { select_last( "QRP" ); }
    void select_last_SVD()  { select_last( "SVD" ); }
    void select_last_LSS()  { select_last( "LSS" ); }
    void select_last_LSY()  { select_last( "LSY" ); }
    void select_last_PINV() { select_last( "PINV" ); }
    void select_last2( std::string_view s ) { chk( bcr_select_last2( m_h, std::string(s).c_str() ) ); }
    void select_last2_NONE() { select_last2( "NONE" ); }
    void select_last2_SVD()  { select_last2( "SVD" ); }
    void select_last2_LSS()  { select_last2( "LSS" ); }
    void select_last2_LSY()  { select_last2( "LSY" ); }
    void select_last2_PINV() { select_last2( "PINV" ); }

    static std::string choice_to_string( BORDERED_Choice c ) {
      switch ( c ) {
        case BORDERED_Choice::LU:  return "CyclicReduction+LU";
        case BORDERED_Choice::QR:  return "CyclicReduction+QR";
        case BORDERED_Choice::QRP: return "CyclicReduction+QRP";
      }
      return "none";
    }
    static std::string choice_to_string( BORDERED_LAST_Choice c ) {
      static char const * nm[] = { "LU", "LUPQ", "QR", "QRP", "SVD", "LSS", "LSY", "PINV" };
      return std::string("LastBlock ") + nm[ integer(c) ];
    }
    static std::string choice_to_string( BORDERED_LAST_Choice2 c ) {
      static char const * nm[] = { "NONE", "SVD", "LSS", "LSY", "PINV" };
      return std::string("LastBlock ") + nm[ integer(c) ];
    }
    std::string info_algo_block() const {
      int a, b, c; bcr_selected( m_h, &a, &b, &c ); return choice_to_string( BORDERED_Choice(a) );
    }
    std::string info_algo_last_block() const {
      int a, b, c; bcr_selected( m_h, &a, &b, &c ); return choice_to_string( BORDERED_LAST_Choice(b) );
    }
    std::string info_algo_last_block2() const {
      int a, b, c; bcr_selected( m_h, &a, &b, &c ); return choice_to_string( BORDERED_LAST_Choice2(c) );
    }
    std::string info_algo() const {
      return info_algo_block() + " and " + info_algo_last_block() + " and " + info_algo_last_block2();
    }
    std::string info( std::string_view indent = "" ) const { return bcr_info( m_h, std::string(indent).c_str() ); }
    void info( std::ostream & s ) const { s << info(); }
    std::string_view last_error() const { return bcr_last_error( m_h ); }

    void set_factorize_use_thread( bool yes ) { chk( bcr_set_factorize_use_thread( m_h, yes ) ); }
    void set_solve_use_thread( bool yes )     { chk( bcr_set_solve_use_thread( m_h, yes ) ); }
    bool factorize_use_thread() const { return bcr_factorize_use_thread( m_h ) != 0; }
    bool solve_use_thread() const     { return bcr_solve_use_thread( m_h ) != 0; }
    void set_num_parallel_block( integer npb ) { chk( bcr_set_num_parallel_block( m_h, npb ) ); }
    void set_debug( bool yes ) { chk( bcr_set_debug( m_h, yes ) ); }
    void check_matrix() { chk( bcr_check_matrix( m_h ) ); }

    // extensions: FP32 factors with FP64 iterative refinement
    void set_precision_mixed( bool yes ) {
      chk( bcr_set_precision( m_h, yes ? BCR_PRECISION_MIXED : BCR_PRECISION_FP64 ) );
    }
    void set_refinement( real_type tol, integer max_iter ) { chk( bcr_set_refinement( m_h, tol, max_iter ) ); }
    void refinement_info( integer & iters, real_type & relres ) const {
      chk( bcr_refinement_info( m_h, &iters, &relres ) );
    }

    // -------------------------------------------------------------- sizes
    integer nrows() const            { return bcr_nrows( m_h ); }
    integer ncols() const            { return bcr_ncols( m_h ); }
    integer number_of_blocks() const { return bcr_number_of_blocks( m_h ); }
    integer block_size() const       { return bcr_block_size( m_h ); }
    integer dim_qr() const { return bcr_dim_qr( m_h ); }
    integer dim_qx() const { return bcr_dim_qx( m_h ); }
    integer dim_nr() const { return bcr_dim_nr( m_h ); }
    integer dim_nx() const { return bcr_dim_nx( m_h ); }
    integer Nr() const { return bcr_Nr( m_h ); }
    integer Nc() const { return bcr_Nc( m_h ); }

    // ------------------------------------------------------------ zeroing
    void zero_D()  { chk( bcr_zero_D( m_h ) ); }
    void zero_E()  { chk( bcr_zero_E( m_h ) ); }
    void zero_B()  { chk( bcr_zero_B( m_h ) ); }
    void zero_F()  { chk( bcr_zero_F( m_h ) ); }
    void zero_H()  { chk( bcr_zero_H( m_h ) ); }
    void zero_C()  { chk( bcr_zero_C( m_h ) ); }
    void zero_Cq() { chk( bcr_zero_Cq( m_h ) ); }
    void fill_zero() { chk( bcr_fill_zero( m_h ) ); }

    // ------------------------------------------------------------ loaders
    void load_B( integer nbl, real_type const B[], integer ldB )   { chk( bcr_load_B( m_h, nbl, B, ldB ) ); }
    void add_to_B( integer nbl, real_type const B[], integer ldB ) { chk( bcr_add_to_B( m_h, nbl, B, ldB ) ); }
    void load_C( integer nbl, real_type const C[], integer ldC )   { chk( bcr_load_C( m_h, nbl, C, ldC ) ); }
    void add_to_C( integer nbl, real_type const C[], integer ldC ) { chk( bcr_add_to_C( m_h, nbl, C, ldC ) ); }
    void add_to_C2( integer nbl, real_type const C[], integer ldC ) { chk( bcr_add_to_C2( m_h, nbl, C, ldC ) ); }
    void add_to_C2F( integer nbl, real_type const C[], integer ldC ) { chk( bcr_add_to_C2F( m_h, nbl, C, ldC ) ); }
    void load_D( integer nbl, real_type const D[], integer ldD )   { chk( bcr_load_D( m_h, nbl, D, ldD ) ); }
    void load_E( integer nbl, real_type const E[], integer ldE )   { chk( bcr_load_E( m_h, nbl, E, ldE ) ); }
    void load_DE( integer nbl, real_type const DE[], integer ld )  { chk( bcr_load_DE( m_h, nbl, DE, ld ) ); }
    void load_DEB( integer nbl, real_type const DEB[], integer ld ){ chk( bcr_load_DEB( m_h, nbl, DEB, ld ) ); }
    void load_F( real_type const F[], integer ldF )     { chk( bcr_load_F( m_h, F, ldF ) ); }
    void add_to_F( real_type const F[], integer ldF )   { chk( bcr_add_to_F( m_h, F, ldF ) ); }
    void load_Cq( real_type const Cq[], integer ldC )   { chk( bcr_load_Cq( m_h, Cq, ldC ) ); }
    void load_CqF( real_type const CqF[], integer ld )  { chk( bcr_load_CqF( m_h, CqF, ld ) ); }
    void load_bottom( real_type const H0[], integer ld0, real_type const HN[], integer ldN,
                      real_type const Hq[], integer ldQ, real_type const Hp[], integer ldP )
    { chk( bcr_load_bottom( m_h, H0, ld0, HN, ldN, Hq, ldQ, Hp, ldP ) ); }
    void load_bottom( real_type const H[], integer ldH ) { chk( bcr_load_bottom_H( m_h, H, ldH ) ); }
    void load_bottom2( real_type const C0[], integer ld0, real_type const CN[], integer ldN,
                       real_type const Cq[], integer ldCq, real_type const F[], integer ldF )
    { chk( bcr_load_bottom2( m_h, C0, ld0, CN, ldN, Cq, ldCq, F, ldF ) ); }

    // MatrixWrapper overloads (the reference checks the sizes and throws)
    void load_B( integer nbl, MatW const & B ) { chk_dims( B, block_size(), dim_nx(), "load_B" ); load_B( nbl, B.data(), B.ldim() ); }
    void add_to_B( integer nbl, MatW const & B ) { chk_dims( B, block_size(), dim_nx(), "add_to_B" ); add_to_B( nbl, B.data(), B.ldim() ); }
    void load_C( integer nbl, MatW const & C ) { chk_dims( C, dim_nr(), block_size(), "load_C" ); load_C( nbl, C.data(), C.ldim() ); }
    void add_to_C( integer nbl, MatW const & C ) { chk_dims( C, dim_nr(), block_size(), "add_to_C" ); add_to_C( nbl, C.data(), C.ldim() ); }
    void add_to_C2( integer nbl, MatW const & C ) { chk_dims( C, dim_nr(), 2*block_size(), "add_to_C2" ); add_to_C2( nbl, C.data(), C.ldim() ); }
    void add_to_C2F( integer nbl, MatW const & C ) { chk_dims( C, dim_nr(), 2*block_size()+dim_nx(), "add_to_C2F" ); add_to_C2F( nbl, C.data(), C.ldim() ); }
    void load_D( integer nbl, MatW const & D ) { chk_dims( D, block_size(), block_size(), "load_D" ); load_D( nbl, D.data(), D.ldim() ); }
    void load_E( integer nbl, MatW const & E ) { chk_dims( E, block_size(), block_size(), "load_E" ); load_E( nbl, E.data(), E.ldim() ); }
    void load_F( MatW const & F ) { chk_dims( F, dim_nr(), dim_nx(), "load_F" ); load_F( F.data(), F.ldim() ); }
    void add_to_F( MatW const & F ) { chk_dims( F, dim_nr(), dim_nx(), "add_to_F" ); add_to_F( F.data(), F.ldim() ); }
    void load_Cq( MatW const & Cq ) { chk_dims( Cq, dim_nr(), dim_qx(), "load_Cq" ); load_Cq( Cq.data(), Cq.ldim() ); }
    void load_bottom( MatW const & H0, MatW const & HN, MatW const & Hq, MatW const & Hp ) {
      integer m = block_size() + dim_qr();
      chk_dims( H0, m, block_size(), "load_bottom" ); chk_dims( HN, m, block_size(), "load_bottom" );
      chk_dims( Hq, m, dim_qx(), "load_bottom" );     chk_dims( Hp, m, dim_nx(), "load_bottom" );
      load_bottom( H0.data(), H0.ldim(), HN.data(), HN.ldim(), Hq.data(), Hq.ldim(), Hp.data(), Hp.ldim() );
    }
    void load_bottom( MatW const & H ) { chk_dims( H, block_size() + dim_qr(), Nc(), "load_bottom" ); load_bottom( H.data(), H.ldim() ); }
    void load_bottom2( MatW const & C0, MatW const & CN, MatW const & Cq, MatW const & F ) {
      chk_dims( C0, dim_nr(), block_size(), "load_bottom2" ); chk_dims( CN, dim_nr(), block_size(), "load_bottom2" );
      chk_dims( Cq, dim_nr(), dim_qx(), "load_bottom2" );     chk_dims( F, dim_nr(), dim_nx(), "load_bottom2" );
      load_bottom2( C0.data(), C0.ldim(), CN.data(), CN.ldim(), Cq.data(), Cq.ldim(), F.data(), F.ldim() );
    }
    void load_bottom2( MatW const & H ) { chk_dims( H, dim_nr(), Nc(), "load_bottom2" ); chk( bcr_load_bottom2_H( m_h, H.data(), H.ldim() ) ); }

    // -------------------------------------------------- element accessors
    double & B( integer nbl, integer i, integer j ) { return bcr_block_data( m_h, 'B', nbl )[ i + j * block_size() ]; }
    double & C( integer nbl, integer i, integer j ) { return bcr_block_data( m_h, 'C', nbl )[ i + j * dim_nr() ]; }
    double & D( integer nbl, integer i, integer j ) { return bcr_block_data( m_h, 'D', nbl )[ i + j * block_size() ]; }
    double & E( integer nbl, integer i, integer j ) { return bcr_block_data( m_h, 'E', nbl )[ i + j * block_size() ]; }
    double & F( integer i, integer j )  { return bcr_block_data( m_h, 'F', 0 )[ i + j * dim_nr() ]; }
    double & Cq( integer i, integer j ) { return bcr_block_data( m_h, 'Q', 0 )[ i + j * dim_nr() ]; }
    double & H( integer i, integer j )  { return bcr_block_data( m_h, 'H', 0 )[ i + j * ( block_size() + dim_qr() ) ]; }

    // --------------------------------------------------- factorize, solve
    bool factorize() override { return ok_or_false( bcr_factorize( m_h ) ); }
    bool solve( real_type x[] ) const override { return ok_or_false( bcr_solve( m_h, x ) ); }
    bool solve( integer nrhs, real_type rhs[], integer ldRhs ) const override { return ok_or_false( bcr_solve_n( m_h, nrhs, rhs, ldRhs ) ); }
    bool t_solve( real_type x[] ) const override { chk( bcr_t_solve( m_h, x ) ); return false; }
    bool t_solve( integer nrhs, real_type rhs[], integer ld ) const override { chk( bcr_t_solve_n( m_h, nrhs, rhs, ld ) ); return false; }

    void Mv( real_type const x[], real_type res[] ) const { chk( bcr_mv( m_h, x, res ) ); }
    void add_Mv( real_type alpha, real_type const x[], real_type res[] ) const { chk( bcr_add_mv( m_h, alpha, x, res ) ); }
    void add_Mv( real_type const x[], real_type res[] ) const { add_Mv( 1.0, x, res ); }

    // ------------------------------------------------------------- sparse
    integer sparse_nnz() const { return bcr_sparse_nnz( m_h ); }
    void sparse_pattern( integer I[], integer J[], integer offs ) const { chk( bcr_sparse_pattern( m_h, I, J, offs ) ); }
    void sparse_values( real_type V[] ) const { chk( bcr_sparse_values( m_h, V ) ); }
    void sparse_load( real_type const V[], integer const I[], integer roff, integer const J[], integer coff,
                      integer nnz, bool do_error = true )
    { chk( bcr_sparse_load( m_h, V, I, roff, J, coff, nnz, do_error ? 1 : 0 ) ); }

    void print_matlab_script( std::ostream & stream ) const {
      integer const nnz = sparse_nnz();
      std::string out;
      std::vector<integer> I( static_cast<size_t>(nnz) ), J( static_cast<size_t>(nnz) );
      std::vector<real_type> V( static_cast<size_t>(nnz) );
      sparse_pattern( I.data(), J.data(), 1 );
      sparse_values( V.data() );
      auto dump = [&]( char const * name, auto const & v ) {
        stream << name << " = [ " << v[0];
        for ( integer i = 1; i < nnz; ++i ) {
          if ( ( i % 20 ) == 0 ) stream << ", ...\n  " << v[i];
          else stream << ",  " << v[i];
        }
        stream << " ];\n\n";
      };
      if ( nnz > 0 ) { dump( "I", I ); dump( "J", J ); dump( "V", V ); }
      stream << "nr  = " << nrows() << ";\nnc  = " << ncols() << ";\n\nnnz = " << nnz
             << ";\n\nMAT = sparse( I, J, V, nr, nc );\n";
    }
  };

} // namespace alglin_b200

#ifdef ALGLIN_B200_AS_ALGLIN
namespace alglin {
  using alglin_b200::BorderedCR;
  using alglin_b200::LinearSystemSolver;
  using alglin_b200::MatrixWrapper;
  using integer = alglin_b200::integer;
}
#endif

#endif
