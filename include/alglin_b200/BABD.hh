// alglin_b200::BABD<double> -- header-only drop-in for the reference's
// dispatch wrapper alglin::BABD<t_Value> (ebertolazzi/alglin,
// src/Alglin/BABD.hxx:56-366), cyclic-reduction branch, over the GPU
// BorderedCR of include/alglin_b200/BorderedCR.hh.
//
// Same choices, method names and return conventions as the reference:
//   * BABD_Choice::CYCLIC_REDUCTION_LU / _QR / _QRP select the BorderedCR
//     backend with the internal LU, QR or QRP panel factorization
//     (configure_cr_choice, BABD.hxx:107-124);
//   * factorize_system() / solve_system() forward to cr().factorize() and
//     cr().solve() (BABD.hxx:271-313) and return false on a numerical
//     failure (the reason is in cr().last_error());
//   * sparse_nnz / sparse_pattern / sparse_values forward to the backend with
//     0-based indices (BABD.hxx:338-366).
// The DiazLU backend (BABD_Choice::DIAZ) is not part of this library:
// selecting it throws std::runtime_error, and using_diaz() is always false.
// The constructor takes the thread count and the number of parallel blocks
// where the reference takes its thread pool; they only affect info().
//
// With ALGLIN_B200_AS_ALGLIN defined, the class is also visible as
// alglin::BABD.
#pragma once
#ifndef ALGLIN_B200_BABD_HH
#define ALGLIN_B200_BABD_HH

#include <stdexcept>
#include <string>

#include "BorderedCR.hh"

namespace alglin_b200 {

  template <typename t_Value> class BABD;

  template <>
  class BABD<double> {
  public:
    using real_type = double;
    using CRBackend = BorderedCR<double>;

    // BABD.hxx:66-71
    enum class BABD_Choice : integer {
      DIAZ                 = 1,
      CYCLIC_REDUCTION_LU  = 2,
      CYCLIC_REDUCTION_QR  = 3,
      CYCLIC_REDUCTION_QRP = 4
    };

    static std::string Choice_to_string( BABD_Choice c ) {
      switch ( c ) {
        case BABD_Choice::DIAZ:                 return "Diaz";
        case BABD_Choice::CYCLIC_REDUCTION_LU:  return "CyclicReduction+LU";
        case BABD_Choice::CYCLIC_REDUCTION_QR:  return "CyclicReduction+QR";
        case BABD_Choice::CYCLIC_REDUCTION_QRP: return "CyclicReduction+QRP";
      }
      return "none";
    }

  private:
    BABD_Choice m_choice{ BABD_Choice::CYCLIC_REDUCTION_LU };
    CRBackend   m_cr;

    void configure_cr_choice() {
      switch ( m_choice ) {
        case BABD_Choice::CYCLIC_REDUCTION_LU:  m_cr.select_LU();  break;
        case BABD_Choice::CYCLIC_REDUCTION_QR:  m_cr.select_QR();  break;
        case BABD_Choice::CYCLIC_REDUCTION_QRP: m_cr.select_QRP(); break;
        case BABD_Choice::DIAZ: break;
      }
    }

  public:
    BABD( BABD const & ) = delete;
    BABD const & operator = ( BABD const & ) = delete;

    explicit BABD( BABD_Choice choice = BABD_Choice::CYCLIC_REDUCTION_LU, integer num_threads = 0,
                   integer num_parallel_block = 0 )
    : m_cr( num_threads, num_parallel_block ) {
      selectSolver( choice );
    }

    BABD_Choice selected_solver() const { return m_choice; }
    bool using_diaz() const { return false; }
    bool using_cyclic_reduction() const { return true; }

    CRBackend & cr() { return m_cr; }
    CRBackend const & cr() const { return m_cr; }

    // BABD.hxx:215-228
    void selectSolver( BABD_Choice choice ) {
      if ( choice == BABD_Choice::DIAZ )
        throw std::runtime_error( "BABD::selectSolver, the DiazLU backend is not available in alglin_b200\n" );
      m_choice = choice;
      configure_cr_choice();
    }

    std::string info() const { return m_cr.info_algo(); }
    integer nrows() const { return m_cr.nrows(); }
    integer ncols() const { return m_cr.ncols(); }

    bool factorize_system() { return m_cr.factorize(); }
    bool solve_system( real_type in_out[] ) const { return m_cr.solve( in_out ); }
    bool solve_system( integer nrhs, real_type in_out[], integer ldIO ) const {
      return m_cr.solve( nrhs, in_out, ldIO );
    }
    bool factorize() { return factorize_system(); }
    bool solve( real_type in_out[] ) const { return solve_system( in_out ); }
    bool solve( integer nrhs, real_type in_out[], integer ldIO ) const {
      return solve_system( nrhs, in_out, ldIO );
    }

    integer sparse_nnz() const { return m_cr.sparse_nnz(); }
    void sparse_pattern( integer I[], integer J[] ) const { m_cr.sparse_pattern( I, J, 0 ); }
    void sparse_values( real_type vals[] ) const { m_cr.sparse_values( vals ); }
  };

} // namespace alglin_b200

#ifdef ALGLIN_B200_AS_ALGLIN
namespace alglin {
  using alglin_b200::BABD;
}
#endif

#endif
