// Minimal stand-in for the Eigen::Map operations the reference BorderedCR path
// uses (copy / add / negate / scale of column-major views, topRows, fill,
// setZero).  Part of the oracle build shim: it only exists so that the
// unmodified reference sources compile without the absent UtilsLite/Eigen
// submodules.  Test infrastructure, not product code.
#pragma once
#ifndef ORACLE_SHIM_UTILS_EIGEN_HH
#define ORACLE_SHIM_UTILS_EIGEN_HH

namespace Eigen {

  constexpr int Dynamic = -1;

  template <typename T, int R, int C>
  struct Matrix { using Scalar = T; };

  template <typename T>
  struct View;

  template <typename T>
  struct ScaledView { T a; View<T> const & v; };

  template <typename T>
  struct NegView { View<T> const & v; };

  template <typename T>
  struct View {
    T * p{nullptr};
    long rows{0}, cols{0}, ld{0};

    View() = default;
    View( T * p_, long r, long c, long l ) : p(p_), rows(r), cols(c), ld(l) {}

    T & at( long i, long j ) const { return p[i + j * ld]; }

    View & noalias() { return *this; }
    View topRows( long r ) const { return View( p, r, cols, ld ); }

    View & operator = ( View const & o ) {
      for ( long j = 0; j < cols; ++j )
        for ( long i = 0; i < rows; ++i ) at(i,j) = o.at(i,j);
      return *this;
    }
    View & operator += ( View const & o ) {
      for ( long j = 0; j < cols; ++j )
        for ( long i = 0; i < rows; ++i ) at(i,j) += o.at(i,j);
      return *this;
    }
    View & operator = ( NegView<T> const & o ) {
      for ( long j = 0; j < cols; ++j )
        for ( long i = 0; i < rows; ++i ) at(i,j) = -o.v.at(i,j);
      return *this;
    }
    View & operator += ( ScaledView<T> const & o ) {
      for ( long j = 0; j < cols; ++j )
        for ( long i = 0; i < rows; ++i ) at(i,j) += o.a * o.v.at(i,j);
      return *this;
    }
    void fill( T v ) {
      for ( long j = 0; j < cols; ++j )
        for ( long i = 0; i < rows; ++i ) at(i,j) = v;
    }
    void setZero() { fill( T(0) ); }

    NegView<T> operator - () const { return NegView<T>{ *this }; }
  };

  template <typename T>
  inline ScaledView<T> operator * ( T a, View<T> const & v ) { return ScaledView<T>{ a, v }; }

  template <typename M>
  struct Map : public View<typename M::Scalar> {
    using S = typename M::Scalar;
    Map( S * p, long n ) : View<S>( p, n, 1, n ) {}
    Map( S * p, long r, long c ) : View<S>( p, r, c, r ) {}
    using View<S>::operator=;
    using View<S>::operator+=;
  };

} // namespace Eigen

#endif
