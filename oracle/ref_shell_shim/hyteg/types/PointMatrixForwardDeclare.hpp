// Stand-in for hyteg/types/PointMatrixForwardDeclare.hpp (which pulls Eigen, absent here) for the
// oracle's shell-map library: small point and dense matrix types with the operations the
// reference's IcosahedralShellMap and generated forms use.  Test infrastructure only.
#pragma once
#include <cmath>
#include <cstdlib>
#include <memory>

#include "core/DataTypes.h"

namespace hyteg {

template < typename T, int N >
class PointND
{
 public:
   PointND() = default;
   PointND( T a, T b, T c )
   : v{ a, b, c }
   {}
   T&       operator[]( int i ) { return v[i]; }
   const T& operator[]( int i ) const { return v[i]; }
   T        dot( const PointND& o ) const
   {
      T s = 0;
      for ( int i = 0; i < N; ++i ) s += v[i] * o.v[i];
      return s;
   }
   T        squaredNorm() const { return dot( *this ); }
   T        norm() const { return std::sqrt( squaredNorm() ); }
   PointND  operator-( const PointND& o ) const
   {
      PointND r;
      for ( int i = 0; i < N; ++i ) r.v[i] = v[i] - o.v[i];
      return r;
   }
   PointND operator+( const PointND& o ) const
   {
      PointND r;
      for ( int i = 0; i < N; ++i ) r.v[i] = v[i] + o.v[i];
      return r;
   }
   PointND& operator/=( T s )
   {
      for ( int i = 0; i < N; ++i ) v[i] /= s;
      return *this;
   }
   PointND operator*( T s ) const
   {
      PointND r;
      for ( int i = 0; i < N; ++i ) r.v[i] = v[i] * s;
      return r;
   }

 private:
   T v[N] = {};
};
template < typename T, int N >
PointND< T, N > operator*( T s, const PointND< T, N >& p )
{
   return p * s;
}

using Point2D = PointND< walberla::real_t, 2 >;
using Point3D = PointND< walberla::real_t, 3 >;

inline Point3D crossProduct( const Point3D& a, const Point3D& b )
{
   return Point3D( a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0] );
}

template < typename T, int R, int C >
class Matrix
{
 public:
   T&       operator()( int r, int c ) { return a[r * C + c]; }
   const T& operator()( int r, int c ) const { return a[r * C + c]; }
   // inverse of a 2x2 or 3x3 matrix by the adjugate
   Matrix inverse() const
   {
      Matrix m;
      if constexpr ( R == 3 && C == 3 )
      {
         const Matrix& A = *this;
         const T det = A( 0, 0 ) * ( A( 1, 1 ) * A( 2, 2 ) - A( 1, 2 ) * A( 2, 1 ) ) - A( 0, 1 ) * ( A( 1, 0 ) * A( 2, 2 ) - A( 1, 2 ) * A( 2, 0 ) ) +
                       A( 0, 2 ) * ( A( 1, 0 ) * A( 2, 1 ) - A( 1, 1 ) * A( 2, 0 ) );
         for ( int i = 0; i < 3; ++i )
            for ( int j = 0; j < 3; ++j )
            {
               const int r0 = ( j + 1 ) % 3, r1 = ( j + 2 ) % 3, c0 = ( i + 1 ) % 3, c1 = ( i + 2 ) % 3;
               m( i, j ) = ( A( r0, c0 ) * A( r1, c1 ) - A( r0, c1 ) * A( r1, c0 ) ) / det;
            }
      }
      else if constexpr ( R == 2 && C == 2 )
      {
         const T det = a[0] * a[3] - a[1] * a[2];
         m.a[0] = a[3] / det, m.a[1] = -a[1] / det, m.a[2] = -a[2] / det, m.a[3] = a[0] / det;
      }
      else
         std::abort();
      return m;
   }
   T a[R * C] = {};
};
template < int R, int C >
using Matrixr  = Matrix< walberla::real_t, R, C >;
using Matrix2r = Matrixr< 2, 2 >;
using Matrix3r = Matrixr< 3, 3 >;
using Matrix4r = Matrixr< 4, 4 >;

}  // namespace hyteg
