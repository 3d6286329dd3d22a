// Minimal stand-in for hyteg/geometry/GeometryMap.hpp: the point/matrix types and the virtual
// blending-map interface (evalF, evalDF) that the reference's generated forms call.  Test
// infrastructure only.
#pragma once
#include <array>
#include <cstdlib>
#include <functional>
#include <memory>

#include "core/DataTypes.h"

#define WALBERLA_ABORT( msg ) std::abort()

namespace hyteg {
using walberla::real_t;

class Point3D
{
 public:
   Point3D() = default;
   Point3D( real_t a, real_t b, real_t c )
   : v{ a, b, c }
   {}
   real_t&       operator[]( int i ) { return v[i]; }
   const real_t& operator[]( int i ) const { return v[i]; }

 private:
   real_t v[3] = { 0, 0, 0 };
};

template < typename T, int R, int C >
class Matrix
{
 public:
   T&       operator()( int r, int c ) { return a[r * C + c]; }
   const T& operator()( int r, int c ) const { return a[r * C + c]; }
   T        a[R * C] = {};
};
template < int R, int C >
using Matrixr  = Matrix< real_t, R, C >;
using Matrix2r = Matrix< real_t, 2, 2 >;
using Matrix3r = Matrix< real_t, 3, 3 >;
using Matrix4r = Matrix< real_t, 4, 4 >;

class GeometryMap
{
 public:
   virtual ~GeometryMap() = default;
   virtual void   evalF( const Point3D& x, Point3D& Fx ) const = 0;
   virtual void   evalDF( const Point3D&, Matrix2r& ) const { std::abort(); }
   virtual real_t evalDF( const Point3D& x, Matrix3r& DFx ) const = 0;
};
}  // namespace hyteg
