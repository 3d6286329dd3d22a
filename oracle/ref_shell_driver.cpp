// Oracle library libhyteg_ref_shell.so: the reference's IcosahedralShellMap
// (src/hyteg/geometry/IcosahedralShellMap.hpp) compiled from its source over the stand-ins in
// oracle/ref_shell_shim, with the reference's own GeometryMap class (which is why it is a library of
// its own: libhyteg_ref.so's form shims declare a smaller GeometryMap).  The map classifies each
// macro-cell itself (ray / reference / third / fourth vertex, skew cells borrowing a neighbour of
// the same prism), so the oracle's restated map is checked against the reference's classification
// and formulas.  TEST INFRASTRUCTURE ONLY.
#include <cstdlib>

#include "hyteg/geometry/IcosahedralShellMap.hpp"

namespace hyteg {
// out-of-line virtual members of GeometryMap (GeometryMap.cpp is not compiled here); the shell map
// overrides every one this library calls
void   GeometryMap::evalFinv( const Point3D&, Point3D& ) const { std::abort(); }
real_t GeometryMap::evalDF( const Point3D&, Matrix3r& ) const { std::abort(); }
void   GeometryMap::evalDFinvDF( const Point3D&, Matrixr< 2, 4 >& ) const { std::abort(); }
void   GeometryMap::evalDFinvDF( const Point3D&, Matrixr< 3, 9 >& ) const { std::abort(); }
void   GeometryMap::evalDFinv( const Point3D&, Matrix3r& ) const { std::abort(); }
bool   GeometryMap::verifyPointPairing( const Point3D&, const Point3D&, real_t ) const { std::abort(); }
}  // namespace hyteg

// F(x) and DF(x) (row-major 3x3) of the shell map of macro-cell `cell` at npts points; det receives
// the value evalDF returns
extern "C" __attribute__( ( visibility( "default" ) ) ) int ref_shell_map_eval( int nv, const double* xyz, int nc, const int* tets, int cell, int npts, const double* x, double* F,
                                   double* DF, double* det )
{
   if ( cell < 0 || cell >= nc ) return 1;
   hyteg::SetupPrimitiveStorage s( nv, xyz, nc, tets );
   hyteg::IcosahedralShellMap   map( *s.getCell( hyteg::PrimitiveID( 2000000 + cell ) ), s );
   for ( int p = 0; p < npts; ++p )
   {
      const hyteg::Point3D xp( x[3 * p], x[3 * p + 1], x[3 * p + 2] );
      hyteg::Point3D       Fx;
      map.evalF( xp, Fx );
      hyteg::Matrix3r D;
      det[p] = map.evalDF( xp, D );
      for ( int i = 0; i < 3; ++i )
      {
         F[3 * p + i] = Fx[i];
         for ( int j = 0; j < 3; ++j ) DF[9 * p + 3 * i + j] = D( i, j );
      }
   }
   return 0;
}
