// A HyTeG-style C++ caller of the B200 path, compiled against include/hyteg_b200.hpp and linked with
// hyteg_b200/libhyteg_b200.so.  It follows the shape of the reference's convergence tests
// (tests/hyteg/convergence/P1GMG3DConvergenceTest.cpp): unit cube of six macro-tetrahedra, P1
// Laplacian, an interpolated right-hand side, V(2,2) weighted-Jacobi cycles with a CG coarse solve.
//
// usage: gmg_apply <output directory> <level>
// writes  y.bin       A x (flag Inner) in the packed layout, doubles, x = u(x, y, z) below
//         y32.bin     the same apply with FP32 storage, converted to doubles
//         x32.bin     its input as stored in FP32, converted to doubles
//         hist.txt    residual norms ||r_0|| .. ||r_6|| of six V(2,2) cycles for b = f(x, y, z)
//         gmg_VertexDoF_level<level>_ts0.vtu   x and y written by VTKOutput (binary)
#include <cmath>
#include <cstdio>
#include <fstream>
#include <string>

#include "hyteg_b200.hpp"

using namespace hyteg;

static double u( const double* p ) { return std::sin( 3.0 * p[0] ) * std::cos( 2.0 * p[1] ) + p[2] * p[2]; }
static double f( const double* p ) { return std::cos( p[0] + 2.0 * p[1] ) * std::exp( p[2] ); }

static void write( const std::string& path, const std::vector< double >& v )
{
   std::ofstream o( path, std::ios::binary );
   o.write( reinterpret_cast< const char* >( v.data() ), std::streamsize( v.size() * sizeof( double ) ) );
}

int main( int argc, char** argv )
{
   if ( argc < 3 )
   {
      std::fprintf( stderr, "usage: %s <output directory> <level>\n", argv[0] );
      return 2;
   }
   const std::string dir   = argv[1];
   const int         level = std::stoi( argv[2] );
   try
   {
      b200::Context    ctx( 0 );
      PrimitiveStorage storage = PrimitiveStorage::cuboid( ctx, { 0, 0, 0 }, { 1, 1, 1 }, 1, 1, 1 );
      const int64_t    packed  = storage.packedSize( level );

      P1ConstantLaplaceOperator A( ctx, storage, 0, level );
      P1Function< double >      x( "x", ctx, storage, 0, level ), y( "y", ctx, storage, 0, level );
      x.interpolate( u, level, All );
      A.apply( x, y, level, Inner, Replace );
      write( dir + "/y.bin", y.download( level, packed ) );
      {
         VTKOutput vtk( dir, "gmg", storage );
         vtk.add( x );
         vtk.add( y );
         vtk.setParameter( "vtkDataFormat", "BINARY" );
         vtk.write( level );
      }

      P1Function< float > x32( "x32", ctx, storage, 0, level ), y32( "y32", ctx, storage, 0, level );
      x32.copyFrom( x, level );
      A.apply( x32, y32, level, Inner, Replace );
      P1Function< double > back( "back", ctx, storage, 0, level );
      back.copyFrom( y32, level );
      write( dir + "/y32.bin", back.download( level, packed ) );
      back.copyFrom( x32, level );
      write( dir + "/x32.bin", back.download( level, packed ) );

      P1Function< double > xs( "xs", ctx, storage, 0, level ), b( "b", ctx, storage, 0, level );
      b.interpolate( f, level, Inner );
      hyb_gmg_params p = GeometricMultigridSolver< P1ConstantLaplaceOperator >::defaultParameters();
      p.min_level = 0;
      p.max_level = level;
      p.pre_smooth = p.post_smooth = 2;
      p.smoother                   = HYB_SMOOTHER_JACOBI;
      p.jacobi_relax               = 2.0 / 3.0;
      GeometricMultigridSolver< P1ConstantLaplaceOperator > gmg( ctx, A, p );
      const std::vector< double > hist = gmg.solveCycles( xs, b, level, 6, 0.0 );
      std::ofstream h( dir + "/hist.txt" );
      h.precision( 17 );
      for ( double r : hist ) h << r << "\n";

      // errors reach the handler instead of aborting: an apply on a level outside the operator's range
      bool caught = false;
      try
      {
         A.apply( x, y, level + 1, Inner );
      } catch ( const b200::Error& e )
      {
         caught = e.status == HYB_EINVAL;
      }
      if ( !caught )
      {
         std::fprintf( stderr, "an invalid level was not reported\n" );
         return 1;
      }
   } catch ( const std::exception& e )
   {
      std::fprintf( stderr, "%s\n", e.what() );
      return 1;
   }
   std::printf( "ok\n" );
   return 0;
}
