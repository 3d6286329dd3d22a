// Data export and checkpoints around the solver path, host side with device-to-host staging:
//  * VTK: the reference's VTKOutput (dataexport/VTKOutput/VTKOutput.hpp:44-139, VTKOutput.cpp:160-230)
//    writes one XML UnstructuredGrid file per DoF type and write call,
//    <dir>/<filename>_<type>_level<L>_ts<T>.vtu; per macro-cell the micro-vertices of the level (P2: of
//    level + 1) at their blended positions, the micro-tetrahedra of the level (P2: as ten-node
//    quadratic tetrahedra), and every added function as point data; ASCII or inline base64 binary.
//  * Checkpoints: the reference stores registered functions for a level range through ADIOS2
//    (checkpointrestore/CheckpointExporter.hpp:26-60, ADIOS2/AdiosCheckpointImporter.hpp:97-170);
//    ADIOS2 is not available here, so a checkpoint is one binary file of this library's own format:
//    a header naming the mesh (primitive counts and a hash of its coordinates and cells), then per
//    function its name, kind, value type, level range and, per level, the packed vector in the
//    reference's per-primitive layout.  Restoring checks name, kind, value type and level range as
//    the reference's importer does.
#include "hyb_internal.hpp"

#include "../../include/hyteg_b200.h"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

extern "C" const hyb::Topology* hyb_internal_topology( const hyb_mesh* m );
extern "C" const hyb::Topology* hyb_internal_fn_topology( const hyb_fn* fn );
extern "C" int64_t              hyb_internal_fn_packed_size( const hyb_fn* fn, int level );
extern "C" void                 hyb_internal_set_error( const char* msg );

using namespace hyb;

#define HYB_X_TRY try {
#define HYB_X_CATCH                                                                                                            \
   }                                                                                                                           \
   catch ( const std::invalid_argument& e )                                                                                    \
   {                                                                                                                           \
      hyb_internal_set_error( e.what() );                                                                                      \
      return HYB_EINVAL;                                                                                                       \
   }                                                                                                                           \
   catch ( const std::bad_alloc& )                                                                                             \
   {                                                                                                                           \
      hyb_internal_set_error( "out of host memory" );                                                                          \
      return HYB_ENOMEM;                                                                                                       \
   }                                                                                                                           \
   catch ( const std::exception& e )                                                                                           \
   {                                                                                                                           \
      hyb_internal_set_error( e.what() );                                                                                      \
      return HYB_EDEVICE;                                                                                                      \
   }                                                                                                                           \
   return HYB_OK;

namespace {

void need( bool cond, const std::string& msg )
{
   if ( !cond ) throw std::invalid_argument( msg );
}

void rc_ok( int rc )
{
   if ( rc != HYB_OK ) throw std::runtime_error( hyb_last_error() );
}

// ------------------------------------------------------------------------------------------ VTK
// micro-cell types of a level: vertex offsets from the anchor, anchors x + y + z <= n - 1 - shift
// (the six types of the uniform refinement, CellDoFIndexing.hpp:155-198)
const int kMicro[6][4][3] = { { { 0, 0, 0 }, { 1, 0, 0 }, { 0, 1, 0 }, { 0, 0, 1 } }, { { 1, 0, 0 }, { 1, 1, 0 }, { 0, 1, 0 }, { 1, 0, 1 } },
                              { { 1, 0, 0 }, { 0, 1, 0 }, { 1, 0, 1 }, { 0, 0, 1 } }, { { 1, 1, 0 }, { 1, 1, 1 }, { 0, 1, 1 }, { 1, 0, 1 } },
                              { { 1, 0, 1 }, { 0, 1, 1 }, { 0, 0, 1 }, { 0, 1, 0 } }, { { 0, 1, 0 }, { 1, 1, 0 }, { 1, 0, 1 }, { 0, 1, 1 } } };
const int kMicroShift[6] = { 0, 1, 1, 2, 1, 1 };
// node pairs of the six edges in the order of VTK's quadratic tetrahedron (nodes 4-9)
const int kQuadEdge[6][2] = { { 0, 1 }, { 1, 2 }, { 0, 2 }, { 0, 3 }, { 1, 3 }, { 2, 3 } };

// IcosahedralShellMap F(x) = x R(x) / |x|, R = r_ray + |lambda| (r_ref - r_ray), lambda the barycentric
// weight of the ref vertex (the position part of the device map used by the elementwise operators)
void shell_point( const CellGeom& g, const double* X, double* F )
{
   const double lam = ( ( X[0] - g.ray[0] ) * g.bxc[0] + ( X[1] - g.ray[1] ) * g.bxc[1] + ( X[2] - g.ray[2] ) * g.bxc[2] ) / g.volT;
   const double R   = g.rad_ray + std::fabs( lam ) * ( g.rad_ref - g.rad_ray );
   const double r   = std::sqrt( X[0] * X[0] + X[1] * X[1] + X[2] * X[2] );
   for ( int d = 0; d < 3; ++d ) F[d] = X[d] * R / r;
}

// base64 of a byte run (RFC 4648, with padding)
void base64( std::ostream& os, const unsigned char* p, size_t n )
{
   static const char tab[] = "ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789+/";
   std::string       out;
   out.reserve( ( n + 2 ) / 3 * 4 );
   size_t i = 0;
   for ( ; i + 2 < n; i += 3 )
   {
      const uint32_t v = ( uint32_t( p[i] ) << 16 ) | ( uint32_t( p[i + 1] ) << 8 ) | p[i + 2];
      out += tab[v >> 18], out += tab[( v >> 12 ) & 63], out += tab[( v >> 6 ) & 63], out += tab[v & 63];
   }
   if ( i < n )
   {
      const uint32_t v = ( uint32_t( p[i] ) << 16 ) | ( i + 1 < n ? uint32_t( p[i + 1] ) << 8 : 0u );
      out += tab[v >> 18], out += tab[( v >> 12 ) & 63];
      out += i + 1 < n ? tab[( v >> 6 ) & 63] : '=';
      out += '=';
   }
   os << out;
}

// one DataArray: ASCII values, or VTK's inline binary (base64 of a 32-bit byte count followed by the
// little-endian values); 64-bit counts where a block exceeds 4 GiB are not supported by that header
template < typename V >
void data_array( std::ostream& os, const char* type, const std::string& name, int ncomp, const std::vector< V >& v, bool binary )
{
   os << "<DataArray type=\"" << type << "\"";
   if ( !name.empty() ) os << " Name=\"" << name << "\"";
   if ( ncomp > 0 ) os << " NumberOfComponents=\"" << ncomp << "\"";
   os << " format=\"" << ( binary ? "binary" : "ascii" ) << "\">\n";
   if ( binary )
   {
      const size_t bytes = v.size() * sizeof( V );
      if ( bytes > 0xffffffffull ) throw std::invalid_argument( "VTK binary block larger than 4 GiB; use the ASCII format" );
      std::vector< unsigned char > buf( 4 + bytes );
      const uint32_t               h = uint32_t( bytes );
      std::memcpy( buf.data(), &h, 4 );
      if ( bytes ) std::memcpy( buf.data() + 4, v.data(), bytes );
      base64( os, buf.data(), buf.size() );
      os << "\n";
   }
   else
   {
      char   tmp[40];
      size_t k = 0;
      for ( const V& x : v )
      {
         if constexpr ( std::is_same< V, double >::value ) std::snprintf( tmp, sizeof( tmp ), "%.17g", x );
         else if constexpr ( std::is_same< V, float >::value ) std::snprintf( tmp, sizeof( tmp ), "%.9g", double( x ) );
         else std::snprintf( tmp, sizeof( tmp ), "%lld", (long long) x );
         os << tmp << ( ++k % 12 == 0 ? '\n' : ' ' );
      }
      os << "\n";
   }
   os << "</DataArray>\n";
}

struct Field
{
   std::string           name;
   int                   dtype;  // HYB_F64: Float64; HYB_F32 / HYB_F16: Float32
   const double*         packed; // packed reference layout of the storage level
};

// the file of one DoF type (order 1: P1 "VertexDoF", order 2: "P2") at `level`
void write_vtu( const Topology& t, const std::vector< int64_t >& cell_off, const std::string& path, int level, int order, int blending,
                bool binary, const std::vector< Field >& fields )
{
   const int     n   = 1 << level;              // micro-cells per macro-edge
   const int     N   = order == 2 ? 2 * n : n;  // point grid (the storage level)
   const int64_t ppc = tet_size( N + 1 );       // points per macro-cell
   const int64_t cpc = int64_t( n ) * n * n;    // micro-cells per macro-cell
   const int64_t np = ppc * t.nC, nc = cpc * t.nC;
   std::ofstream os( path, std::ios::out | std::ios::trunc );
   if ( !os ) throw std::runtime_error( "cannot open " + path );
   os << "<?xml version=\"1.0\"?>\n<VTKFile type=\"UnstructuredGrid\" version=\"0.1\" byte_order=\"LittleEndian\">\n<UnstructuredGrid>\n";
   os << "<Piece NumberOfPoints=\"" << np << "\" NumberOfCells=\"" << nc << "\">\n";
   // points: per macro-cell its grid in storage order (x fastest, then y, then z), blended
   {
      std::vector< double > pts( size_t( np ) * 3 );
      for ( int c = 0; c < t.nC; ++c )
      {
         CellGeom g;
         cell_geometry( t, c, blending, g );
         for ( int z = 0; z <= N; ++z )
            for ( int y = 0; y + z <= N; ++y )
               for ( int x = 0; x + y + z <= N; ++x )
               {
                  double X[3], F[3];
                  for ( int d = 0; d < 3; ++d )
                     X[d] = g.P[0][d] + ( ( g.P[1][d] - g.P[0][d] ) * x + ( g.P[2][d] - g.P[0][d] ) * y + ( g.P[3][d] - g.P[0][d] ) * z ) / N;
                  if ( blending == HYB_BLEND_SHELL ) shell_point( g, X, F );
                  else std::memcpy( F, X, sizeof( X ) );
                  std::memcpy( &pts[size_t( ppc * c + cidx( N, x, y, z ) ) * 3], F, sizeof( F ) );
               }
      }
      os << "<Points>\n";
      data_array( os, "Float64", "", 3, pts, binary );
      os << "</Points>\n";
   }
   // cells: the micro-tetrahedra of the level, type by type, anchors in storage order
   {
      const int            nv = order == 2 ? 10 : 4;
      std::vector< int64_t > conn, offs;
      conn.reserve( size_t( nc ) * nv );
      offs.reserve( size_t( nc ) );
      for ( int c = 0; c < t.nC; ++c )
         for ( int ty = 0; ty < 6; ++ty )
            for ( int z = 0; z <= n - 1 - kMicroShift[ty]; ++z )
               for ( int y = 0; y + z <= n - 1 - kMicroShift[ty]; ++y )
                  for ( int x = 0; x + y + z <= n - 1 - kMicroShift[ty]; ++x )
                  {
                     const int s = order == 2 ? 2 : 1;
                     int       V[4][3];
                     for ( int k = 0; k < 4; ++k )
                     {
                        V[k][0] = s * ( x + kMicro[ty][k][0] ), V[k][1] = s * ( y + kMicro[ty][k][1] ), V[k][2] = s * ( z + kMicro[ty][k][2] );
                        conn.push_back( ppc * c + cidx( N, V[k][0], V[k][1], V[k][2] ) );
                     }
                     if ( order == 2 )
                        for ( const auto& e : kQuadEdge )
                           conn.push_back( ppc * c + cidx( N, ( V[e[0]][0] + V[e[1]][0] ) / 2, ( V[e[0]][1] + V[e[1]][1] ) / 2,
                                                           ( V[e[0]][2] + V[e[1]][2] ) / 2 ) );
                     offs.push_back( int64_t( conn.size() ) );
                  }
      if ( int64_t( offs.size() ) != nc ) throw std::logic_error( "VTK: micro-cell count" );
      std::vector< uint8_t > types( static_cast< size_t >( nc ), uint8_t( order == 2 ? 24 : 10 ) );
      os << "<Cells>\n";
      data_array( os, "Int64", "connectivity", 0, conn, binary );
      data_array( os, "Int64", "offsets", 0, offs, binary );
      data_array( os, "UInt8", "types", 0, types, binary );
      os << "</Cells>\n";
   }
   // point data: each macro-cell's array of every function (the cell arrays hold the values of the
   // cell's faces, edges and vertices as well)
   os << "<PointData>\n";
   for ( const Field& f : fields )
   {
      if ( f.dtype == HYB_F64 )
      {
         std::vector< double > v( static_cast< size_t >( np ) );
         for ( int c = 0; c < t.nC; ++c ) std::memcpy( &v[size_t( ppc * c )], f.packed + cell_off[c], size_t( ppc ) * sizeof( double ) );
         data_array( os, "Float64", f.name, 1, v, binary );
      }
      else
      {
         std::vector< float > v( static_cast< size_t >( np ) );
         for ( int c = 0; c < t.nC; ++c )
            for ( int64_t i = 0; i < ppc; ++i ) v[size_t( ppc * c + i )] = float( f.packed[cell_off[c] + i] );
         data_array( os, "Float32", f.name, 1, v, binary );
      }
   }
   os << "</PointData>\n</Piece>\n</UnstructuredGrid>\n</VTKFile>\n";
   if ( !os ) throw std::runtime_error( "write failed: " + path );
}

// packed offsets of the macro-cells at storage level Ls
std::vector< int64_t > cell_offsets( hyb_mesh* mesh, const Topology& t, int Ls )
{
   const int              np = t.nV + t.nE + t.nF + t.nC;
   std::vector< int64_t > off( np ), sz( np );
   rc_ok( hyb_layout_primitive_offsets( mesh, Ls, off.data(), sz.data() ) );
   return std::vector< int64_t >( off.begin() + ( np - t.nC ), off.end() );
}

std::string type_name( int order ) { return order == 2 ? "P2" : "VertexDoF"; }

}  // namespace

struct hyb_vtk
{
   hyb_mesh*                  mesh = nullptr;
   std::string                dir, filename;
   int                        frequency = 1;
   int                        blending  = HYB_BLEND_NONE;
   bool                       binary    = false;
   std::vector< hyb_fn* >     fns;
   std::vector< std::string > names;
};

extern "C" {

int hyb_vtk_create( hyb_mesh* mesh, const char* dir, const char* filename, int write_frequency, hyb_vtk** out )
{
   HYB_X_TRY
   need( mesh && dir && filename && out, "NULL argument" );
   need( write_frequency >= 0, "negative write frequency" );
   auto* w      = new hyb_vtk();
   w->mesh      = mesh;
   w->dir       = dir;
   w->filename  = filename;
   w->frequency = write_frequency;
   *out         = w;
   HYB_X_CATCH
}

int hyb_vtk_destroy( hyb_vtk* w )
{
   delete w;
   return HYB_OK;
}

int hyb_vtk_set_blending( hyb_vtk* w, int blending )
{
   HYB_X_TRY
   need( w, "NULL argument" );
   need( blending == HYB_BLEND_NONE || blending == HYB_BLEND_SHELL, "unknown blending" );
   w->blending = blending;
   HYB_X_CATCH
}

int hyb_vtk_set_parameter( hyb_vtk* w, const char* key, const char* value )
{
   HYB_X_TRY
   need( w && key && value, "NULL argument" );
   need( std::string( key ) == "vtkDataFormat", std::string( "VTKOutput does not support key '" ) + key + "'" );
   const std::string v = value;
   need( v == "ASCII" || v == "BINARY", "vtkDataFormat '" + v + "' is not supported" );
   w->binary = v == "BINARY";
   HYB_X_CATCH
}

int hyb_vtk_add( hyb_vtk* w, hyb_fn* fn, const char* name )
{
   HYB_X_TRY
   need( w && fn && name, "NULL argument" );
   for ( size_t i = 0; i < w->fns.size(); ++i ) need( w->fns[i] != fn, "function already added" );
   w->fns.push_back( fn );
   w->names.push_back( name );
   HYB_X_CATCH
}

int hyb_vtk_remove( hyb_vtk* w, hyb_fn* fn )
{
   HYB_X_TRY
   need( w && fn, "NULL argument" );
   for ( size_t i = 0; i < w->fns.size(); ++i )
      if ( w->fns[i] == fn )
      {
         w->fns.erase( w->fns.begin() + long( i ) );
         w->names.erase( w->names.begin() + long( i ) );
         return HYB_OK;
      }
   need( false, "function was not added" );
   HYB_X_CATCH
}

int hyb_vtk_write( hyb_vtk* w, int level, int timestep )
{
   HYB_X_TRY
   need( w, "NULL argument" );
   need( level >= 0 && timestep >= 0, "negative level or time step" );
   if ( w->frequency == 0 || timestep % w->frequency != 0 ) return HYB_OK;
   const Topology* t = hyb_internal_topology( w->mesh );
   for ( int order = 1; order <= 2; ++order )
   {
      std::vector< std::vector< double > > data;
      std::vector< Field >                 fields;
      for ( size_t i = 0; i < w->fns.size(); ++i )
      {
         int o = 0, dt = 0, lo = 0, hi = 0;
         rc_ok( hyb_fn_info( w->fns[i], &o, &dt, &lo, &hi ) );
         if ( o != order ) continue;
         need( level >= lo && level <= hi, "function '" + w->names[i] + "' has no level " + std::to_string( level ) );
         int64_t cnt = 0;
         rc_ok( hyb_layout_packed_size( w->mesh, level + order - 1, &cnt ) );
         data.emplace_back( size_t( cnt ) );
         rc_ok( hyb_fn_download( w->fns[i], level, data.back().data() ) );
         fields.push_back( Field{ w->names[i], dt, nullptr } );
      }
      if ( fields.empty() ) continue;
      for ( size_t i = 0; i < fields.size(); ++i ) fields[i].packed = data[i].data();
      const std::string path = w->dir + "/" + w->filename + "_" + type_name( order ) + "_level" + std::to_string( level ) + "_ts" +
                               std::to_string( timestep ) + ".vtu";
      write_vtu( *t, cell_offsets( w->mesh, *t, level + order - 1 ), path, level, order, w->blending, w->binary, fields );
   }
   HYB_X_CATCH
}

int hyb_vtk_write_packed( hyb_mesh* mesh, const char* path, int level, int order, int blending, int binary, int nfields,
                          const char* const* names, const int* dtypes, const double* const* packed )
{
   HYB_X_TRY
   need( mesh && path && ( nfields == 0 || ( names && dtypes && packed ) ), "NULL argument" );
   need( order == 1 || order == 2, "order must be 1 or 2" );
   need( level >= 0 && level <= 12, "invalid level" );
   need( blending == HYB_BLEND_NONE || blending == HYB_BLEND_SHELL, "unknown blending" );
   std::vector< Field > fields;
   for ( int i = 0; i < nfields; ++i )
   {
      need( names[i] && packed[i], "NULL field" );
      need( dtypes[i] == HYB_F64 || dtypes[i] == HYB_F32 || dtypes[i] == HYB_F16, "unknown value type" );
      fields.push_back( Field{ names[i], dtypes[i], packed[i] } );
   }
   const Topology* t = hyb_internal_topology( mesh );
   write_vtu( *t, cell_offsets( mesh, *t, level + order - 1 ), path, level, order, blending, binary != 0, fields );
   HYB_X_CATCH
}

}  // extern "C"

// ------------------------------------------------------------------------------------------ checkpoints
namespace {

const char     kMagic[8]       = { 'H', 'Y', 'B', 'C', 'K', 'P', 'T', '1' };
const uint32_t kFormatVersion = 1;

// FNV-1a over the mesh's coordinates and cell vertex ids: a checkpoint is restored only on the mesh
// it was written from
uint64_t mesh_hash( const Topology& t )
{
   uint64_t h   = 1469598103934665603ull;
   auto     mix = [&]( const void* p, size_t n ) {
      const unsigned char* b = static_cast< const unsigned char* >( p );
      for ( size_t i = 0; i < n; ++i ) h = ( h ^ b[i] ) * 1099511628211ull;
   };
   for ( const auto& v : t.vx ) mix( v.data(), sizeof( double ) * 3 );
   for ( const auto& c : t.cv ) mix( c.data(), sizeof( int ) * 4 );
   return h;
}

const char* value_type_name( int dt ) { return dt == HYB_F64 ? "double" : dt == HYB_F32 ? "float" : "float16"; }

struct Writer
{
   std::ofstream os;
   void          bytes( const void* p, size_t n ) { os.write( static_cast< const char* >( p ), std::streamsize( n ) ); }
   template < typename V >
   void pod( const V& v )
   {
      bytes( &v, sizeof( V ) );
   }
   void str( const std::string& s )
   {
      pod( uint32_t( s.size() ) );
      bytes( s.data(), s.size() );
   }
};

struct Reader
{
   std::ifstream is;
   std::string   path;
   void          bytes( void* p, size_t n )
   {
      is.read( static_cast< char* >( p ), std::streamsize( n ) );
      if ( !is ) throw std::invalid_argument( "checkpoint " + path + " is truncated" );
   }
   template < typename V >
   V pod()
   {
      V v;
      bytes( &v, sizeof( V ) );
      return v;
   }
   std::string str()
   {
      const uint32_t n = pod< uint32_t >();
      if ( n > ( 1u << 20 ) ) throw std::invalid_argument( "checkpoint " + path + " is corrupt" );
      std::string s( n, '\0' );
      bytes( &s[0], n );
      return s;
   }
};

std::string ckpt_path( const char* dir, const char* filename ) { return std::string( dir ) + "/" + filename + ".hybckpt"; }

struct Entry
{
   std::string name, kind, vtype;
   int         lo = 0, hi = 0;
   std::streampos data;  // first level's count
};

// the header and the function table of a checkpoint (the data are skipped, their offsets kept)
std::vector< Entry > read_table( Reader& r, const Topology* t )
{
   char magic[8];
   r.bytes( magic, 8 );
   if ( std::memcmp( magic, kMagic, 8 ) != 0 ) throw std::invalid_argument( "not a hyteg_b200 checkpoint: " + r.path );
   const uint32_t ver = r.pod< uint32_t >();
   if ( ver != kFormatVersion ) throw std::invalid_argument( "unsupported checkpoint format version " + std::to_string( ver ) );
   int32_t counts[4];
   r.bytes( counts, sizeof( counts ) );
   const uint64_t h = r.pod< uint64_t >();
   if ( t && ( counts[0] != t->nV || counts[1] != t->nE || counts[2] != t->nF || counts[3] != t->nC || h != mesh_hash( *t ) ) )
      throw std::invalid_argument( "checkpoint " + r.path + " was written on a different mesh" );
   const uint32_t       nf = r.pod< uint32_t >();
   std::vector< Entry > out;
   for ( uint32_t i = 0; i < nf; ++i )
   {
      Entry e;
      e.name  = r.str();
      e.kind  = r.str();
      e.vtype = r.str();
      e.lo    = r.pod< int32_t >();
      e.hi    = r.pod< int32_t >();
      if ( e.lo < 0 || e.hi < e.lo || e.hi > 14 ) throw std::invalid_argument( "checkpoint " + r.path + " is corrupt" );
      e.data = r.is.tellg();
      for ( int l = e.lo; l <= e.hi; ++l )
      {
         const int64_t cnt = r.pod< int64_t >();
         if ( cnt < 0 ) throw std::invalid_argument( "checkpoint " + r.path + " is corrupt" );
         r.is.seekg( std::streamoff( cnt ) * std::streamoff( sizeof( double ) ), std::ios::cur );
      }
      out.push_back( e );
   }
   return out;
}

}  // namespace

extern "C" {

int hyb_checkpoint_store( const char* dir, const char* filename, int nfn, hyb_fn* const* fns, const char* const* names, const int* min_levels,
                          const int* max_levels )
{
   HYB_X_TRY
   need( dir && filename && nfn >= 0 && ( nfn == 0 || ( fns && names && min_levels && max_levels ) ), "NULL argument" );
   need( nfn > 0, "no function to store" );
   for ( int i = 0; i < nfn; ++i )
   {
      need( fns[i] && names[i], "NULL function or name" );
      for ( int j = 0; j < i; ++j ) need( std::string( names[i] ) != names[j], std::string( "function name stored twice: " ) + names[i] );
   }
   // every function lives on one mesh, which the header names
   const Topology* t = hyb_internal_fn_topology( fns[0] );
   for ( int i = 1; i < nfn; ++i ) need( hyb_internal_fn_topology( fns[i] ) == t, "functions of one checkpoint must live on one mesh" );
   Writer            w;
   const std::string path = ckpt_path( dir, filename );
   w.os.open( path, std::ios::binary | std::ios::trunc );
   if ( !w.os ) throw std::runtime_error( "cannot open " + path );
   w.bytes( kMagic, 8 );
   w.pod( kFormatVersion );
   const int32_t counts[4] = { t->nV, t->nE, t->nF, t->nC };
   w.bytes( counts, sizeof( counts ) );
   w.pod( mesh_hash( *t ) );
   w.pod( uint32_t( nfn ) );
   for ( int i = 0; i < nfn; ++i )
   {
      int o = 0, dt = 0, lo = 0, hi = 0;
      rc_ok( hyb_fn_info( fns[i], &o, &dt, &lo, &hi ) );
      need( min_levels[i] >= lo && max_levels[i] <= hi && min_levels[i] <= max_levels[i],
            std::string( "level range not held by function " ) + names[i] );
      w.str( names[i] );
      w.str( o == 2 ? "P2Function" : "P1Function" );
      w.str( value_type_name( dt ) );
      w.pod( int32_t( min_levels[i] ) );
      w.pod( int32_t( max_levels[i] ) );
      for ( int l = min_levels[i]; l <= max_levels[i]; ++l )
      {
         const int64_t         cnt = hyb_internal_fn_packed_size( fns[i], l );
         std::vector< double > v( static_cast< size_t >( cnt ) );
         rc_ok( hyb_fn_download( fns[i], l, v.data() ) );
         w.pod( cnt );
         w.bytes( v.data(), v.size() * sizeof( double ) );
      }
   }
   w.os.close();
   if ( !w.os ) throw std::runtime_error( "write failed: " + path );
   HYB_X_CATCH
}

int hyb_checkpoint_function_count( const char* dir, const char* filename, int* count )
{
   HYB_X_TRY
   need( dir && filename && count, "NULL argument" );
   Reader r;
   r.path = ckpt_path( dir, filename );
   r.is.open( r.path, std::ios::binary );
   need( bool( r.is ), "cannot open checkpoint " + r.path );
   *count = int( read_table( r, nullptr ).size() );
   HYB_X_CATCH
}

int hyb_checkpoint_function_info( const char* dir, const char* filename, int index, char* name, int name_cap, char* kind, int kind_cap,
                                  char* value_type, int vtype_cap, int* min_level, int* max_level )
{
   HYB_X_TRY
   need( dir && filename, "NULL argument" );
   Reader r;
   r.path = ckpt_path( dir, filename );
   r.is.open( r.path, std::ios::binary );
   need( bool( r.is ), "cannot open checkpoint " + r.path );
   const auto tab = read_table( r, nullptr );
   need( index >= 0 && index < int( tab.size() ), "function index out of range" );
   const Entry& e    = tab[size_t( index )];
   auto         copy = [&]( char* dst, int cap, const std::string& s ) {
      if ( !dst ) return;
      need( cap > int( s.size() ), "buffer too small" );
      std::memcpy( dst, s.c_str(), s.size() + 1 );
   };
   copy( name, name_cap, e.name );
   copy( kind, kind_cap, e.kind );
   copy( value_type, vtype_cap, e.vtype );
   if ( min_level ) *min_level = e.lo;
   if ( max_level ) *max_level = e.hi;
   HYB_X_CATCH
}

int hyb_checkpoint_restore( const char* dir, const char* filename, hyb_fn* fn, const char* name, int min_level, int max_level )
{
   HYB_X_TRY
   need( dir && filename && fn && name, "NULL argument" );
   need( min_level <= max_level, "min_level > max_level" );
   int o = 0, dt = 0, lo = 0, hi = 0;
   rc_ok( hyb_fn_info( fn, &o, &dt, &lo, &hi ) );
   need( min_level >= lo && max_level <= hi, "the function does not hold the requested levels" );
   Reader r;
   r.path = ckpt_path( dir, filename );
   r.is.open( r.path, std::ios::binary );
   need( bool( r.is ), "cannot open checkpoint " + r.path );
   const auto tab = read_table( r, hyb_internal_fn_topology( fn ) );
   for ( const Entry& e : tab )
   {
      if ( e.name != name ) continue;
      need( e.kind == ( o == 2 ? "P2Function" : "P1Function" ), std::string( name ) + ": stored as " + e.kind );
      need( e.lo <= min_level, std::string( name ) + ": minLevel = " + std::to_string( min_level ) + " not present in checkpoint" );
      need( e.hi >= max_level, std::string( name ) + ": maxLevel = " + std::to_string( max_level ) + " not present in checkpoint" );
      need( e.vtype == value_type_name( dt ),
            std::string( name ) + ": requested valueType = " + value_type_name( dt ) + " not present in checkpoint" );
      r.is.clear();
      r.is.seekg( e.data );
      for ( int l = e.lo; l <= e.hi; ++l )
      {
         const int64_t cnt = r.pod< int64_t >();
         if ( l < min_level || l > max_level )
         {
            r.is.seekg( std::streamoff( cnt ) * std::streamoff( sizeof( double ) ), std::ios::cur );
            continue;
         }
         need( cnt == hyb_internal_fn_packed_size( fn, l ), "checkpoint level size does not match the mesh" );
         std::vector< double > v( static_cast< size_t >( cnt ) );
         r.bytes( v.data(), v.size() * sizeof( double ) );
         rc_ok( hyb_fn_upload( fn, l, v.data() ) );
      }
      return HYB_OK;
   }
   need( false, std::string( "function '" ) + name + "' not present in checkpoint" );
   HYB_X_CATCH
}

}  // extern "C"
