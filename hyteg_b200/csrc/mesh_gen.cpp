// Macro-mesh generators and readers (host).
#include "hyb_internal.hpp"

#include <algorithm>
#include <cmath>
#include <fstream>
#include <map>
#include <sstream>
#include <stdexcept>

namespace hyb {

// MeshInfo::meshCuboid (src/hyteg/mesh/MeshGenCuboid.cpp:35-172): vertices on an
// (nx+1)x(ny+1)x(nz+1) lattice, x fastest, and every sub-cube split into six tetrahedra that all
// share the sub-cube diagonal from corner 3 (0,1,0) to corner 5 (1,0,1).  The split table is the
// reference's, because the tetrahedra and their vertex order define the macro-cell orientation
// and thereby the vertex-DoF layout.
void cuboid( const double* lo, const double* hi, int nx, int ny, int nz, std::vector< std::array< double, 3 > >& coords,
             std::vector< std::array< int, 4 > >& tets )
{
   const double hx = ( hi[0] - lo[0] ) / nx, hy = ( hi[1] - lo[1] ) / ny, hz = ( hi[2] - lo[2] ) / nz;
   coords.clear();
   for ( int iz = 0; iz <= nz; ++iz )
      for ( int iy = 0; iy <= ny; ++iy )
         for ( int ix = 0; ix <= nx; ++ix ) coords.push_back( { lo[0] + ix * hx, lo[1] + iy * hy, lo[2] + iz * hz } );
   static const int corner[8][3] = { { 0, 0, 0 }, { 1, 0, 0 }, { 1, 1, 0 }, { 0, 1, 0 },
                                     { 0, 0, 1 }, { 1, 0, 1 }, { 1, 1, 1 }, { 0, 1, 1 } };
   static const int split[6][4]  = { { 4, 5, 7, 3 }, { 0, 3, 1, 4 }, { 4, 1, 5, 3 },
                                     { 5, 6, 7, 2 }, { 1, 3, 2, 5 }, { 7, 2, 3, 5 } };
   tets.clear();
   for ( int iz = 0; iz < nz; ++iz )
      for ( int iy = 0; iy < ny; ++iy )
         for ( int ix = 0; ix < nx; ++ix )
            for ( const auto& t : split )
            {
               std::array< int, 4 > ids;
               for ( int m = 0; m < 4; ++m )
               {
                  const int* o = corner[t[m]];
                  ids[m]       = ( iz + o[2] ) * ( nx + 1 ) * ( ny + 1 ) + ( iy + o[1] ) * ( nx + 1 ) + ( ix + o[0] );
               }
               tets.push_back( ids );
            }
}

// Gmsh MSH 2.2 / 4.1 ASCII reader for tetrahedral meshes (element type 4).  Node tags are
// mapped to vertex ids in increasing tag order, like MeshInfo's id-keyed vertex map.
int read_gmsh( const std::string& path, std::vector< std::array< double, 3 > >& coords, std::vector< std::array< int, 4 > >& tets )
{
   std::ifstream in( path );
   if ( !in ) throw std::invalid_argument( "cannot open mesh file " + path );
   std::string                                  tok;
   double                                       version = 0;
   std::map< long, std::array< double, 3 > >    nodes;
   std::vector< std::array< long, 4 > >         raw;
   while ( in >> tok )
   {
      if ( tok == "$MeshFormat" )
      {
         int ft, ds;
         in >> version >> ft >> ds;
         if ( ft != 0 ) throw std::invalid_argument( "only ASCII gmsh files are supported" );
      }
      else if ( tok == "$Nodes" )
      {
         if ( version < 4 )
         {
            long n;
            in >> n;
            for ( long i = 0; i < n; ++i )
            {
               long   id;
               double x, y, z;
               in >> id >> x >> y >> z;
               nodes[id] = { x, y, z };
            }
         }
         else
         {
            long nb, nn, mn, mx;
            in >> nb >> nn >> mn >> mx;
            for ( long b = 0; b < nb; ++b )
            {
               int  dim, ent, param;
               long cnt;
               in >> dim >> ent >> param >> cnt;
               std::vector< long > ids( cnt );
               for ( auto& id : ids ) in >> id;
               for ( long i = 0; i < cnt; ++i )
               {
                  double x, y, z;
                  in >> x >> y >> z;
                  nodes[ids[i]] = { x, y, z };
               }
            }
         }
      }
      else if ( tok == "$Elements" )
      {
         if ( version < 4 )
         {
            long n;
            in >> n;
            std::string line;
            std::getline( in, line );
            for ( long i = 0; i < n; ++i )
            {
               std::getline( in, line );
               std::istringstream ls( line );
               long               id, type, ntags;
               ls >> id >> type >> ntags;
               for ( long k = 0; k < ntags; ++k )
               {
                  long t;
                  ls >> t;
               }
               if ( type == 4 )
               {
                  std::array< long, 4 > v;
                  for ( auto& q : v ) ls >> q;
                  raw.push_back( v );
               }
            }
         }
         else
         {
            long nb, ne, mn, mx;
            in >> nb >> ne >> mn >> mx;
            for ( long b = 0; b < nb; ++b )
            {
               int  dim, ent, type;
               long cnt;
               in >> dim >> ent >> type >> cnt;
               const int nv = type == 1 ? 2 : type == 2 ? 3 : type == 4 ? 4 : type == 15 ? 1 : -1;
               if ( nv < 0 ) throw std::invalid_argument( "unsupported gmsh element type" );
               for ( long i = 0; i < cnt; ++i )
               {
                  long id;
                  in >> id;
                  std::array< long, 4 > v{};
                  for ( int k = 0; k < nv; ++k ) in >> v[k];
                  if ( type == 4 ) raw.push_back( v );
               }
            }
         }
      }
   }
   if ( nodes.empty() || raw.empty() ) throw std::invalid_argument( "mesh file holds no tetrahedra: " + path );
   std::map< long, int > idx;
   coords.clear();
   for ( auto& kv : nodes )
   {
      idx[kv.first] = int( coords.size() );
      coords.push_back( kv.second );
   }
   tets.clear();
   for ( auto& r : raw )
   {
      std::array< int, 4 > t;
      for ( int k = 0; k < 4; ++k )
      {
         auto it = idx.find( r[k] );
         if ( it == idx.end() ) throw std::invalid_argument( "element references an unknown node" );
         t[k] = it->second;
      }
      tets.push_back( t );
   }
   return 0;
}

}  // namespace hyb

namespace hyb {

// MeshInfo::meshSphericalShell (src/hyteg/mesh/MeshGenSphericalShell.cpp:642-765, default flavour
// SHELLMESH_CLASSIC): the unit sphere is covered by the ten diamonds of an icosahedron, each
// diamond refined by repeated great-circle midpoints to (ntan-1)^2 quadrilaterals (ntan-1 must be a
// power of two); each quadrilateral times each radial layer gives a prism-like cell split into six
// tetrahedra.  Vertex numbering, the diamond/pole tables and the hemisphere-dependent split tables
// follow the reference because they define the macro mesh (and thereby the vertex-DoF layout).
void spherical_shell( int ntan, const std::vector< double >& layers, std::vector< std::array< double, 3 > >& coords,
                      std::vector< std::array< int, 4 > >& tets )
{
   const int nrad = int( layers.size() );
   if ( nrad < 2 ) throw std::invalid_argument( "spherical shell needs at least two layers" );
   for ( int i = 0; i + 1 < nrad; ++i )
      if ( !( layers[i] < layers[i + 1] ) || !( layers[0] > 0 ) ) throw std::invalid_argument( "layers must be positive and ascending" );
   if ( ntan < 2 || ( ( ntan - 1 ) & ( ntan - 2 ) ) != 0 ) throw std::invalid_argument( "ntan - 1 must be a power of two" );

   // icosahedron nodes: poles and two pentagonal rings
   double       ico[12][3];
   const double fifthpi = 0.4 * std::asin( 1.0 );
   const double w       = 2.0 * std::acos( 1.0 / ( 2.0 * std::sin( fifthpi ) ) );
   const double cosw = std::cos( w ), sinw = std::sin( w );
   ico[0][0] = 0, ico[0][1] = 0, ico[0][2] = 1;
   ico[11][0] = 0, ico[11][1] = 0, ico[11][2] = -1;
   for ( int k = 1; k <= 5; ++k )
   {
      const double phi = 2.0 * ( double( k ) - 0.5 ) * fifthpi;
      ico[k][0] = sinw * std::cos( phi ), ico[k][1] = sinw * std::sin( phi ), ico[k][2] = cosw;
      const double phl = 2.0 * ( double( k ) - 1 ) * fifthpi;
      ico[k + 5][0] = sinw * std::cos( phl ), ico[k + 5][1] = sinw * std::sin( phl ), ico[k + 5][2] = -cosw;
   }
   // diamond corners: pole, then counter-clockwise
   static const int dia[10][4] = { { 0, 5, 6, 1 },   { 0, 1, 7, 2 },  { 0, 2, 8, 3 },  { 0, 3, 9, 4 },  { 0, 4, 10, 5 },
                                   { 11, 7, 1, 6 },  { 11, 8, 2, 7 }, { 11, 9, 3, 8 }, { 11, 10, 4, 9 }, { 11, 6, 5, 10 } };
   const int nt = ntan;
   // unit-sphere node coordinates per diamond, [i1][i2][id][3]
   std::vector< double > nc( size_t( nt ) * nt * 10 * 3, 0.0 );
   auto                  N = [&]( int i1, int i2, int id ) { return &nc[( ( size_t( i1 ) * nt + i2 ) * 10 + id ) * 3]; };
   auto set_mid = [&]( double* out, const double* a, const double* b ) {
      double x = a[0] + b[0], y = a[1] + b[1], z = a[2] + b[2];
      const double scl = std::sqrt( x * x + y * y + z * z );
      out[0] = x / scl, out[1] = y / scl, out[2] = z / scl;
   };
   for ( int id = 0; id < 10; ++id )
   {
      const int L = id < 5 ? 1 : 3, R = id < 5 ? 3 : 1;
      for ( int d = 0; d < 3; ++d )
      {
         N( 0, 0, id )[d]           = ico[dia[id][0]][d];
         N( nt - 1, 0, id )[d]      = ico[dia[id][L]][d];
         N( nt - 1, nt - 1, id )[d] = ico[dia[id][2]][d];
         N( 0, nt - 1, id )[d]      = ico[dia[id][R]][d];
      }
      for ( int m = 1; m < nt - 1; m *= 2 )
      {
         const int l = ( nt - 1 ) / m, l2 = l / 2;
         for ( int j1 = 0; j1 <= m; ++j1 )  // rows
            for ( int j2 = 0; j2 < m; ++j2 )
            {
               const int i1 = j1 * l, i2 = j2 * l + l2;
               set_mid( N( i1, i2, id ), N( i1, i2 - l2, id ), N( i1, i2 + l2, id ) );
            }
         for ( int j1 = 0; j1 <= m; ++j1 )  // columns
            for ( int j2 = 0; j2 < m; ++j2 )
            {
               const int i1 = j2 * l + l2, i2 = j1 * l;
               set_mid( N( i1, i2, id ), N( i1 - l2, i2, id ), N( i1 + l2, i2, id ) );
            }
         for ( int j1 = 0; j1 < m; ++j1 )  // diagonals
            for ( int j2 = 0; j2 < m; ++j2 )
            {
               const int i1 = j1 * l + l2, i2 = j2 * l + l2;
               set_mid( N( i1, i2, id ), N( i1 - l2, i2 + l2, id ), N( i1 + l2, i2 - l2, id ) );
            }
      }
   }
   // vertices: 2*nrad poles first (north per layer, then south per layer), then per layer, diamond,
   // is2 in 1..nt-1, is1 in 0..nt-2
   const int nverts = ( 10 * ( nt - 1 ) * ( nt - 1 ) + 2 ) * nrad;
   coords.assign( nverts, { 0, 0, 0 } );
   for ( int v = 0; v < nverts; ++v )
   {
      int is1, is2, id, ir;
      if ( v >= 2 * nrad )
      {
         int idx = v - 2 * nrad;
         ir      = idx / ( 10 * ( nt - 1 ) * ( nt - 1 ) );
         idx -= ir * 10 * ( nt - 1 ) * ( nt - 1 );
         id = idx / ( ( nt - 1 ) * ( nt - 1 ) );
         idx -= id * ( nt - 1 ) * ( nt - 1 );
         is2 = idx / ( nt - 1 ) + 1;
         is1 = idx % ( nt - 1 );
      }
      else if ( v < nrad ) is1 = 0, is2 = 0, id = 0, ir = v;
      else is1 = 0, is2 = 0, id = 5, ir = v - nrad;
      const double* p = N( is1, is2, id );
      coords[v]       = { p[0] * layers[ir], p[1] * layers[ir], p[2] * layers[ir] };
   }
   auto vidx = [&]( int is1, int is2, int id, int ir ) {
      if ( is1 == 0 && is2 == 0 ) return id < 5 ? ir : nrad + ir;
      if ( is2 == 0 )
      {
         is2 = is1;
         is1 = 0;
         id  = id < 5 ? ( id + 4 ) % 5 : ( id + 4 ) % 5 + 5;
      }
      else if ( is1 == nt - 1 )
      {
         is1 = ( nt - 1 ) - is2;
         is2 = nt - 1;
         id  = id < 5 ? ( id + 4 ) % 5 + 5 : id % 5;
      }
      return ir * ( nt - 1 ) * ( nt - 1 ) * 10 + id * ( nt - 1 ) * ( nt - 1 ) + ( is2 - 1 ) * ( nt - 1 ) + is1 + 2 * nrad;
   };
   static const int off[8][3]   = { { 0, 0, 1 }, { 1, 0, 1 }, { 1, 1, 1 }, { 0, 1, 1 }, { 0, 0, 0 }, { 1, 0, 0 }, { 1, 1, 0 }, { 0, 1, 0 } };
   static const int north[6][4] = { { 0, 1, 3, 7 }, { 4, 7, 5, 0 }, { 0, 5, 1, 7 }, { 1, 2, 3, 6 }, { 5, 7, 6, 1 }, { 3, 6, 7, 1 } };
   static const int south[6][4] = { { 4, 7, 5, 1 }, { 0, 1, 3, 4 }, { 4, 3, 7, 1 }, { 7, 6, 5, 2 }, { 3, 1, 2, 7 }, { 5, 2, 1, 7 } };
   tets.clear();
   const int nel = ( nt - 1 ) * ( nt - 1 ) * ( nrad - 1 ) * 10 * 6;
   for ( int e = 0; e < nel; ++e )
   {
      int idx = e;
      const int ir = idx / ( 60 * ( nt - 1 ) * ( nt - 1 ) );
      idx -= ir * 60 * ( nt - 1 ) * ( nt - 1 );
      const int id = idx / ( 6 * ( nt - 1 ) * ( nt - 1 ) );
      idx -= id * 6 * ( nt - 1 ) * ( nt - 1 );
      const int is2 = idx / ( 6 * ( nt - 1 ) );
      idx -= is2 * 6 * ( nt - 1 );
      const int is1 = idx / 6;
      const int it  = idx - 6 * is1;
      int       vk[8];
      for ( int k = 0; k < 8; ++k )
      {
         const int ks1 = is1 + ( id <= 4 ? off[k][0] : off[k][1] );
         const int ks2 = is2 + ( id <= 4 ? off[k][1] : off[k][0] );
         vk[k]         = vidx( ks1, ks2, id, ir + off[k][2] );
      }
      const int( *tab )[4] = id <= 4 ? north : south;
      tets.push_back( { vk[tab[it][0]], vk[tab[it][1]], vk[tab[it][2]], vk[tab[it][3]] } );
   }
}

}  // namespace hyb
