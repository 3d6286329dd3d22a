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
