// Macro-mesh topology with HyTeG's primitive order and local orientations, mesh generators,
// and the per-level P1 layout tables.
//
// Ordering rules restated from the reference:
//  * MeshInfo::addEdge / addFace (src/hyteg/mesh/MeshInfo.cpp) store edges and faces under their
//    sorted vertex ids; cells keep the vertex order given by the mesh and are kept in a map keyed
//    by that vertex list.
//  * SetupPrimitiveStorage (src/hyteg/primitivestorage/SetupPrimitiveStorage.cpp:130-412) creates
//    primitive ids vertex -> edge -> face -> cell in that map order.  A face's vertex order follows
//    its first two edges, which for sorted edges is the sorted order.  Cell local edges are
//    (01, 02, 12, 03, 13, 23) and local faces (012, 013, 023, 123) (:305-315).
//  * setMeshBoundaryFlagsOnBoundary / onBoundary (:977-988, :1092-1150): a face is on the
//    boundary if it has one neighbour cell, an edge or a vertex if a neighbouring face is.
#include "hyb_internal.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <fstream>
#include <queue>
#include <set>
#include <sstream>
#include <stdexcept>

namespace hyb {

const int kDirs[kNumDirs][3] = { { 0, 0, 0 },  { -1, 0, 0 }, { 1, 0, 0 },  { 0, -1, 0 }, { 0, 1, 0 },
                                 { 0, 0, -1 }, { 0, 0, 1 },  { -1, 1, 0 }, { 1, -1, 0 }, { -1, 0, 1 },
                                 { 1, 0, -1 }, { 0, -1, 1 }, { 0, 1, -1 }, { 1, -1, 1 }, { -1, 1, -1 } };

static bool dir_ok_for_faces( int faces, const int* d )
{
   if ( ( faces & 1 ) && d[2] < 0 ) return false;                    // face 012: z = 0
   if ( ( faces & 2 ) && d[1] < 0 ) return false;                    // face 013: y = 0
   if ( ( faces & 4 ) && d[0] < 0 ) return false;                    // face 023: x = 0
   if ( ( faces & 8 ) && d[0] + d[1] + d[2] > 0 ) return false;      // face 123: x+y+z = n
   return true;
}

static std::array< uint16_t, kNumClasses > make_class_masks()
{
   std::array< uint16_t, kNumClasses > m{};
   for ( int c = 0; c < kNumClasses; ++c )
      for ( int d = 0; d < kNumDirs; ++d )
         if ( dir_ok_for_faces( kClassFaces[c], kDirs[d] ) ) m[c] |= uint16_t( 1u << d );
   return m;
}
static const std::array< uint16_t, kNumClasses > g_masks = make_class_masks();
const uint16_t kClassDirMask[kNumClasses] = { g_masks[0],  g_masks[1],  g_masks[2],  g_masks[3], g_masks[4],
                                              g_masks[5],  g_masks[6],  g_masks[7],  g_masks[8], g_masks[9],
                                              g_masks[10], g_masks[11], g_masks[12], g_masks[13], g_masks[14] };

int class_of_point( int n, int x, int y, int z )
{
   const int m = ( z == 0 ) | ( ( y == 0 ) << 1 ) | ( ( x == 0 ) << 2 ) | ( ( x + y + z == n ) << 3 );
   for ( int c = 0; c < kNumClasses; ++c )
      if ( kClassFaces[c] == m ) return c;
   return -1;
}

// ---------------------------------------------------------------------------------------------
void Topology::build( const std::vector< std::array< double, 3 > >& coords, const std::vector< std::array< int, 4 > >& tets )
{
   nV = int( coords.size() );
   vx = coords;
   std::vector< std::array< int, 4 > > cells = tets;
   for ( auto& t : cells )
      for ( int k = 0; k < 4; ++k )
         if ( t[k] < 0 || t[k] >= nV ) throw std::invalid_argument( "tet references a vertex out of range" );
   std::sort( cells.begin(), cells.end() );
   if ( std::adjacent_find( cells.begin(), cells.end() ) != cells.end() ) throw std::invalid_argument( "duplicate tet" );
   std::set< std::array< int, 2 > > es;
   std::set< std::array< int, 3 > > fs;
   for ( auto& c : cells )
   {
      for ( int a = 0; a < 4; ++a )
         for ( int b = a + 1; b < 4; ++b )
         {
            if ( c[a] == c[b] ) throw std::invalid_argument( "degenerate tet (repeated vertex)" );
            es.insert( { std::min( c[a], c[b] ), std::max( c[a], c[b] ) } );
         }
      static const int tri[4][3] = { { 0, 1, 2 }, { 0, 1, 3 }, { 0, 2, 3 }, { 1, 2, 3 } };
      for ( auto& t : tri )
      {
         std::array< int, 3 > f = { c[t[0]], c[t[1]], c[t[2]] };
         std::sort( f.begin(), f.end() );
         fs.insert( f );
      }
   }
   ev.assign( es.begin(), es.end() );
   fv.assign( fs.begin(), fs.end() );
   cv = cells;
   nE = int( ev.size() );
   nF = int( fv.size() );
   nC = int( cv.size() );
   std::map< std::array< int, 2 >, int > eid;
   std::map< std::array< int, 3 >, int > fid;
   for ( int i = 0; i < nE; ++i ) eid[ev[i]] = i;
   for ( int i = 0; i < nF; ++i ) fid[fv[i]] = i;
   v_edges.assign( nV, {} );
   v_faces.assign( nV, {} );
   v_cells.assign( nV, {} );
   e_faces.assign( nE, {} );
   e_cells.assign( nE, {} );
   f_cells.assign( nF, {} );
   for ( int i = 0; i < nE; ++i )
   {
      v_edges[ev[i][0]].push_back( i );
      v_edges[ev[i][1]].push_back( i );
   }
   auto E = [&]( int a, int b ) { return eid.at( { std::min( a, b ), std::max( a, b ) } ); };
   for ( int i = 0; i < nF; ++i )
   {
      for ( int k = 0; k < 3; ++k ) v_faces[fv[i][k]].push_back( i );
      e_faces[E( fv[i][0], fv[i][1] )].push_back( i );
      e_faces[E( fv[i][0], fv[i][2] )].push_back( i );
      e_faces[E( fv[i][1], fv[i][2] )].push_back( i );
   }
   ce.assign( nC, {} );
   cf.assign( nC, {} );
   for ( int c = 0; c < nC; ++c )
   {
      const auto& v = cv[c];
      ce[c]         = { E( v[0], v[1] ), E( v[0], v[2] ), E( v[1], v[2] ), E( v[0], v[3] ), E( v[1], v[3] ), E( v[2], v[3] ) };
      auto F        = [&]( int a, int b, int d ) {
         std::array< int, 3 > f = { a, b, d };
         std::sort( f.begin(), f.end() );
         return fid.at( f );
      };
      cf[c] = { F( v[0], v[1], v[2] ), F( v[0], v[1], v[3] ), F( v[0], v[2], v[3] ), F( v[1], v[2], v[3] ) };
      for ( int k = 0; k < 4; ++k ) v_cells[v[k]].push_back( c );
      for ( int k = 0; k < 6; ++k ) e_cells[ce[c][k]].push_back( c );
      for ( int k = 0; k < 4; ++k ) f_cells[cf[c][k]].push_back( c );
   }
   for ( int f = 0; f < nF; ++f )
      if ( f_cells[f].size() > 2 ) throw std::invalid_argument( "non-manifold mesh: face with more than two cells" );
   flag_v.assign( nV, 0 );
   flag_e.assign( nE, 0 );
   flag_f.assign( nF, 0 );
   flag_c.assign( nC, 0 );
   set_boundary_flags_on_boundary( 1, 0 );
}

void Topology::set_boundary_flags_on_boundary( int onBoundary, int inner )
{
   std::vector< char > fb( nF ), eb( nE, 0 ), vb( nV, 0 );
   for ( int f = 0; f < nF; ++f ) fb[f] = f_cells[f].size() == 1;
   for ( int e = 0; e < nE; ++e )
      for ( int f : e_faces[e] ) eb[e] |= fb[f];
   for ( int v = 0; v < nV; ++v )
      for ( int f : v_faces[v] ) vb[v] |= fb[f];
   for ( int v = 0; v < nV; ++v ) flag_v[v] = vb[v] ? onBoundary : inner;
   for ( int e = 0; e < nE; ++e ) flag_e[e] = eb[e] ? onBoundary : inner;
   for ( int f = 0; f < nF; ++f ) flag_f[f] = fb[f] ? onBoundary : inner;
   for ( int c = 0; c < nC; ++c ) flag_c[c] = inner;
}

// ---------------------------------------------------------------------------------------------
// per-level layout tables
// ---------------------------------------------------------------------------------------------
static int local_vertex( const std::array< int, 4 >& cv, int v )
{
   for ( int k = 0; k < 4; ++k )
      if ( cv[k] == v ) return k;
   throw std::logic_error( "vertex not in cell" );
}

static void corner( int k, int8_t* o )
{
   o[0] = k == 1;
   o[1] = k == 2;
   o[2] = k == 3;
}

void build_level( Mesh* m, int L )
{
   const Topology& t  = m->topo;
   auto            lv = std::make_unique< P1Level >();
   P1Level&        P  = *lv;
   P.L                = L;
   const int n        = 1 << L;
   P.n                = n;
   const int nP       = t.nV + t.nE + t.nF + t.nC;
   P.off.resize( nP );
   P.packed_off.resize( nP );
   P.psize.resize( nP );
   int64_t o = 0, po = 0;
   auto    add = [&]( int idx, int64_t s ) {
      P.off[idx]        = o;
      P.packed_off[idx] = po;
      P.psize[idx]      = s;
      o += ( s + 31 ) / 32 * 32;
      po += s;
   };
   for ( int v = 0; v < t.nV; ++v ) add( v, 1 + int64_t( t.v_edges[v].size() ) );
   for ( int e = 0; e < t.nE; ++e )
      add( t.nV + e, ( n + 1 ) + int64_t( t.e_faces[e].size() ) * n + int64_t( t.e_cells[e].size() ) * ( n - 1 ) );
   for ( int f = 0; f < t.nF; ++f ) add( t.nV + t.nE + f, tri_size( n + 1 ) + int64_t( t.f_cells[f].size() ) * tri_size( n ) );
   for ( int c = 0; c < t.nC; ++c ) add( t.nV + t.nE + t.nF + c, tet_size( n + 1 ) );
   P.size        = o;
   P.packed_size = po;

   // incidences of boundary primitives
   P.nB = t.nV + t.nE + t.nF;
   P.inc_begin.assign( P.nB + 1, 0 );
   for ( int v = 0; v < t.nV; ++v )
   {
      P.inc_begin[v] = int( P.inc.size() );
      for ( int c : t.v_cells[v] )
      {
         Incidence I{};
         I.cell = c;
         int k  = local_vertex( t.cv[c], v );
         I.cls  = 11 + k;
         corner( k, I.o );
         P.inc.push_back( I );
      }
   }
   static const int edge_pairs[6][2] = { { 0, 1 }, { 0, 2 }, { 1, 2 }, { 0, 3 }, { 1, 3 }, { 2, 3 } };
   for ( int e = 0; e < t.nE; ++e )
   {
      P.inc_begin[t.nV + e] = int( P.inc.size() );
      for ( int c : t.e_cells[e] )
      {
         Incidence I{};
         I.cell = c;
         int ka = local_vertex( t.cv[c], t.ev[e][0] ), kb = local_vertex( t.cv[c], t.ev[e][1] );
         int le = -1;
         for ( int q = 0; q < 6; ++q )
            if ( ( edge_pairs[q][0] == std::min( ka, kb ) ) && ( edge_pairs[q][1] == std::max( ka, kb ) ) ) le = q;
         I.cls = 5 + le;
         int8_t a[3], b[3];
         corner( ka, a );
         corner( kb, b );
         for ( int d = 0; d < 3; ++d )
         {
            I.o[d]  = a[d];
            I.e1[d] = int8_t( b[d] - a[d] );
         }
         P.inc.push_back( I );
      }
   }
   for ( int f = 0; f < t.nF; ++f )
   {
      P.inc_begin[t.nV + t.nE + f] = int( P.inc.size() );
      for ( int c : t.f_cells[f] )
      {
         Incidence I{};
         I.cell = c;
         int ka = local_vertex( t.cv[c], t.fv[f][0] ), kb = local_vertex( t.cv[c], t.fv[f][1] ),
             kc = local_vertex( t.cv[c], t.fv[f][2] );
         int missing = 6 - ka - kb - kc;
         I.cls       = 1 + ( 3 - missing );  // missing 3 -> face 012 (0), 2 -> 013 (1), 1 -> 023 (2), 0 -> 123 (3)
         int8_t a[3], b[3], cc[3];
         corner( ka, a );
         corner( kb, b );
         corner( kc, cc );
         for ( int d = 0; d < 3; ++d )
         {
            I.o[d]  = a[d];
            I.e1[d] = int8_t( b[d] - a[d] );
            I.e2[d] = int8_t( cc[d] - a[d] );
         }
         P.inc.push_back( I );
      }
   }
   P.inc_begin[P.nB] = int( P.inc.size() );

   // owned DoFs of boundary primitives
   for ( int v = 0; v < t.nV; ++v ) P.tasks.push_back( { v, 0, 0, 0 } );
   for ( int e = 0; e < t.nE; ++e )
      for ( int i = 1; i < n; ++i ) P.tasks.push_back( { t.nV + e, i, 0, 0 } );
   // face DoFs: consecutive tasks step along the cell x direction of one incidence where the face
   // contains it (i fastest if that cell maps face-local i to +-x, j fastest if it maps j), so the
   // boundary sweep reads that cell's array in contiguous runs
   for ( int f = 0; f < t.nF; ++f )
   {
      const int b   = t.nV + t.nE + f;
      bool      jx  = false;
      bool      any = false;
      for ( int q = P.inc_begin[b]; q < P.inc_begin[b + 1] && !any; ++q )
      {
         const Incidence& I = P.inc[q];
         if ( I.e1[1] == 0 && I.e1[2] == 0 ) any = true;
         else if ( I.e2[1] == 0 && I.e2[2] == 0 ) any = true, jx = true;
      }
      if ( jx )
         for ( int i = 1; i < n; ++i )
            for ( int j = 1; i + j < n; ++j ) P.tasks.push_back( { b, i, j, 0 } );
      else
         for ( int j = 1; j < n; ++j )
            for ( int i = 1; i + j < n; ++i ) P.tasks.push_back( { b, i, j, 0 } );
   }
   // y-marching work items (interior points: x, y, z >= 1, x+y+z <= n-1)
   {
      const int YC = 16;
      for ( int z = 1; z <= n - 3; ++z )
         for ( int x0 = 1; x0 <= n - 2 - z; x0 += 32 )
         {
            const int ylast = n - 1 - z - x0;
            for ( int y0 = 1; y0 <= ylast; y0 += YC ) P.march.push_back( { z, x0, y0, std::min( ylast, y0 + YC - 1 ) } );
         }
   }
   // cell interior rows (y, z), memory order
   for ( int z = 1; z <= n - 2; ++z )
      for ( int y = 1; y + z <= n - 2; ++y )
      {
         P.rows.push_back( { y, z } );
         P.n_owned_cell += n - 1 - y - z;
      }

   m->levels[L] = std::move( lv );
}

// Work units of the rolled-register sweep.  A unit is the tile x0..x0+63, y0..y0+kZTileY-1 of slices
// z_first..z_last (interior points only: x, y, z >= 1, x+y+z <= n-1).  The slice range is cut into
// chunks of zc slices, zc the largest power of two in [8, 32] that still gives at least one unit
// per two blocks (every chunk re-reads two halo slices, and every slice load costs a fixed hand-off,
// so long chunks win over finer balance); units are then handed out longest-first to the least
// loaded block.
void build_zunits( P1Level& P, int nblocks, int ncells )
{
   const int n = P.n, kZTileX = 64, kTY = kZTileY;
   auto&     zunits = P.zunits;
   auto&     zcell  = P.zcell;
   auto&     zbegin = P.zbegin;
   zunits.clear();
   zcell.clear();
   zbegin.assign( 1, 0 );
   if ( n < 4 || ncells < 1 ) return;
   struct Unit
   {
      std::array< int, 4 > u;
      int64_t              work;
   };
   auto make = [&]( int zc ) {
      std::vector< Unit > us;
      for ( int y0 = 1; y0 <= n - 3; y0 += kTY )
         for ( int x0 = 1; x0 + y0 <= n - 2; x0 += kZTileX )
         {
            const int zmax = n - 1 - x0 - y0;
            // from slice zh on, every row of the tile ends within its first 32 points (row y0, the
            // longest, has n - y0 - z - x0 interior points from x0 on): those slices form half-width
            // units, run with one point per lane
            const int zh = kZTileX > 32 ? std::max( 1, n - y0 - x0 - 32 ) : zmax + 1;
            for ( int part = 0; part < 2; ++part )
            {
               const int lo = part == 0 ? 1 : std::max( 1, zh ), hi = part == 0 ? std::min( zmax, zh - 1 ) : zmax;
               for ( int za = lo; za <= hi; za += zc )
               {
                  // cost: the slice steps of the unit (its slices plus the two halo slices and the
                  // prologue) times the points per lane; every step issues the whole tile, clipped
                  // lanes included, so the number of interior points would underestimate the units
                  // along the diagonal
                  const int zb = std::min( hi, za + zc - 1 );
                  us.push_back( { { part ? ( x0 | kSwUnitHalf ) : x0, y0, za, zb }, int64_t( zb - za + 3 ) * ( part ? 1 : 2 ) } );
               }
            }
         }
      return us;
   };
   // longest slice ranges that still give every block about two units (all cells together)
   int                 zc = 32;
   std::vector< Unit > us = make( zc );
   while ( zc > 8 && 2 * int64_t( us.size() ) * ncells < int64_t( nblocks ) ) us = make( zc /= 2 );
   std::stable_sort( us.begin(), us.end(), []( const Unit& a, const Unit& b ) { return a.work > b.work; } );
   const int64_t items = int64_t( us.size() ) * ncells;
   const int     nb    = int( std::max< int64_t >( 1, std::min< int64_t >( nblocks, items ) ) );
   std::vector< std::vector< std::pair< int, int > > >                                      per( nb );  // (cell, unit)
   std::priority_queue< std::pair< int64_t, int >, std::vector< std::pair< int64_t, int > >, std::greater<> > heap;
   for ( int b = 0; b < nb; ++b ) heap.push( { 0, b } );
   for ( size_t k = 0; k < us.size(); ++k )  // longest first; the cells of one unit shape in turn
      for ( int c = 0; c < ncells; ++c )
      {
         auto [load, b] = heap.top();
         heap.pop();
         per[b].push_back( { c, int( k ) } );
         heap.push( { load + us[k].work, b } );
      }
   for ( int b = 0; b < nb; ++b )
   {
      // cell-major inside a block: a warp reloads its cell's weights only when the cell changes
      std::stable_sort( per[b].begin(), per[b].end(), []( const auto& a, const auto& b ) { return a.first < b.first; } );
      for ( const auto& cu : per[b] )
      {
         zunits.push_back( us[cu.second].u );
         zcell.push_back( cu.first );
      }
      zbegin.push_back( int( zunits.size() ) );
   }
}

// Work of the cell-interior sweep.  A unit is the tile x0..x0+kSwTX-1, y0..y0+kSwR-1 of the
// slices z_first..z_last of one macro-cell (interior points only: x, y, z >= 1, x+y+z <= n-1).  From
// the slice on which every row of the tile ends within 32 points of x0 the tile is half-width (one
// point per lane).  Each tile column's slice range (full-width and half-width parts separately) is
// cut into equal chunks of at most 32 slices: every chunk reads two halo slices, so longer chunks
// cost fewer re-reads, and 32 slices still give every warp a few units on the level-8 cube.  The
// units of all cells are dealt longest-first to the least loaded of the launch's nwarps warps (cost:
// slice steps, a half-width step counted as 0.6), and each warp's list is ordered by cell, so a warp
// reloads its cell's stencil only when the cell changes.

void build_sweep_units( P1Level& P, int b, int nwarps, int ncells )
{
   const int n     = P.n;
   auto&     units = P.swunits[b];
   auto&     cells = P.swcell[b];
   auto&     begin = P.swbegin[b];
   units.clear();
   cells.clear();
   begin.assign( 1, 0 );
   if ( n < 4 || ncells < 1 || nwarps < 1 ) return;
   struct Unit
   {
      std::array< int, 4 > u;
      double               work;
   };
   std::vector< Unit > us;
   for ( int y0 = 1; y0 <= n - 3; y0 += kSwR )
      for ( int x0 = 1; x0 + y0 <= n - 2; x0 += kSwTX )
      {
         const int zmax = n - 1 - x0 - y0;
         // row y0, the longest of the tile, has n - y0 - z - x0 interior points from x0 on
         const int zh = kSwTX > 32 ? std::max( 1, n - y0 - x0 - 32 ) : zmax + 1;
         for ( int part = 0; part < 2; ++part )
         {
            const int lo = part == 0 ? 1 : zh, hi = part == 0 ? std::min( zmax, zh - 1 ) : zmax;
            if ( hi < lo ) continue;
            const int len = hi - lo + 1, nch = ( len + 31 ) / 32;
            for ( int k = 0; k < nch; ++k )
            {
               const int za = lo + int( int64_t( len ) * k / nch ), zb = lo + int( int64_t( len ) * ( k + 1 ) / nch ) - 1;
               us.push_back( { { part ? ( x0 | kSwUnitHalf ) : x0, y0, za, zb }, double( zb - za + 3 ) * ( part ? 0.6 : 1.0 ) } );
            }
         }
      }
   std::stable_sort( us.begin(), us.end(), []( const Unit& a, const Unit& c ) { return a.work > c.work; } );
   std::vector< std::vector< std::pair< int, int > > > per( nwarps );  // (cell, unit)
   std::priority_queue< std::pair< double, int >, std::vector< std::pair< double, int > >, std::greater<> > heap;
   for ( int w = 0; w < nwarps; ++w ) heap.push( { 0.0, w } );
   for ( size_t k = 0; k < us.size(); ++k )  // longest first; the cells of one unit shape in turn
      for ( int c = 0; c < ncells; ++c )
      {
         auto [load, w] = heap.top();
         heap.pop();
         per[w].push_back( { c, int( k ) } );
         heap.push( { load + us[k].work, w } );
      }
   for ( int w = 0; w < nwarps; ++w )
   {
      std::stable_sort( per[w].begin(), per[w].end(), []( const auto& a, const auto& c ) { return a.first < c.first; } );
      for ( const auto& cu : per[w] )
      {
         units.push_back( us[cu.second].u );
         cells.push_back( cu.first );
      }
      begin.push_back( int( units.size() ) );
   }
}

void ensure_device( Mesh* m, P1Level& P )
{
   if ( P.d_off ) return;
   const Topology& t  = m->topo;
   const int       nP = t.nV + t.nE + t.nF + t.nC;
   auto up = [&]( auto** dptr, const auto* host, size_t count ) {
      using T = std::remove_pointer_t< std::remove_reference_t< decltype( *dptr ) > >;
      size_t bytes = std::max< size_t >( count, 1 ) * sizeof( T );
      check_cuda( cudaMalloc( (void**) dptr, bytes ), "cudaMalloc(level tables)" );
      if ( count ) check_cuda( cudaMemcpy( *dptr, host, count * sizeof( T ), cudaMemcpyHostToDevice ), "upload level tables" );
   };
   up( &P.d_off, P.off.data(), P.off.size() );
   {
      std::vector< int64_t > po( P.packed_off.begin(), P.packed_off.end() );
      po.push_back( P.packed_size );
      up( &P.d_poff, po.data(), po.size() );
   }
   up( &P.d_inc_begin, P.inc_begin.data(), P.inc_begin.size() );
   up( &P.d_inc, P.inc.data(), P.inc.size() );
   std::vector< int4 > tk( P.tasks.size() );
   for ( size_t i = 0; i < tk.size(); ++i ) tk[i] = make_int4( P.tasks[i][0], P.tasks[i][1], P.tasks[i][2], 0 );
   up( &P.d_tasks, tk.data(), tk.size() );
   {
      // the tasks grouped by the boundary type of their primitive (order kept inside a group), so
      // that a stencil operation launches only the groups its flag selects
      const uint32_t      type_bit[4] = { kInner, kDirichlet, kNeumann, kFreeslip };
      std::vector< int4 > bt;
      for ( int g = 0; g < 4; ++g )
      {
         P.bcount[g] = 0;
         for ( const int4& q : tk )
         {
            const int      b  = q.x;
            const uint32_t ty = b < t.nV ? t.bc( t.flag_v[b] )
                                         : ( b < t.nV + t.nE ? t.bc( t.flag_e[b - t.nV] ) : t.bc( t.flag_f[b - t.nV - t.nE] ) );
            if ( ty == type_bit[g] ) bt.push_back( q ), ++P.bcount[g];
         }
      }
      if ( bt.size() != tk.size() ) throw std::logic_error( "boundary task without a single boundary type" );
      up( &P.d_btasks, bt.data(), bt.size() );
      std::vector< FaceRec > fr( bt.size() );
      const int              n = P.n;
      for ( size_t k = 0; k < bt.size(); ++k )
      {
         FaceRec&  r = fr[k];
         const int b = bt[k].x, i = bt[k].y, j = bt[k].z;
         r         = FaceRec{};
         r.cell0   = -1;
         if ( b < t.nV + t.nE || P.inc_begin[b + 1] - P.inc_begin[b] != 2 ) continue;
         r.owner = P.off[b] + fidx( n, i, j );
         r.b     = b;
         r.bc    = uint8_t( t.bc( t.flag_f[b - t.nV - t.nE] ) );
         for ( int s = 0; s < 2; ++s )
         {
            const Incidence& I = P.inc[P.inc_begin[b] + s];
            const int        x = n * I.o[0] + i * I.e1[0] + j * I.e2[0];
            const int        y = n * I.o[1] + i * I.e1[1] + j * I.e2[1];
            const int        z = n * I.o[2] + i * I.e1[2] + j * I.e2[2];
            const int64_t    c = P.off[P.nB + I.cell] + cidx( n, x, y, z );
            ( s ? r.c1 : r.c0 )     = c;
            ( s ? r.cell1 : r.cell0 ) = I.cell;
            ( s ? r.y1 : r.y0 )     = int16_t( y );
            ( s ? r.z1 : r.z0 )     = int16_t( z );
            ( s ? r.cls1 : r.cls0 ) = int8_t( I.cls );
         }
      }
      up( &P.d_frec, fr.data(), fr.size() );
   }
   std::vector< int2 > rw( P.rows.size() );
   for ( size_t i = 0; i < rw.size(); ++i ) rw[i] = make_int2( P.rows[i][0], P.rows[i][1] );
   up( &P.d_rows, rw.data(), rw.size() );
   std::vector< int4 > mi( P.march.size() );
   for ( size_t i = 0; i < mi.size(); ++i ) mi[i] = make_int4( P.march[i][0], P.march[i][1], P.march[i][2], P.march[i][3] );
   up( &P.d_march, mi.data(), mi.size() );
   int dev = 0, sms = 0;
   check_cuda( cudaGetDevice( &dev ), "cudaGetDevice" );
   check_cuda( cudaDeviceGetAttribute( &sms, cudaDevAttrMultiProcessorCount, dev ), "device attribute" );
   {
      build_zunits( P, 2 * std::max( sms, 1 ), t.nC );
      std::vector< int4 > zu( P.zunits.size() );
      for ( size_t i = 0; i < zu.size(); ++i ) zu[i] = make_int4( P.zunits[i][0], P.zunits[i][1], P.zunits[i][2], P.zunits[i][3] );
      up( &P.d_zunits, zu.data(), zu.size() );
      up( &P.d_zcell, P.zcell.data(), P.zcell.size() );
      up( &P.d_zbegin, P.zbegin.data(), P.zbegin.size() );
   }
   for ( int b = 0; b < kSwLists; ++b )
   {
      // one list set per blocks-per-SM count (b + 2) of the sweep's instantiations
      build_sweep_units( P, b, sms * ( b + 2 ) * kSwWarps, t.nC );
      const auto&         U = P.swunits[b];
      std::vector< int4 > su( U.size() );
      for ( size_t i = 0; i < su.size(); ++i ) su[i] = make_int4( U[i][0], U[i][1], U[i][2], U[i][3] );
      up( &P.d_swunits[b], su.data(), su.size() );
      up( &P.d_swcell[b], P.swcell[b].data(), P.swcell[b].size() );
      up( &P.d_swbegin[b], P.swbegin[b].data(), P.swbegin[b].size() );
   }
   std::vector< uint8_t > bc( nP );
   std::vector< int8_t >  bk( P.nB );
   for ( int v = 0; v < t.nV; ++v ) bc[v] = uint8_t( t.bc( t.flag_v[v] ) ), bk[v] = 0;
   for ( int e = 0; e < t.nE; ++e ) bc[t.nV + e] = uint8_t( t.bc( t.flag_e[e] ) ), bk[t.nV + e] = 1;
   for ( int f = 0; f < t.nF; ++f ) bc[t.nV + t.nE + f] = uint8_t( t.bc( t.flag_f[f] ) ), bk[t.nV + t.nE + f] = 2;
   for ( int c = 0; c < t.nC; ++c ) bc[t.nV + t.nE + t.nF + c] = uint8_t( t.bc( t.flag_c[c] ) );
   up( &P.d_bc, bc.data(), bc.size() );
   up( &P.d_bkind, bk.data(), bk.size() );
   std::vector< float > ncc( size_t( t.nC ) * kNumClasses );
   for ( int c = 0; c < t.nC; ++c )
   {
      float* r = &ncc[size_t( c ) * kNumClasses];
      r[0]     = 1.f;
      for ( int k = 0; k < 4; ++k ) r[1 + k] = float( t.f_cells[t.cf[c][k]].size() );
      for ( int k = 0; k < 6; ++k ) r[5 + k] = float( t.e_cells[t.ce[c][k]].size() );
      for ( int k = 0; k < 4; ++k ) r[11 + k] = float( t.v_cells[t.cv[c][k]].size() );
   }
   up( &P.d_ncell_cls, ncc.data(), ncc.size() );
}

P1Level& Mesh::level( int L )
{
   auto it = levels.find( L );
   if ( it == levels.end() )
   {
      build_level( this, L );
      it = levels.find( L );
   }
   return *it->second;
}

Mesh::~Mesh()
{
   for ( auto& kv : levels )
   {
      P1Level& P = *kv.second;
      cudaFree( P.d_off );
      cudaFree( P.d_poff );
      cudaFree( P.d_inc_begin );
      cudaFree( P.d_inc );
      cudaFree( P.d_tasks );
      cudaFree( P.d_btasks );
      cudaFree( P.d_frec );
      cudaFree( P.d_rows );
      cudaFree( P.d_march );
      cudaFree( P.d_zunits ), cudaFree( P.d_zcell ), cudaFree( P.d_zbegin );
      for ( int b = 0; b < kSwLists; ++b ) cudaFree( P.d_swunits[b] ), cudaFree( P.d_swcell[b] ), cudaFree( P.d_swbegin[b] );
      cudaFree( P.d_bc );
      cudaFree( P.d_bkind );
      cudaFree( P.d_ncell_cls );
   }
}

// ---------------------------------------------------------------------------------------------
// operator stencils
// ---------------------------------------------------------------------------------------------
// Micro-cell types: vertex offsets (CellDoFIndexing.hpp:155-198).
static const int kMicroCells[6][4][3] = {
    { { 0, 0, 0 }, { 1, 0, 0 }, { 0, 1, 0 }, { 0, 0, 1 } },  // white up
    { { 1, 0, 0 }, { 1, 1, 0 }, { 0, 1, 0 }, { 1, 0, 1 } },  // blue up
    { { 1, 0, 0 }, { 0, 1, 0 }, { 1, 0, 1 }, { 0, 0, 1 } },  // green up
    { { 1, 1, 0 }, { 1, 1, 1 }, { 0, 1, 1 }, { 1, 0, 1 } },  // white down
    { { 1, 0, 1 }, { 0, 1, 1 }, { 0, 0, 1 }, { 0, 1, 0 } },  // blue down
    { { 0, 1, 0 }, { 1, 1, 0 }, { 1, 0, 1 }, { 0, 1, 1 } },  // green down
};

static int dir_index( int dx, int dy, int dz )
{
   for ( int d = 0; d < kNumDirs; ++d )
      if ( kDirs[d][0] == dx && kDirs[d][1] == dy && kDirs[d][2] == dz ) return d;
   throw std::logic_error( "not a stencil direction" );
}

// Row 0 of the element matrix of the tet with vertices X[0..3] (the first vertex is the centre).
// kind 1: P1 Laplace |det J|/6 * G G^T (p1_tet_diffusion); kind 2: P1 mass |det J|/120 (1+delta).
static void element_row0( int kind, const double X[4][3], double row[4] )
{
   double J[3][3];
   for ( int r = 0; r < 3; ++r )
      for ( int c = 0; c < 3; ++c ) J[r][c] = X[c + 1][r] - X[0][r];
   const double det = J[0][0] * ( J[1][1] * J[2][2] - J[1][2] * J[2][1] ) - J[0][1] * ( J[1][0] * J[2][2] - J[1][2] * J[2][0] ) +
                      J[0][2] * ( J[1][0] * J[2][1] - J[1][1] * J[2][0] );
   if ( kind == 2 )
   {
      const double v = std::fabs( det ) / 120.0;
      row[0]         = 2 * v;
      row[1] = row[2] = row[3] = v;
      return;
   }
   // inverse of J: rows are the gradients of the barycentric coordinates 1..3
   double inv[3][3];
   inv[0][0] = ( J[1][1] * J[2][2] - J[1][2] * J[2][1] ) / det;
   inv[0][1] = ( J[0][2] * J[2][1] - J[0][1] * J[2][2] ) / det;
   inv[0][2] = ( J[0][1] * J[1][2] - J[0][2] * J[1][1] ) / det;
   inv[1][0] = ( J[1][2] * J[2][0] - J[1][0] * J[2][2] ) / det;
   inv[1][1] = ( J[0][0] * J[2][2] - J[0][2] * J[2][0] ) / det;
   inv[1][2] = ( J[0][2] * J[1][0] - J[0][0] * J[1][2] ) / det;
   inv[2][0] = ( J[1][0] * J[2][1] - J[1][1] * J[2][0] ) / det;
   inv[2][1] = ( J[0][1] * J[2][0] - J[0][0] * J[2][1] ) / det;
   inv[2][2] = ( J[0][0] * J[1][1] - J[0][1] * J[1][0] ) / det;
   double G[4][3];
   for ( int d = 0; d < 3; ++d )
   {
      G[1][d] = inv[0][d];
      G[2][d] = inv[1][d];
      G[3][d] = inv[2][d];
      G[0][d] = -( G[1][d] + G[2][d] + G[3][d] );
   }
   const double vol = std::fabs( det ) / 6.0;
   for ( int m = 0; m < 4; ++m ) row[m] = vol * ( G[0][0] * G[m][0] + G[0][1] * G[m][1] + G[0][2] * G[m][2] );
}

void build_operator_level( Operator* A, int L )
{
   const Topology& t = A->mesh->topo;
   const P1Level&  P = A->mesh->level( L );
   OpLevel         ol;
   const int       n = 1 << L;
   ol.W.assign( size_t( t.nC ) * kNumClasses * kNumDirs, 0.0 );
   for ( int c = 0; c < t.nC; ++c )
   {
      const auto& P0 = t.vx[t.cv[c][0]];
      const auto& P1 = t.vx[t.cv[c][1]];
      const auto& P2 = t.vx[t.cv[c][2]];
      const auto& P3 = t.vx[t.cv[c][3]];
      const double step = 1.0 / double( n );
      double xs[3], ys[3], zs[3];
      for ( int d = 0; d < 3; ++d )
      {
         xs[d] = ( P1[d] - P0[d] ) * step;
         ys[d] = ( P2[d] - P0[d] ) * step;
         zs[d] = ( P3[d] - P0[d] ) * step;
      }
      auto coord = [&]( int x, int y, int z, double* X ) {
         for ( int d = 0; d < 3; ++d ) X[d] = P0[d] + xs[d] * x + ys[d] * y + zs[d] * z;
      };
      // the 24 micro-cells around a micro-vertex: every micro-cell type, anchored so that each
      // of its four vertices in turn sits on the centre
      for ( int ty = 0; ty < 6; ++ty )
         for ( int k = 0; k < 4; ++k )
         {
            int rel[4][3];
            int order[4] = { k, ( k + 1 ) % 4, ( k + 2 ) % 4, ( k + 3 ) % 4 };
            for ( int q = 0; q < 4; ++q )
               for ( int d = 0; d < 3; ++d ) rel[q][d] = kMicroCells[ty][order[q]][d] - kMicroCells[ty][k][d];
            double X[4][3];
            for ( int q = 0; q < 4; ++q ) coord( 1 + rel[q][0], 1 + rel[q][1], 1 + rel[q][2], X[q] );
            double row[4];
            element_row0( A->kind, X, row );
            for ( int cls = 0; cls < kNumClasses; ++cls )
            {
               bool inside = true;
               for ( int q = 0; q < 4; ++q ) inside = inside && dir_ok_for_faces( kClassFaces[cls], rel[q] );
               if ( !inside ) continue;
               double* W = &ol.W[( size_t( c ) * kNumClasses + cls ) * kNumDirs];
               for ( int q = 0; q < 4; ++q ) W[dir_index( rel[q][0], rel[q][1], rel[q][2] )] += row[q];
            }
         }
   }
   ol.invd_c.resize( t.nC );
   for ( int c = 0; c < t.nC; ++c ) ol.invd_c[c] = 1.0 / ol.W[( size_t( c ) * kNumClasses + 0 ) * kNumDirs + 0];
   ol.invd_b.resize( P.nB );
   for ( int b = 0; b < P.nB; ++b )
   {
      double d = 0;
      for ( int q = P.inc_begin[b]; q < P.inc_begin[b + 1]; ++q )
         d += ol.W[( size_t( P.inc[q].cell ) * kNumClasses + P.inc[q].cls ) * kNumDirs + 0];
      ol.invd_b[b] = 1.0 / d;
   }
   A->lv[L] = std::move( ol );
}

void ensure_device_op( OpLevel& ol )
{
   if ( ol.d_W ) return;
   std::vector< float > Wf( ol.W.begin(), ol.W.end() ), ibf( ol.invd_b.begin(), ol.invd_b.end() ),
       icf( ol.invd_c.begin(), ol.invd_c.end() );
   auto up = [&]( auto** dptr, const auto& vec ) {
      using T = typename std::decay_t< decltype( vec ) >::value_type;
      check_cuda( cudaMalloc( (void**) dptr, std::max< size_t >( vec.size(), 1 ) * sizeof( T ) ), "cudaMalloc(stencils)" );
      if ( !vec.empty() )
         check_cuda( cudaMemcpy( *dptr, vec.data(), vec.size() * sizeof( T ), cudaMemcpyHostToDevice ), "upload stencils" );
   };
   up( &ol.d_W, ol.W );
   up( &ol.d_Wf, Wf );
   up( &ol.d_invd_b, ol.invd_b );
   up( &ol.d_invd_c, ol.invd_c );
   up( &ol.d_invd_bf, ibf );
   up( &ol.d_invd_cf, icf );
}

Operator::~Operator()
{
   for ( auto& kv : lv )
   {
      cudaFree( kv.second.d_W );
      cudaFree( kv.second.d_Wf );
      cudaFree( kv.second.d_invd_b );
      cudaFree( kv.second.d_invd_c );
      cudaFree( kv.second.d_invd_bf );
      cudaFree( kv.second.d_invd_cf );
   }
   for ( auto& kv : p2c )
   {
      cudaFree( kv.second.d_W );
      cudaFree( kv.second.d_Wf );
      cudaFree( kv.second.d_tasks );
   }
   for ( auto& kv : el )
   {
      cudaFree( kv.second.d_acc );
      for ( void* p : kv.second.d_invd ) cudaFree( p );
      for ( void* p : kv.second.d_K ) cudaFree( p );
      for ( void* p : kv.second.d_S ) cudaFree( p );
      cudaFree( kv.second.d_sacc );
      cudaFree( kv.second.d_kn );
      cudaFree( kv.second.d_anch );
   }
   cudaFree( d_geom );
}

size_t Function::bytes( int L ) const { return size_t( mesh->level( L ).size ) * dtype_size( dtype ); }


void check_cuda( cudaError_t e, const char* what )
{
   if ( e != cudaSuccess ) throw std::runtime_error( std::string( what ) + ": " + cudaGetErrorString( e ) );
}

}  // namespace hyb
