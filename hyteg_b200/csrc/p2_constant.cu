// P2 constant-stencil operator (P2ConstantOperator< P2FenicsForm< p2_diffusion > >, the reference's
// P2ConstantLaplaceOperator: constant_stencil_operator/P2ConstantOperator.cpp:100-114 applies its four
// stencil parts vertexToVertex, edgeToVertex, edgeToEdge and vertexToEdge).
//
// A P2 function of level l lives on the node set of level l+1 (vertex DoFs at even coordinates, edge
// DoFs at the micro-edge midpoints), so the operator is one stencil per parity class of that grid:
// the eight classes (x, y, z mod 2) are the vertex nodes and the midpoints of the seven micro-edge
// directions, with 65, 27, 19, 27, 27, 19, 27 and 19 entries reaching at most two points in every
// direction.  On an affine macro-cell the stencil of a class is the same at every interior point: the
// sum, over the level-l micro-cells that contain the point, of the row of their P2 element matrix.
// Points on a macro-cell's faces, edges and vertices take the same sum over the micro-cells inside
// each neighbouring macro-cell (one partial stencil per position class and parity) and add the
// cells' parts, as the P1 boundary kernel does.
//
// Kernels:
//  * k_p2c_sweep: cell interiors.  Each warp streams its units (4 rows by 64 x-points over a range of
//    slices) through a private ring of shared-memory stages with cp.async.bulk; lane l owns the two
//    points x0 + 2l and x0 + 2l + 1 of every row, so every lane of a warp applies the same class
//    stencil at the same time and the weights are warp-uniform shared-memory reads.  Each slice is
//    read once: its values are folded into running sums of the five output slices z-2..z+2 they
//    reach (partial sums in y and z), and a slice's points are written two steps after it arrives.
//  * k_p2c_bnd: owned face/edge/vertex nodes, one thread each: the partial stencils of every
//    neighbouring cell, summed in incidence order, written through to all copies.
// Both use the operation epilogues of the P1 path (apply, residual, Jacobi, Chebyshev steps).
#include "hyb_internal.hpp"
#include "hyb_device.cuh"

#include <algorithm>
#include <cmath>
#include <type_traits>

namespace hyb {

// ---------------------------------------------------------------------------------------------
// node pattern (compile time)
// ---------------------------------------------------------------------------------------------
// micro-cell types: vertex offsets in level-l units (CellDoFIndexing.hpp:155-198)
constexpr int kP2MC[6][4][3] = {
    { { 0, 0, 0 }, { 1, 0, 0 }, { 0, 1, 0 }, { 0, 0, 1 } }, { { 1, 0, 0 }, { 1, 1, 0 }, { 0, 1, 0 }, { 1, 0, 1 } },
    { { 1, 0, 0 }, { 0, 1, 0 }, { 1, 0, 1 }, { 0, 0, 1 } }, { { 1, 1, 0 }, { 1, 1, 1 }, { 0, 1, 1 }, { 1, 0, 1 } },
    { { 1, 0, 1 }, { 0, 1, 1 }, { 0, 0, 1 }, { 0, 1, 0 } }, { { 0, 1, 0 }, { 1, 1, 0 }, { 1, 0, 1 }, { 0, 1, 1 } },
};
// local nodes of the P2 element used here: the four vertices, then the midpoints of the edges below
constexpr int kP2Edge[6][2] = { { 0, 1 }, { 0, 2 }, { 0, 3 }, { 1, 2 }, { 1, 3 }, { 2, 3 } };

// node m (0..9) of a micro-cell of type t, in level-(l+1) units relative to twice its anchor
constexpr int p2_node( int t, int m, int d )
{
   return m < 4 ? 2 * kP2MC[t][m][d] : kP2MC[t][kP2Edge[m - 4][0]][d] + kP2MC[t][kP2Edge[m - 4][1]][d];
}

struct P2Pattern
{
   int    cnt[8];              // stencil entries of parity class k
   int    base[9];             // first entry of class k in the concatenated list
   int    centre[8];           // class-relative entry of the offset (0, 0, 0)
   int8_t off[kP2cEntries][3]; // (dx, dy, dz) of every entry; within a class sorted by dz, dy, dx
   int    rng[8][5][5][2];     // [k][dz+2][dy+2]: class-relative [begin, end) of the entries with that dz, dy
};

// The offsets reached from an interior point of parity class k: every node of every micro-cell that
// has the point as one of its nodes.
constexpr P2Pattern make_p2_pattern()
{
   P2Pattern P{};
   int       at = 0;
   for ( int k = 0; k < 8; ++k )
   {
      at                     = ( at + 3 ) / 4 * 4;  // classes start on 16-byte (double2 / float4) boundaries
      bool      hit[5][5][5] = {};
      const int p[3]         = { 8 + ( k & 1 ), 8 + ( ( k >> 1 ) & 1 ), 8 + ( k >> 2 ) };
      for ( int t = 0; t < 6; ++t )
         for ( int m = 0; m < 10; ++m )
         {
            int  a2[3] = {};
            bool ok    = true;
            for ( int d = 0; d < 3; ++d )
            {
               a2[d] = p[d] - p2_node( t, m, d );
               ok    = ok && ( a2[d] % 2 == 0 );
            }
            if ( !ok ) continue;
            for ( int m2 = 0; m2 < 10; ++m2 )
               hit[a2[2] + p2_node( t, m2, 2 ) - p[2] + 2][a2[1] + p2_node( t, m2, 1 ) - p[1] + 2][a2[0] + p2_node( t, m2, 0 ) - p[0] + 2] =
                   true;
         }
      P.base[k] = at;
      for ( int dz = 0; dz < 5; ++dz )
         for ( int dy = 0; dy < 5; ++dy )
         {
            P.rng[k][dz][dy][0] = at - P.base[k];
            for ( int dx = 0; dx < 5; ++dx )
               if ( hit[dz][dy][dx] )
               {
                  if ( dx == 2 && dy == 2 && dz == 2 ) P.centre[k] = at - P.base[k];
                  P.off[at][0] = int8_t( dx - 2 );
                  P.off[at][1] = int8_t( dy - 2 );
                  P.off[at][2] = int8_t( dz - 2 );
                  ++at;
               }
            P.rng[k][dz][dy][1] = at - P.base[k];
         }
      P.cnt[k] = at - P.base[k];
   }
   P.base[8] = at;
   return P;
}

constexpr P2Pattern kP2Pat = make_p2_pattern();
static_assert( kP2Pat.cnt[0] + kP2Pat.cnt[1] + kP2Pat.cnt[2] + kP2Pat.cnt[3] + kP2Pat.cnt[4] + kP2Pat.cnt[5] + kP2Pat.cnt[6] +
                       kP2Pat.cnt[7] == 230 &&
                   kP2Pat.cnt[0] == 65 && kP2Pat.cnt[1] == 27 && kP2Pat.cnt[2] == 19,
               "P2 stencil sizes of the six-type refinement" );
static_assert( kP2Pat.base[8] <= kP2cEntries, "entry block too small" );
static_assert( kSwR == 4 && kSwTX == 64, "the P2 sweep reuses the cell-sweep units: 4 rows by 64 x-points, x0 and y0 odd" );

__constant__ int c_p2c_faces[kNumClasses];  // kClassFaces
// the pattern for lanes that read different classes (boundary owners): offsets (dx, dy, dz) of every
// entry, and per class its first entry, entry count and centre entry
__device__ char4 g_p2c_off[kP2cEntries];
__device__ int   g_p2c_base[24];

// ---------------------------------------------------------------------------------------------
// host: tables
// ---------------------------------------------------------------------------------------------
// P2 stiffness matrix of the tet X[0..3] in the node order above, integrated exactly with the
// degree-2 four-point rule (barycentric points (a, a, a, b) and permutations, a = (5 - sqrt 5)/20,
// b = (5 + 3 sqrt 5)/20, weight |T|/4): the basis gradients are linear, their products quadratic.
static void p2_laplace_element( const double X[4][3], double K[10][10] )
{
   double J[3][3];
   for ( int r = 0; r < 3; ++r )
      for ( int c = 0; c < 3; ++c ) J[r][c] = X[c + 1][r] - X[0][r];
   const double det = J[0][0] * ( J[1][1] * J[2][2] - J[1][2] * J[2][1] ) - J[0][1] * ( J[1][0] * J[2][2] - J[1][2] * J[2][0] ) +
                      J[0][2] * ( J[1][0] * J[2][1] - J[1][1] * J[2][0] );
   // rows of J^-1: gradients of the barycentric coordinates 1..3
   double g[4][3];
   g[1][0] = ( J[1][1] * J[2][2] - J[1][2] * J[2][1] ) / det;
   g[1][1] = ( J[0][2] * J[2][1] - J[0][1] * J[2][2] ) / det;
   g[1][2] = ( J[0][1] * J[1][2] - J[0][2] * J[1][1] ) / det;
   g[2][0] = ( J[1][2] * J[2][0] - J[1][0] * J[2][2] ) / det;
   g[2][1] = ( J[0][0] * J[2][2] - J[0][2] * J[2][0] ) / det;
   g[2][2] = ( J[0][2] * J[1][0] - J[0][0] * J[1][2] ) / det;
   g[3][0] = ( J[1][0] * J[2][1] - J[1][1] * J[2][0] ) / det;
   g[3][1] = ( J[0][1] * J[2][0] - J[0][0] * J[2][1] ) / det;
   g[3][2] = ( J[0][0] * J[1][1] - J[0][1] * J[1][0] ) / det;
   for ( int d = 0; d < 3; ++d ) g[0][d] = -( g[1][d] + g[2][d] + g[3][d] );
   const double vol = std::fabs( det ) / 6.0;
   const double a = ( 5.0 - std::sqrt( 5.0 ) ) / 20.0, b = ( 5.0 + 3.0 * std::sqrt( 5.0 ) ) / 20.0;
   for ( int i = 0; i < 10; ++i )
      for ( int j = 0; j < 10; ++j ) K[i][j] = 0.0;
   for ( int q = 0; q < 4; ++q )
   {
      double lam[4] = { a, a, a, a };
      lam[q]        = b;
      double G[10][3];
      for ( int m = 0; m < 4; ++m )
         for ( int d = 0; d < 3; ++d ) G[m][d] = ( 4.0 * lam[m] - 1.0 ) * g[m][d];
      for ( int e = 0; e < 6; ++e )
      {
         const int i = kP2Edge[e][0], j = kP2Edge[e][1];
         for ( int d = 0; d < 3; ++d ) G[4 + e][d] = 4.0 * ( lam[i] * g[j][d] + lam[j] * g[i][d] );
      }
      for ( int i = 0; i < 10; ++i )
         for ( int j = 0; j < 10; ++j ) K[i][j] += 0.25 * vol * ( G[i][0] * G[j][0] + G[i][1] * G[j][1] + G[i][2] * G[j][2] );
   }
}

static int pattern_entry( int k, int dx, int dy, int dz )
{
   for ( int e = 0; e < kP2Pat.cnt[k]; ++e )
   {
      const int8_t* o = kP2Pat.off[kP2Pat.base[k] + e];
      if ( o[0] == dx && o[1] == dy && o[2] == dz ) return e;
   }
   throw std::logic_error( "P2 stencil offset outside the class pattern" );
}

static int block_offset( int cls ) { return cls == 0 ? 0 : kP2cInterior + ( cls - 1 ) * kP2cEntries; }

// Stencil tables of storage level Ls (P2 level Ls-1) of a P2 constant Laplace operator.
void build_p2_constant_level( Operator* A, int Ls )
{
   const Topology& t  = A->mesh->topo;
   const int       nl = 1 << ( Ls - 1 );  // micro-cells per macro-edge at the P2 level
   P2cLevel        pl;
   pl.W.assign( size_t( t.nC ) * kP2cCellStride, 0.0 );
   // a representative point of every (position class, parity) on a virtual grid of 16 intervals: the
   // micro-cells inside the macro-cell around a point depend only on the faces the point lies on
   constexpr int NV = 16;
   int           rep[kNumClasses][8][3];
   bool          has[kNumClasses][8] = {};
   for ( int z = 0; z <= NV; ++z )
      for ( int y = 0; y + z <= NV; ++y )
         for ( int x = 0; x + y + z <= NV; ++x )
         {
            const int cls = class_of_point( NV, x, y, z ), k = ( x & 1 ) | ( ( y & 1 ) << 1 ) | ( ( z & 1 ) << 2 );
            if ( !has[cls][k] )
            {
               has[cls][k] = true;
               rep[cls][k][0] = x, rep[cls][k][1] = y, rep[cls][k][2] = z;
            }
         }
   for ( int c = 0; c < t.nC; ++c )
   {
      const auto& P0 = t.vx[t.cv[c][0]];
      double      dir[3][3];
      for ( int v = 0; v < 3; ++v )
         for ( int d = 0; d < 3; ++d ) dir[v][d] = ( t.vx[t.cv[c][v + 1]][d] - P0[d] ) / double( nl );
      double K[6][10][10];
      for ( int ty = 0; ty < 6; ++ty )
      {
         double X[4][3];
         for ( int q = 0; q < 4; ++q )
            for ( int d = 0; d < 3; ++d )
               X[q][d] = P0[d] + dir[0][d] * kP2MC[ty][q][0] + dir[1][d] * kP2MC[ty][q][1] + dir[2][d] * kP2MC[ty][q][2];
         p2_laplace_element( X, K[ty] );
      }
      double* Wc = &pl.W[size_t( c ) * kP2cCellStride];
      for ( int cls = 0; cls < kNumClasses; ++cls )
         for ( int k = 0; k < 8; ++k )
         {
            if ( !has[cls][k] ) continue;
            const int* p  = rep[cls][k];
            double*    Wb = Wc + block_offset( cls ) + kP2Pat.base[k];
            for ( int ty = 0; ty < 6; ++ty )
               for ( int m = 0; m < 10; ++m )
               {
                  int  a2[3];
                  bool ok = true;
                  for ( int d = 0; d < 3; ++d )
                  {
                     a2[d] = p[d] - p2_node( ty, m, d );
                     ok    = ok && ( ( a2[d] & 1 ) == 0 );
                  }
                  if ( !ok ) continue;
                  for ( int q = 0; q < 4 && ok; ++q )
                  {
                     const int vx = a2[0] + 2 * kP2MC[ty][q][0], vy = a2[1] + 2 * kP2MC[ty][q][1], vz = a2[2] + 2 * kP2MC[ty][q][2];
                     ok = vx >= 0 && vy >= 0 && vz >= 0 && vx + vy + vz <= NV;
                  }
                  if ( !ok ) continue;
                  for ( int m2 = 0; m2 < 10; ++m2 )
                     Wb[pattern_entry( k, a2[0] + p2_node( ty, m2, 0 ) - p[0], a2[1] + p2_node( ty, m2, 1 ) - p[1],
                                       a2[2] + p2_node( ty, m2, 2 ) - p[2] )] += K[ty][m][m2];
               }
         }
      for ( int k = 0; k < 8; ++k ) Wc[kP2cEntries + k] = 1.0 / Wc[kP2Pat.base[k] + kP2Pat.centre[k]];
   }
   // boundary tasks in the grouping of the P1 level (by boundary type, so that a launch covers the
   // flagged groups), inside a group sorted by primitive and by the parity class of the node in its
   // first cell: the lanes of a warp then walk the same stencil pattern
   const P1Level& P = A->mesh->level( Ls );
   const int      N = P.n;
   const uint32_t type_bit[4] = { kInner, kDirichlet, kNeumann, kFreeslip };
   auto           btype = [&]( int b ) {
      return b < t.nV ? t.bc( t.flag_v[b] ) : ( b < t.nV + t.nE ? t.bc( t.flag_e[b - t.nV] ) : t.bc( t.flag_f[b - t.nV - t.nE] ) );
   };
   auto parity = [&]( const std::array< int, 4 >& q ) {
      const Incidence& I = P.inc[P.inc_begin[q[0]]];
      const int        x = N * I.o[0] + q[1] * I.e1[0] + q[2] * I.e2[0];
      const int        y = N * I.o[1] + q[1] * I.e1[1] + q[2] * I.e2[1];
      const int        z = N * I.o[2] + q[1] * I.e1[2] + q[2] * I.e2[2];
      return ( x & 1 ) | ( ( y & 1 ) << 1 ) | ( ( z & 1 ) << 2 );
   };
   for ( int g = 0; g < 4; ++g )
   {
      std::vector< std::pair< int64_t, int > > key;
      for ( size_t q = 0; q < P.tasks.size(); ++q )
         if ( btype( P.tasks[q][0] ) == type_bit[g] ) key.push_back( { int64_t( P.tasks[q][0] ) * 8 + parity( P.tasks[q] ), int( q ) } );
      std::stable_sort( key.begin(), key.end(), []( const auto& a, const auto& c ) { return a.first < c.first; } );
      for ( const auto& kq : key ) pl.tasks.push_back( make_int4( P.tasks[kq.second][0], P.tasks[kq.second][1], P.tasks[kq.second][2], 0 ) );
   }
   if ( pl.tasks.size() != P.tasks.size() ) throw std::logic_error( "boundary task without a single boundary type" );
   A->p2c[Ls] = std::move( pl );
}

static PerDeviceOnce g_p2c_once;
static void          p2c_attributes_all();

// constant pattern and kernel attributes, once per device (before any capture: operator creation)
void ensure_p2_constant_device()
{
   g_p2c_once.run( [] {
      char4 off[kP2cEntries] = {};
      for ( int e = 0; e < kP2cEntries; ++e ) off[e] = make_char4( kP2Pat.off[e][0], kP2Pat.off[e][1], kP2Pat.off[e][2], 0 );
      int base[24];
      for ( int k = 0; k < 8; ++k ) base[k] = kP2Pat.base[k], base[k + 8] = kP2Pat.cnt[k], base[k + 16] = kP2Pat.centre[k];
      check_cuda( cudaMemcpyToSymbol( g_p2c_off, off, sizeof( off ) ), "constants(P2 pattern)" );
      check_cuda( cudaMemcpyToSymbol( g_p2c_base, base, sizeof( base ) ), "constants(P2 pattern)" );
      check_cuda( cudaMemcpyToSymbol( c_p2c_faces, kClassFaces, sizeof( kClassFaces ) ), "constants(P2 classes)" );
      p2c_attributes_all();
   } );
}

void ensure_p2_constant_tables( P2cLevel& pl )
{
   if ( pl.d_W ) return;
   std::vector< float > wf( pl.W.begin(), pl.W.end() );
   check_cuda( cudaMalloc( &pl.d_W, pl.W.size() * sizeof( double ) ), "cudaMalloc(P2 stencils)" );
   check_cuda( cudaMalloc( &pl.d_Wf, wf.size() * sizeof( float ) ), "cudaMalloc(P2 stencils)" );
   check_cuda( cudaMemcpy( pl.d_W, pl.W.data(), pl.W.size() * sizeof( double ), cudaMemcpyHostToDevice ), "upload P2 stencils" );
   check_cuda( cudaMemcpy( pl.d_Wf, wf.data(), wf.size() * sizeof( float ), cudaMemcpyHostToDevice ), "upload P2 stencils" );
   check_cuda( cudaMalloc( &pl.d_tasks, std::max< size_t >( pl.tasks.size(), 1 ) * sizeof( int4 ) ), "cudaMalloc(P2 tasks)" );
   if ( !pl.tasks.empty() )
      check_cuda( cudaMemcpy( pl.d_tasks, pl.tasks.data(), pl.tasks.size() * sizeof( int4 ), cudaMemcpyHostToDevice ), "upload P2 tasks" );
}

// inverse diagonal of every owned slot flagged by `flag` (padded level layout), from the tables
void p2_constant_inverse_diagonal( const Operator* A, int Ls, uint32_t flag, std::vector< double >& padded )
{
   const Topology& t  = A->mesh->topo;
   const P1Level&  P  = A->mesh->level( Ls );
   const P2cLevel& pl = A->p2c.at( Ls );
   const int       N  = P.n;
   for ( const auto& tk : P.tasks )
   {
      const int b  = tk[0];
      uint32_t  bc = b < t.nV ? t.bc( t.flag_v[b] ) : b < t.nV + t.nE ? t.bc( t.flag_e[b - t.nV] ) : t.bc( t.flag_f[b - t.nV - t.nE] );
      if ( !( bc & flag ) ) continue;
      double d = 0;
      for ( int q = P.inc_begin[b]; q < P.inc_begin[b + 1]; ++q )
      {
         const Incidence& I = P.inc[q];
         const int        x = N * I.o[0] + tk[1] * I.e1[0] + tk[2] * I.e2[0];
         const int        y = N * I.o[1] + tk[1] * I.e1[1] + tk[2] * I.e2[1];
         const int        z = N * I.o[2] + tk[1] * I.e1[2] + tk[2] * I.e2[2];
         const int        k = ( x & 1 ) | ( ( y & 1 ) << 1 ) | ( ( z & 1 ) << 2 );
         d += pl.W[size_t( I.cell ) * kP2cCellStride + block_offset( I.cls ) + kP2Pat.base[k] + kP2Pat.centre[k]];
      }
      const int64_t o = P.off[b] + ( b < t.nV ? 0 : b < t.nV + t.nE ? tk[1] : fidx( N, tk[1], tk[2] ) );
      padded[o]       = 1.0 / d;
   }
   for ( int c = 0; c < t.nC; ++c )
   {
      if ( !( t.bc( t.flag_c[c] ) & flag ) ) continue;
      const int64_t base = P.off[P.nB + c];
      const double* inv  = &pl.W[size_t( c ) * kP2cCellStride + kP2cEntries];
      for ( int z = 1; z < N; ++z )
         for ( int y = 1; y + z < N; ++y )
            for ( int x = 1; x + y + z < N; ++x ) padded[base + cidx( N, x, y, z )] = inv[( x & 1 ) | ( ( y & 1 ) << 1 ) | ( ( z & 1 ) << 2 )];
   }
}

// ---------------------------------------------------------------------------------------------
// device: interior sweep
// ---------------------------------------------------------------------------------------------
constexpr int kP2cWarps = 4;  // warps per block; two blocks per SM (unit list 0 of the cell sweep)

template < typename T, typename A >
struct P2cCfg
{
   static constexpr int    AL    = 16 / int( sizeof( T ) );               // elements per 16 bytes
   static constexpr int    RW    = ( 68 + 2 * AL + AL - 1 ) / AL * AL;    // stage row: x0-2..x0+65 plus alignment
   static constexpr int    ROWS  = kSwR + 4;                              // tile rows and two halo rows each side
   static constexpr int    stage = ROWS * RW;                             // elements per stage
   static constexpr int    WS    = ( kP2cInterior * int( sizeof( A ) ) + 15 ) / 16 * 16 / int( sizeof( A ) );
   static constexpr int    Draw  = int( ( 96 * 1024 - WS * int( sizeof( A ) ) * kP2cWarps ) / ( kP2cWarps * stage * int( sizeof( T ) ) ) );
   static constexpr int    D     = Draw < 3 ? 3 : ( Draw > 8 ? 8 : Draw );  // ring depth
   static constexpr size_t warp_elems = size_t( D ) * stage;
   static constexpr size_t smem_bytes = kP2cWarps * ( warp_elems * sizeof( T ) + WS * sizeof( A ) );
   static_assert( ( stage * sizeof( T ) ) % 16 == 0 && ( RW * sizeof( T ) ) % 16 == 0, "bulk copies need 16-byte aligned rows" );
   static_assert( ROWS <= 32, "one row copy per lane" );
};

// 16-byte vectors of weights
template < typename A >
struct WVec;
template <>
struct WVec< double >
{
   using type              = double2;
   static constexpr int n = 2;
};
template <>
struct WVec< float >
{
   using type              = float4;
   static constexpr int n = 4;
};
template < typename A >
using WVec_t = typename WVec< A >::type;
template < int I >
__device__ __forceinline__ double vget( const double2& v )
{
   return I == 0 ? v.x : v.y;
}
template < int I >
__device__ __forceinline__ float vget( const float4& v )
{
   return I == 0 ? v.x : I == 1 ? v.y : I == 2 ? v.z : v.w;
}

// the six values x0 - 2 + 2 lane + i (i < 6) of a stage row; q = row start + 2 lane, sh = the row's
// shift (the stage row starts sh elements before x0 - 2).  FP64 and FP32 rows are read in 16- and
// 8-byte pairs from an aligned pair boundary (conflict-free), FP16 value by value.
__device__ __forceinline__ void load_row6( const double* q, int sh, double val[6] )
{
   const double2* p = reinterpret_cast< const double2* >( q );  // 2 lane even, rows of even width
   if ( sh & 1 )
   {
      const double2 a = p[0], b = p[1], c = p[2], d = p[3];
      val[0] = a.y, val[1] = b.x, val[2] = b.y, val[3] = c.x, val[4] = c.y, val[5] = d.x;
   }
   else
   {
      const double2 a = p[0], b = p[1], c = p[2];
      val[0] = a.x, val[1] = a.y, val[2] = b.x, val[3] = b.y, val[4] = c.x, val[5] = c.y;
   }
}
__device__ __forceinline__ void load_row6( const float* q, int sh, float val[6] )
{
   const float2* p = reinterpret_cast< const float2* >( q + ( sh & ~1 ) );
   if ( sh & 1 )
   {
      const float2 a = p[0], b = p[1], c = p[2], d = p[3];
      val[0] = a.y, val[1] = b.x, val[2] = b.y, val[3] = c.x, val[4] = c.y, val[5] = d.x;
   }
   else
   {
      const float2 a = p[0], b = p[1], c = p[2];
      val[0] = a.x, val[1] = a.y, val[2] = b.x, val[3] = b.y, val[4] = c.x, val[5] = c.y;
   }
}
__device__ __forceinline__ void load_row6( const __half* q, int sh, float val[6] )
{
#pragma unroll
   for ( int i = 0; i < 6; ++i ) val[i] = __half2float( q[sh + i] );
}

template < int B, int E, typename F >
__device__ __forceinline__ void static_for( F&& f )
{
   if constexpr ( B < E )
   {
      f( std::integral_constant< int, B >{} );
      static_for< B + 1, E >( f );
   }
}

template < typename T, typename A, int OP >
__global__ void __launch_bounds__( kP2cWarps * 32, 2 )
    k_p2c_sweep( LevelView v, const A* __restrict__ W, uint32_t flag, const T* __restrict__ src, const T* __restrict__ v1, T* v2, T* dst,
                 A a0, A a1, int nC, int* err )
{
   using Cfg = P2cCfg< T, A >;
   constexpr int D = Cfg::D, RW = Cfg::RW, AL = Cfg::AL, R = kSwR;
   extern __shared__ __align__( 128 ) unsigned char p2c_raw[];
   __shared__ uint64_t bars[kP2cWarps][D];
   const int           warp = threadIdx.x >> 5, lane = threadIdx.x & 31, N = v.n;
   T* const            ring = reinterpret_cast< T* >( p2c_raw ) + size_t( warp ) * Cfg::warp_elems;
   A* const            Wsm  = reinterpret_cast< A* >( p2c_raw + kP2cWarps * Cfg::warp_elems * sizeof( T ) ) + warp * Cfg::WS;
   uint64_t* const     full = bars[warp];
   if ( lane == 0 )
   {
      for ( int s = 0; s < D; ++s ) mbar_init( &full[s], 1 );
      asm volatile( "fence.mbarrier_init.release.cluster;" ::: "memory" );
   }
   __syncwarp();
   const int   gw  = blockIdx.x * kP2cWarps + warp;
   const int*  ucl = v.swcell[0];
   const int4* uu  = v.swunits[0];
   const int   u1  = v.swbegin[0][gw + 1];
   auto        active = [&]( int u ) {
      const int c = ucl[u];
      return c < nC && ( v.cell_bc[c] & flag ) != 0;
   };

   // ---- loads: lane r < R+4 copies row y0-2+r of every slice z_first-2 .. z_last+2 of the warp's units
   const bool is_row = lane < R + 4;
   int        pu = v.swbegin[0][gw], ps = 0, pyy = 0, px0 = 0;
   int64_t    pcb = 0, prb = 0;  // cell offset; start of this lane's row in slice ps (cell-relative)
   int4       PU  = make_int4( 0, 0, 0, 0 );
   auto       open = [&]() {
      while ( pu < u1 && !active( pu ) ) ++pu;
      if ( pu < u1 )
      {
         PU  = uu[pu];
         pcb = v.cell_off[ucl[pu]];
         ps  = PU.z - 2;
         pyy = PU.y - 2 + lane;
         px0 = PU.x & kSwUnitXMask;
         prb = cidx( N, 0, pyy, ps );  // the polynomial also serves rows and slices outside the cell
      }
   };
   open();
   int  issued = 0, ist = 0;
   auto issue  = [&]() {
      if ( pu >= u1 ) return;
      const int st = ist;
      uint32_t  bytes = 0;
      int64_t   a0s   = 0;
      if ( is_row && pyy >= 0 && ps >= 0 && pyy + ps <= N )
      {
         const int xe = min( px0 + 65, N - pyy - ps );  // last x of the row segment
         if ( xe >= px0 - 2 && xe >= 0 )
         {
            const int64_t rs = pcb + prb;
            const int64_t g0 = rs + px0 - 2;  // x0 - 2 >= -1: at worst the slot before the row, inside the buffer
            a0s              = g0 & ~int64_t( AL - 1 );
            bytes            = uint32_t( ( ( rs + xe + 1 + AL - 1 ) / AL * AL - a0s ) * int64_t( sizeof( T ) ) );
         }
      }
      const uint32_t total = __reduce_add_sync( 0xffffffffu, bytes );
      if ( lane == 0 ) mbar_expect_tx( &full[st], total );
      __syncwarp();
      if ( bytes ) bulk_copy_g2s( ring + st * Cfg::stage + lane * RW, src + a0s, bytes, &full[st] );
      ++issued;
      ist = ist + 1 == D ? 0 : ist + 1;
      prb += slice_step( N, ps ) - pyy;
      if ( ++ps > PU.w + 2 )
      {
         ++pu;
         open();
      }
   };
   for ( int i = 0; i < D; ++i ) issue();

   int      ld = 0, cst = 0;
   uint32_t cph  = 0;
   auto     fail = [&]() {
      if ( lane == 0 )
      {
         atomicExch( err, 1 );
         for ( int i = ld; i < issued; ++i )
            if ( !mbar_wait_bounded( &full[i % D], uint32_t( ( i / D ) & 1 ), nullptr ) ) break;
      }
      __syncwarp();
   };

   int cw = -1;
   for ( int u = v.swbegin[0][gw]; u < u1; ++u )
   {
      if ( !active( u ) ) continue;
      const int c = ucl[u];
      if ( c != cw )
      {
         __syncwarp();
         for ( int i = lane; i < kP2cInterior; i += 32 ) Wsm[i] = W[size_t( c ) * kP2cCellStride + i];
         __syncwarp();
         cw = c;
      }
      const int4    U  = uu[u];
      const int     x0 = U.x & kSwUnitXMask, y0 = U.y, za = U.z, zb = U.w;
      const int64_t cb = v.cell_off[c];
      // row starts, kept by additions from slice to slice (cidx(0, y, z+1) = cidx(0, y, z) + tri(N+1-z) - y,
      // a polynomial identity that also holds for the rows and slices outside the cell): shw packs the
      // shift (row start + x0 - 2 mod 8) of the eight stage rows of slice s in 3-bit fields, rbo the
      // cell-relative starts of the four output rows of slice s - 2
      uint32_t shw = 0;
#pragma unroll
      for ( int jj = 0; jj < R + 4; ++jj ) shw |= uint32_t( ( cb + cidx( N, 0, y0 - 2 + jj, za - 2 ) + x0 - 2 ) & 7 ) << ( 3 * jj );
      int rbo[R];
#pragma unroll
      for ( int j = 0; j < R; ++j ) rbo[j] = int( cidx( N, 0, y0 + j, za - 4 ) );
      A acc[5][R][2];  // [slot k: output slice s-2+k][row][point]
#pragma unroll
      for ( int k = 0; k < 5; ++k )
#pragma unroll
         for ( int j = 0; j < R; ++j ) acc[k][j][0] = acc[k][j][1] = A( 0 );
      // one slice: slice s (parity SP) folded into slots KO .. KO+4 (outputs s-2 .. s+2), then the
      // stage is handed back and output slice s-2 (slot KO) written
      auto slice = [&]( int s, auto sp_c, auto ko_c ) -> bool {
         constexpr int SP = decltype( sp_c )::value, KO = decltype( ko_c )::value;
         if ( !__all_sync( 0xffffffffu, mbar_wait_bounded( &full[cst], cph, nullptr ) ) ) return false;
         const T* Rg = ring + cst * Cfg::stage;
         static_for< 0, R + 4 >( [&]( auto jj_c ) {
            constexpr int JJ = decltype( jj_c )::value;
            const int     sh = int( ( shw >> ( 3 * JJ ) ) & ( AL - 1 ) );  // shift of the row in its stage row
            A             val[6];  // values at x0 - 2 + 2 lane + i
            load_row6( Rg + JJ * RW + 2 * lane, sh, val );
            static_for< 0, R >( [&]( auto j_c ) {
               constexpr int J  = decltype( j_c )::value;
               constexpr int DY = JJ - 2 - J;
               if constexpr ( DY >= -2 && DY <= 2 )
                  static_for< 0, 5 >( [&]( auto k_c ) {
                     constexpr int KS = decltype( k_c )::value;  // output slice s - 2 + KS
                     constexpr int DZ = 2 - KS;
                     static_for< 0, 2 >( [&]( auto p_c ) {
                        constexpr int PP = decltype( p_c )::value;
                        // parity class of the output point (x0 + 2 lane + PP, y0 + J, s - 2 + KS); x0, y0 odd
                        constexpr int KC = ( ( 1 + PP ) & 1 ) | ( ( ( 1 + J ) & 1 ) << 1 ) | ( ( ( SP + KS ) & 1 ) << 2 );
                        constexpr int E0 = kP2Pat.rng[KC][DZ + 2][DY + 2][0], E1 = kP2Pat.rng[KC][DZ + 2][DY + 2][1];
                        WVec_t< A > wv;
                        static_for< E0, E1 >( [&]( auto e_c ) {
                           constexpr int EI = decltype( e_c )::value;
                           constexpr int WI = kP2Pat.base[KC] + EI;
                           constexpr int I  = kP2Pat.off[WI][0] + 2 + PP;
                           constexpr int VW = WVec< A >::n;
                           // weights in 16-byte vectors: one shared load per vector of the group
                           if constexpr ( EI == E0 || WI % VW == 0 ) wv = *reinterpret_cast< const WVec_t< A >* >( Wsm + WI / VW * VW );
                           acc[KO + KS][J][PP] += vget< WI % VW >( wv ) * val[I];
                        } );
                     } );
                  } );
            } );
         } );
         // every lane has read the stage: hand it back to the async proxy and refill it
         asm volatile( "fence.proxy.async.shared::cta;" ::: "memory" );
         __syncwarp();
         ++ld;
         if ( ++cst == D ) cst = 0, cph ^= 1u;
         issue();
         const int z = s - 2;  // complete
         if ( z >= za && z <= zb )
         {
            static_for< 0, R >( [&]( auto j_c ) {
               constexpr int J  = decltype( j_c )::value;
               const int     y  = y0 + J;
               const int     xl = x0 + 2 * lane;
               if ( y + z <= N - 2 )
               {
                  const int64_t rb = cb + rbo[J];
                  static_for< 0, 2 >( [&]( auto p_c ) {
                     constexpr int PP = decltype( p_c )::value;
                     constexpr int KX = ( ( 1 + PP ) & 1 ) | ( ( ( 1 + J ) & 1 ) << 1 ) | ( ( SP & 1 ) << 2 );
                     const int     x  = xl + PP;
                     if ( x + y + z <= N - 1 )
                        stencil_epilogue< T, A, OP >( rb + x, acc[KO][J][PP], Wsm[kP2cEntries + KX], src, v1, v2, dst, a0, a1 );
                  } );
               }
            } );
         }
         // advance the row starts to slice s + 1 (stage rows) and s - 1 (output rows)
         const uint32_t ts = uint32_t( int64_t( N + 1 - s ) * ( N + 2 - s ) / 2 );
         uint32_t       nw = 0;
#pragma unroll
         for ( int jj = 0; jj < R + 4; ++jj )
            nw |= ( ( ( shw >> ( 3 * jj ) ) + ts - uint32_t( y0 - 2 + jj ) ) & 7u ) << ( 3 * jj );
         shw          = nw;
         const int tz = int( int64_t( N + 3 - s ) * ( N + 4 - s ) / 2 );  // tri(N + 1 - (s - 2))
#pragma unroll
         for ( int j = 0; j < R; ++j ) rbo[j] += tz - ( y0 + j );
         return true;
      };
      using I0 = std::integral_constant< int, 0 >;
      using I1 = std::integral_constant< int, 1 >;
      // after each slice, outputs s-1 .. s+2 move down one slot and slot 4 starts output s+3
      auto step = [&]( int s, auto sp_c ) -> bool {
         if ( !slice( s, sp_c, I0{} ) ) return false;
#pragma unroll
         for ( int k = 0; k < 4; ++k )
#pragma unroll
            for ( int j = 0; j < R; ++j ) acc[k][j][0] = acc[k + 1][j][0], acc[k][j][1] = acc[k + 1][j][1];
#pragma unroll
         for ( int j = 0; j < R; ++j ) acc[4][j][0] = acc[4][j][1] = A( 0 );
         return true;
      };
      // one call site per parity, so both instantiations are inlined
      bool ok = true;
      for ( int s = za - 2; ok && s <= zb + 2; ++s )
      {
         if ( s & 1 ) ok = step( s, I1{} );
         else ok = step( s, I0{} );
      }
      if ( !ok ) return fail();
   }
}

// ---------------------------------------------------------------------------------------------
// device: boundary owners
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ bool p2c_inside( int faces, int dx, int dy, int dz )
{
   return !( ( ( faces & 1 ) && dz < 0 ) || ( ( faces & 2 ) && dy < 0 ) || ( ( faces & 4 ) && dx < 0 ) ||
             ( ( faces & 8 ) && dx + dy + dz > 0 ) );
}

template < typename T, typename A, int OP >
__global__ void __launch_bounds__( 256 ) k_p2c_bnd( LevelView v, const A* __restrict__ W, const int4* __restrict__ tasks, TaskSegments seg,
                                                     uint32_t flag, int copy_unflagged, const T* __restrict__ src, const T* __restrict__ v1,
                                                     T* v2, T* dst, A a0, A a1 )
{
   int t = blockIdx.x * blockDim.x + threadIdx.x, at = -1;
#pragma unroll
   for ( int g = 0; g < 4; ++g )
   {
      if ( at < 0 && t < seg.count[g] ) at = seg.start[g] + t;
      if ( at < 0 ) t -= seg.count[g];
   }
   if ( at < 0 ) return;
   const int4    tk    = tasks[at];
   const int     b     = tk.x, i = tk.y, j = tk.z, N = v.n;
   const int64_t owner = owner_slot( v, b, i, j );
   if ( !( v.bc[b] & flag ) )
   {
      if ( !copy_unflagged ) return;
      if constexpr ( OP == OP_JAC || OP == OP_CHEB0 ) write_through( v, dst, b, i, j, owner, A( ldv( src + owner ) ) );
      else if constexpr ( OP == OP_CHEBI ) write_through( v, dst, b, i, j, owner, A( ldc( v2 + owner ) ) );
      return;
   }
   A acc = A( 0 ), diag = A( 0 );
   for ( int q = v.inc_begin[b]; q < v.inc_begin[b + 1]; ++q )
   {
      const Incidence I = v.inc[q];
      int             x, y, z;
      inc_point( I, N, i, j, x, y, z );
      const int      k     = ( x & 1 ) | ( ( y & 1 ) << 1 ) | ( ( z & 1 ) << 2 );
      const int      faces = c_p2c_faces[I.cls];
      const int      e0    = g_p2c_base[k], ne = g_p2c_base[k + 8];
      const A*       w     = W + size_t( I.cell ) * kP2cCellStride + ( I.cls == 0 ? 0 : kP2cInterior + ( I.cls - 1 ) * kP2cEntries ) + e0;
      const T*       s     = src + v.cell_off[I.cell];
      A              part  = A( 0 );
      // cell-relative starts of the slices z-2 .. z+2 (32-bit: the host limits the level), from
      // slice z by the slice sizes tri(N+1-z') = (N+1-z')(N+2-z')/2
      const int w1 = N + 1;
      int       S[5];
      S[2] = int( cidx( N, 0, 0, z ) );
      S[3] = S[2] + ( w1 - z ) * ( w1 - z + 1 ) / 2;
      S[4] = S[3] + ( w1 - z - 1 ) * ( w1 - z ) / 2;
      S[1] = S[2] - ( w1 - z + 1 ) * ( w1 - z + 2 ) / 2;
      S[0] = S[1] - ( w1 - z + 2 ) * ( w1 - z + 3 ) / 2;
      // entries are sorted by (dz, dy): the row start is recomputed only when that pair changes
      int pr = 0x7fffffff, rb = 0;
      for ( int e = 0; e < ne; ++e )
      {
         const char4 o = g_p2c_off[e0 + e];
         if ( !p2c_inside( faces, o.x, o.y, o.z ) ) continue;
         const int r = o.y * 8 + o.z;
         if ( r != pr )
         {
            const int yy = y + o.y, zz = z + o.z;
            rb = S[o.z + 2] + yy * ( w1 - zz ) - ( yy * ( yy - 1 ) ) / 2;  // start of row yy of slice zz
            pr = r;
         }
         part += w[e] * A( ldv( s + rb + x + o.x ) );
      }
      acc += part;
      diag += w[g_p2c_base[k + 16]];
   }
   const A invd = A( 1 ) / diag;
   if constexpr ( OP == OP_APPLY ) write_through( v, dst, b, i, j, owner, acc );
   else if constexpr ( OP == OP_APPLY_ADD ) write_through( v, dst, b, i, j, owner, A( ldc( dst + owner ) ) + acc );
   else if constexpr ( OP == OP_RESID ) write_through( v, dst, b, i, j, owner, A( ldv( v1 + owner ) ) - acc );
   else if constexpr ( OP == OP_JAC )
      write_through( v, dst, b, i, j, owner, A( ldv( src + owner ) ) + a0 * ( invd * ( A( ldv( v1 + owner ) ) - acc ) ) );
   else if constexpr ( OP == OP_CHEB0 ) write_through( v, dst, b, i, j, owner, invd * ( A( ldv( v1 + owner ) ) - acc ) );
   else if constexpr ( OP == OP_CHEBI )
   {
      write_through( v, dst, b, i, j, owner, invd * acc );
      write_through( v, v2, b, i, j, owner, A( ldc( v2 + owner ) ) + a0 * A( ldv( src + owner ) ) );
   }
   else if constexpr ( OP == OP_CHEBL )
      write_through( v, v2, b, i, j, owner, ( A( ldc( v2 + owner ) ) + a0 * A( ldv( src + owner ) ) ) + a1 * ( invd * acc ) );
   else if constexpr ( OP == OP_DINV_APPLY ) write_through( v, dst, b, i, j, owner, invd * acc );
}

// ---------------------------------------------------------------------------------------------
// host: launch
// ---------------------------------------------------------------------------------------------
template < typename T, typename A, int OP >
static void p2c_attr_one()
{
   check_cuda( cudaFuncSetAttribute( k_p2c_sweep< T, A, OP >, cudaFuncAttributeMaxDynamicSharedMemorySize, int( P2cCfg< T, A >::smem_bytes ) ),
               "cudaFuncSetAttribute(P2 sweep)" );
}

template < typename T, typename A >
static void p2c_attr_type()
{
   p2c_attr_one< T, A, OP_APPLY >();
   p2c_attr_one< T, A, OP_APPLY_ADD >();
   p2c_attr_one< T, A, OP_RESID >();
   p2c_attr_one< T, A, OP_JAC >();
   p2c_attr_one< T, A, OP_CHEB0 >();
   p2c_attr_one< T, A, OP_CHEBI >();
   p2c_attr_one< T, A, OP_CHEBL >();
   p2c_attr_one< T, A, OP_DINV_APPLY >();
}

static void p2c_attributes_all()
{
   p2c_attr_type< double, double >();
   p2c_attr_type< float, float >();
   p2c_attr_type< __half, float >();
}

template < typename T, typename A, int OP >
static void run_p2c( Context* ctx, const LevelView& v, const A* W, const int4* tasks, int nC, const StencilArgs& a )
{
   using Cfg            = P2cCfg< T, A >;
   const T*           src = (const T*) a.src;
   const T*           v1  = (const T*) a.v1;
   T*                 v2  = (T*) a.v2;
   T*                 dst = (T*) a.dst;
   const TaskSegments seg = task_segments( v, a.flag, a.copy_unflagged );
   const int          nt  = seg.count[0] + seg.count[1] + seg.count[2] + seg.count[3];
   // boundary owners and cell interiors write disjoint slots and read only src and their own slots of
   // the second vector, so the two kernels run one after the other on the context stream
   if ( nt > 0 )
   {
      k_p2c_bnd< T, A, OP ><<< ( nt + 255 ) / 256, 256, 0, ctx->stream >>>( v, W, tasks, seg, a.flag, a.copy_unflagged, src, v1, v2, dst, A( a.a0 ),
                                                                            A( a.a1 ) );
      ++ctx->launches;
   }
   const int nw = v.nswarps[0];
   if ( nw > 0 && nC > 0 && v.n >= 4 )
   {
      // the sweep keeps cell-relative row starts in 32-bit integers
      if ( tet_size( int64_t( v.n ) + 1 ) > int64_t( 0x7fffffff ) ) throw std::invalid_argument( "P2 constant operator: level too large" );
      k_p2c_sweep< T, A, OP ><<< nw / kP2cWarps, kP2cWarps * 32, Cfg::smem_bytes, ctx->stream >>>( v, W, a.flag, src, v1, v2, dst, A( a.a0 ),
                                                                                              A( a.a1 ), nC, ctx->d_error );
      ++ctx->launches;
   }
   check_cuda( cudaGetLastError(), "P2 constant stencil launch" );
}

template < typename T, typename A >
static void dispatch_p2c( Context* ctx, const LevelView& v, const A* W, const int4* tasks, int nC, const StencilArgs& a )
{
   switch ( a.op )
   {
   case OP_APPLY: return run_p2c< T, A, OP_APPLY >( ctx, v, W, tasks, nC, a );
   case OP_APPLY_ADD: return run_p2c< T, A, OP_APPLY_ADD >( ctx, v, W, tasks, nC, a );
   case OP_RESID: return run_p2c< T, A, OP_RESID >( ctx, v, W, tasks, nC, a );
   case OP_JAC: return run_p2c< T, A, OP_JAC >( ctx, v, W, tasks, nC, a );
   case OP_CHEB0: return run_p2c< T, A, OP_CHEB0 >( ctx, v, W, tasks, nC, a );
   case OP_CHEBI: return run_p2c< T, A, OP_CHEBI >( ctx, v, W, tasks, nC, a );
   case OP_CHEBL: return run_p2c< T, A, OP_CHEBL >( ctx, v, W, tasks, nC, a );
   case OP_DINV_APPLY: return run_p2c< T, A, OP_DINV_APPLY >( ctx, v, W, tasks, nC, a );
   default: throw std::invalid_argument( "unknown stencil operation" );
   }
}

void launch_p2_constant( Context* ctx, Mesh* m, Operator* op, int Ls, int dtype, const StencilArgs& a )
{
   ensure_p2_constant_device();
   P2cLevel& pl = op->p2c.at( Ls );
   ensure_p2_constant_tables( pl );
   const LevelView v  = make_view( m, Ls );
   const int       nC = m->topo.nC;
   if ( dtype == F64 ) dispatch_p2c< double, double >( ctx, v, pl.d_W, pl.d_tasks, nC, a );
   else if ( dtype == F32 ) dispatch_p2c< float, float >( ctx, v, pl.d_Wf, pl.d_tasks, nC, a );
   else dispatch_p2c< __half, float >( ctx, v, pl.d_Wf, pl.d_tasks, nC, a );
}

}  // namespace hyb
