// Elementwise P1 operator for -div(k grad u) with optional icosahedral-shell blending (sm_100a).
//
// Reference: P1ElementwiseOperator with the HyTeG form p1_div_k_grad_blending_q3
// (src/hyteg/elementwiseoperators/P1ElementwiseOperator.cpp, src/hyteg/forms/form_hyteg_generated/p1/
// p1_div_k_grad_blending_q3.cpp): every micro-cell gets its 4x4 element matrix from a 5-point
// degree-3 quadrature (Yu's rule: centroid weight -2/15, four points with barycentric weights
// (1/2, 1/6, 1/6, 1/6) and weight 3/40), the coefficient is evaluated at the blended (physical)
// quadrature point and the blending Jacobian enters the gradients and the volume factor.
//
// GPU scheme: the micro-cells of a macro-cell are grouped by the parity of their anchor index; two
// anchors of the same parity differ by at least 2 in some coordinate, so the micro-cells of one
// parity class never share a vertex and a thread can add its element contributions without atomics.
// Eight passes (one per parity) accumulate A x into a scratch array laid out like the function; a
// combine kernel then applies the same epilogues as the constant-stencil path (apply, residual,
// Jacobi, Chebyshev steps) with a per-DoF inverse diagonal, summing the cell copies of face, edge
// and vertex DoFs into their owners (the additive communication of the reference).  Deterministic:
// the order of every sum is fixed.  The path is FP64-compute-bound.
#include "hyb_internal.hpp"

#include <cmath>
#include <stdexcept>

namespace hyb {

// ---------------------------------------------------------------------------------------------
// host: cell geometry and IcosahedralShellMap classification
// ---------------------------------------------------------------------------------------------
static void cross3( const double* a, const double* b, double* c )
{
   c[0] = a[1] * b[2] - a[2] * b[1];
   c[1] = a[2] * b[0] - a[0] * b[2];
   c[2] = a[0] * b[1] - a[1] * b[0];
}

// IcosahedralShellMap::classifyVertices (geometry/IcosahedralShellMap.hpp:606-705): the two vertices
// on a radial ray become ref/ray (ref is the single outer vertex of an outward tet, the single inner
// vertex of an inward tet); skew tets borrow the classification of a non-skew tet of the same prism.
static void classify_shell( const Topology& t, int c, CellGeom& g, int depth = 0 )
{
   if ( depth > 4 ) throw std::runtime_error( "shell blending: cannot classify macro-cell" );
   double P[4][3], rad[4];
   for ( int k = 0; k < 4; ++k )
   {
      for ( int d = 0; d < 3; ++d ) P[k][d] = t.vx[t.cv[c][k]][d];
      rad[k] = std::sqrt( P[k][0] * P[k][0] + P[k][1] * P[k][1] + P[k][2] * P[k][2] );
   }
   double inner = rad[0], outer = rad[0];
   for ( int k = 1; k < 4; ++k ) inner = std::min( inner, rad[k] ), outer = std::max( outer, rad[k] );
   const double eps     = ( outer - inner ) * 0.001;
   int          n_outer = 0;
   for ( int k = 0; k < 4; ++k ) n_outer += ( outer - rad[k] ) < eps ? 1 : 0;
   int iref = -1, iray = -1;
   for ( int k = 0; k < 4 && iref < 0; ++k )
      for ( int j = k + 1; j < 4 && iref < 0; ++j )
      {
         double cr[3];
         cross3( P[k], P[j], cr );
         const double s = rad[k] * rad[j];
         if ( std::fabs( cr[0] ) / s <= 1e-14 && std::fabs( cr[1] ) / s <= 1e-14 && std::fabs( cr[2] ) / s <= 1e-14 ) iref = k, iray = j;
      }
   if ( iref < 0 ) throw std::runtime_error( "shell blending: no radial vertex pair in a macro-cell (not a shell mesh?)" );
   if ( n_outer == 2 )
   {
      const int vref = t.cv[c][iref], vray = t.cv[c][iray];
      for ( int f : t.cf[c] )
      {
         const auto& fv     = t.fv[f];
         const bool  hasRef = fv[0] == vref || fv[1] == vref || fv[2] == vref;
         const bool  hasRay = fv[0] == vray || fv[1] == vray || fv[2] == vray;
         if ( !( hasRef && hasRay ) )
            for ( int cc : t.f_cells[f] )
               if ( cc != c ) return classify_shell( t, cc, g, depth + 1 );
      }
      throw std::runtime_error( "shell blending: no non-skew neighbour" );
   }
   int rest[2], nr = 0;
   for ( int k = 0; k < 4; ++k )
      if ( k != iref && k != iray ) rest[nr++] = k;
   const int ithr = rest[1], ifor = rest[0];
   if ( ( n_outer == 1 && rad[iref] < rad[iray] ) || ( n_outer == 3 && rad[iref] > rad[iray] ) ) std::swap( iref, iray );
   double a[3], b[3];
   for ( int d = 0; d < 3; ++d )
   {
      g.ray[d] = P[iray][d];
      a[d]     = P[ithr][d] - P[iray][d];
      b[d]     = P[ifor][d] - P[iray][d];
   }
   cross3( a, b, g.bxc );
   g.volT    = ( P[iref][0] - P[iray][0] ) * g.bxc[0] + ( P[iref][1] - P[iray][1] ) * g.bxc[1] + ( P[iref][2] - P[iray][2] ) * g.bxc[2];
   g.rad_ray = rad[iray];
   g.rad_ref = rad[iref];
}

void cell_geometry( const Topology& t, int c, int blending, CellGeom& g )
{
   g = CellGeom{};
   for ( int k = 0; k < 4; ++k )
      for ( int d = 0; d < 3; ++d ) g.P[k][d] = t.vx[t.cv[c][k]][d];
   g.blend = blending;
   if ( blending == 1 ) classify_shell( t, c, g );
}

void build_elementwise_operator( Operator* A )
{
   const Topology& t = A->mesh->topo;
   A->geom.assign( t.nC, CellGeom{} );
   for ( int c = 0; c < t.nC; ++c ) cell_geometry( t, c, A->blending, A->geom[c] );
}

// ---------------------------------------------------------------------------------------------
// device: blending, coefficient and element matrix
// ---------------------------------------------------------------------------------------------
__constant__ double c_yu5_pts[5][3] = { { 0.25, 0.25, 0.25 },
                                        { 1.0 / 6.0, 1.0 / 6.0, 1.0 / 6.0 },
                                        { 0.5, 1.0 / 6.0, 1.0 / 6.0 },
                                        { 1.0 / 6.0, 0.5, 1.0 / 6.0 },
                                        { 1.0 / 6.0, 1.0 / 6.0, 0.5 } };
__constant__ double c_yu5_w[5]      = { -2.0 / 15.0, 3.0 / 40.0, 3.0 / 40.0, 3.0 / 40.0, 3.0 / 40.0 };

template < typename A >
__device__ __forceinline__ A coeff_eval( const Coefficient& k, const A* P )
{
   if ( k.kind == 0 ) return A( k.value );
   if ( k.kind == 2 )  // radial profile exp(amp (value - |x|) / freq)
      return exp( A( k.amp ) * ( A( k.value ) - sqrt( P[0] * P[0] + P[1] * P[1] + P[2] * P[2] ) ) / A( k.freq ) );
   const A tp = A( 2.0 * 3.14159265358979323846 * k.freq );
   return exp( A( k.amp ) * sin( tp * ( P[0] + A( k.phase[0] ) ) ) * cos( tp * ( P[1] + A( k.phase[1] ) ) ) *
               sin( tp * ( P[2] + A( k.phase[2] ) ) ) );
}

// IcosahedralShellMap: F(x) = x r(x)/|x|, r(x) = r_ray + lambda(x) (r_ref - r_ray) with lambda the
// barycentric weight of the ref vertex; DF = s I + x (grad s)^T with s = r/|x|.
template < typename A >
__device__ __forceinline__ void shell_map( const CellGeom& g, const A* X, A* F, A DF[3][3] )
{
   const A dx = X[0] - A( g.ray[0] ), dy = X[1] - A( g.ray[1] ), dz = X[2] - A( g.ray[2] );
   const A lam_s = ( dx * A( g.bxc[0] ) + dy * A( g.bxc[1] ) + dz * A( g.bxc[2] ) ) / A( g.volT );
   const A sgn   = lam_s < A( 0 ) ? A( -1 ) : A( 1 );
   const A dr    = A( g.rad_ref ) - A( g.rad_ray );
   const A R     = A( g.rad_ray ) + fabs( lam_s ) * dr;
   const A r2    = X[0] * X[0] + X[1] * X[1] + X[2] * X[2];
   const A r     = sqrt( r2 );
   const A s     = R / r;
   A       gs[3];
   for ( int j = 0; j < 3; ++j ) gs[j] = ( dr * sgn * A( g.bxc[j] ) / A( g.volT ) ) / r - R * X[j] / ( r2 * r );
   for ( int i = 0; i < 3; ++i )
   {
      F[i] = X[i] * s;
      for ( int j = 0; j < 3; ++j ) DF[i][j] = ( i == j ? s : A( 0 ) ) + X[i] * gs[j];
   }
}

// P1 PSPG stabilisation element matrix of an affine micro-cell (form p1_tet_pspg_tet.h, whose inverted
// diagonal P1PSPGInvDiagOperator scales the Uzawa pressure update): -(|T|^(2/3) / 12) |T| grad l_i .
// grad l_j, the l_i barycentric coordinates and |T| the volume.  Exact (constant integrand).
template < typename A >
__device__ __forceinline__ void p1_pspg_element( const A X[4][3], A K[4][4] )
{
   A J[3][3];
   for ( int r = 0; r < 3; ++r )
      for ( int c = 0; c < 3; ++c ) J[r][c] = X[c + 1][r] - X[0][r];
   const A c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1], c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2],
           c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
   const A det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
   // rows of J^-1 are the gradients of l_1, l_2, l_3
   A G[4][3];
   G[1][0] = c00 / det, G[1][1] = ( J[0][2] * J[2][1] - J[0][1] * J[2][2] ) / det, G[1][2] = ( J[0][1] * J[1][2] - J[0][2] * J[1][1] ) / det;
   G[2][0] = c01 / det, G[2][1] = ( J[0][0] * J[2][2] - J[0][2] * J[2][0] ) / det, G[2][2] = ( J[0][2] * J[1][0] - J[0][0] * J[1][2] ) / det;
   G[3][0] = c02 / det, G[3][1] = ( J[0][1] * J[2][0] - J[0][0] * J[2][1] ) / det, G[3][2] = ( J[0][0] * J[1][1] - J[0][1] * J[1][0] ) / det;
   for ( int d = 0; d < 3; ++d ) G[0][d] = -( G[1][d] + G[2][d] + G[3][d] );
   const A vol = fabs( det ) / A( 6 );
   const A f   = -( pow( vol, A( 2.0 / 3.0 ) ) / A( 12 ) ) * vol;
   for ( int i = 0; i < 4; ++i )
      for ( int j = 0; j < 4; ++j ) K[i][j] = f * ( G[i][0] * G[j][0] + G[i][1] * G[j][1] + G[i][2] * G[j][2] );
}

// Minus the lumped P1 mass matrix weighted by 1/k, diag_i = -int l_i / k over the (blended) micro-cell
// (Yu's 5-point degree-3 rule): with k the viscosity, the scaling of the pressure update that follows
// the viscosity-weighted pressure mass matrix, the usual approximation of the Schur complement
// B A^-1 B^T for variable viscosity (negative like the PSPG diagonal, so the Uzawa update keeps its sign).
template < typename A >
__device__ __forceinline__ void p1_lumped_mass_inv_k_element( const CellGeom& g, const Coefficient& kc, const A X[4][3], A K[4][4] )
{
   A J[3][3];
   for ( int r = 0; r < 3; ++r )
      for ( int c = 0; c < 3; ++c ) J[r][c] = X[c + 1][r] - X[0][r];
   for ( int i = 0; i < 4; ++i )
      for ( int j = 0; j < 4; ++j ) K[i][j] = A( 0 );
#pragma unroll 1
   for ( int q = 0; q < 5; ++q )
   {
      const A xi[3] = { A( c_yu5_pts[q][0] ), A( c_yu5_pts[q][1] ), A( c_yu5_pts[q][2] ) };
      A       Xq[3];
      for ( int r = 0; r < 3; ++r ) Xq[r] = X[0][r] + J[r][0] * xi[0] + J[r][1] * xi[1] + J[r][2] * xi[2];
      A M[3][3], Fq[3];
      if ( g.blend == 1 )
      {
         A DF[3][3];
         shell_map( g, Xq, Fq, DF );
         for ( int r = 0; r < 3; ++r )
            for ( int c = 0; c < 3; ++c ) M[r][c] = DF[r][0] * J[0][c] + DF[r][1] * J[1][c] + DF[r][2] * J[2][c];
      }
      else
         for ( int r = 0; r < 3; ++r )
         {
            Fq[r] = Xq[r];
            for ( int c = 0; c < 3; ++c ) M[r][c] = J[r][c];
         }
      const A det = M[0][0] * ( M[1][1] * M[2][2] - M[1][2] * M[2][1] ) - M[0][1] * ( M[1][0] * M[2][2] - M[1][2] * M[2][0] ) +
                    M[0][2] * ( M[1][0] * M[2][1] - M[1][1] * M[2][0] );
      const A f     = A( c_yu5_w[q] ) * fabs( det ) / coeff_eval( kc, Fq );
      const A lam[4] = { A( 1 ) - xi[0] - xi[1] - xi[2], xi[0], xi[1], xi[2] };
      for ( int i = 0; i < 4; ++i ) K[i][i] -= f * lam[i];
   }
}

template < typename A >
__device__ __forceinline__ void p1_divkgrad_element( const CellGeom& g, const Coefficient& kc, const A X[4][3], A K[4][4] )
{
   A J[3][3];
   for ( int r = 0; r < 3; ++r )
      for ( int c = 0; c < 3; ++c ) J[r][c] = X[c + 1][r] - X[0][r];
   for ( int i = 0; i < 4; ++i )
      for ( int j = 0; j < 4; ++j ) K[i][j] = A( 0 );
#pragma unroll 1
   for ( int q = 0; q < 5; ++q )
   {
      A Xq[3];
      for ( int r = 0; r < 3; ++r )
         Xq[r] = X[0][r] + J[r][0] * A( c_yu5_pts[q][0] ) + J[r][1] * A( c_yu5_pts[q][1] ) + J[r][2] * A( c_yu5_pts[q][2] );
      A M[3][3], Fq[3];
      if ( g.blend == 1 )
      {
         A DF[3][3];
         shell_map( g, Xq, Fq, DF );
         for ( int r = 0; r < 3; ++r )
            for ( int c = 0; c < 3; ++c ) M[r][c] = DF[r][0] * J[0][c] + DF[r][1] * J[1][c] + DF[r][2] * J[2][c];
      }
      else
      {
         for ( int r = 0; r < 3; ++r )
         {
            Fq[r] = Xq[r];
            for ( int c = 0; c < 3; ++c ) M[r][c] = J[r][c];
         }
      }
      // inverse of M: rows of M^-1 are the reference gradients mapped to physical space
      const A c00 = M[1][1] * M[2][2] - M[1][2] * M[2][1];
      const A c01 = M[1][2] * M[2][0] - M[1][0] * M[2][2];
      const A c02 = M[1][0] * M[2][1] - M[1][1] * M[2][0];
      const A det = M[0][0] * c00 + M[0][1] * c01 + M[0][2] * c02;
      const A id  = A( 1 ) / det;
      A       Mi[3][3];
      Mi[0][0] = c00 * id;
      Mi[1][0] = c01 * id;
      Mi[2][0] = c02 * id;
      Mi[0][1] = ( M[0][2] * M[2][1] - M[0][1] * M[2][2] ) * id;
      Mi[1][1] = ( M[0][0] * M[2][2] - M[0][2] * M[2][0] ) * id;
      Mi[2][1] = ( M[0][1] * M[2][0] - M[0][0] * M[2][1] ) * id;
      Mi[0][2] = ( M[0][1] * M[1][2] - M[0][2] * M[1][1] ) * id;
      Mi[1][2] = ( M[0][2] * M[1][0] - M[0][0] * M[1][2] ) * id;
      Mi[2][2] = ( M[0][0] * M[1][1] - M[0][1] * M[1][0] ) * id;
      // gradient of phi_i (i = 1..3) is row i-1 of Mi; phi_0 is minus their sum
      A G[4][3];
      for ( int d = 0; d < 3; ++d )
      {
         G[1][d] = Mi[0][d];
         G[2][d] = Mi[1][d];
         G[3][d] = Mi[2][d];
         G[0][d] = -( G[1][d] + G[2][d] + G[3][d] );
      }
      const A f = A( c_yu5_w[q] ) * coeff_eval( kc, Fq ) * fabs( det );
      for ( int i = 0; i < 4; ++i )
         for ( int j = i; j < 4; ++j ) K[i][j] += f * ( G[i][0] * G[j][0] + G[i][1] * G[j][1] + G[i][2] * G[j][2] );
   }
   for ( int i = 0; i < 4; ++i )
      for ( int j = 0; j < i; ++j ) K[i][j] = K[j][i];
}

}  // namespace hyb

namespace hyb {

// micro-cell types: vertex offsets and anchor range shift (CellDoFIndexing.hpp:155-198)
__constant__ int c_mc_off[6][4][3] = {
    { { 0, 0, 0 }, { 1, 0, 0 }, { 0, 1, 0 }, { 0, 0, 1 } }, { { 1, 0, 0 }, { 1, 1, 0 }, { 0, 1, 0 }, { 1, 0, 1 } },
    { { 1, 0, 0 }, { 0, 1, 0 }, { 1, 0, 1 }, { 0, 0, 1 } }, { { 1, 1, 0 }, { 1, 1, 1 }, { 0, 1, 1 }, { 1, 0, 1 } },
    { { 1, 0, 1 }, { 0, 1, 1 }, { 0, 0, 1 }, { 0, 1, 0 } }, { { 0, 1, 0 }, { 1, 1, 0 }, { 1, 0, 1 }, { 0, 1, 1 } } };
__constant__ int c_mc_shift[6] = { 0, 1, 1, 2, 1, 1 };
// stencil direction (index into kVarDirs) from vertex i to vertex j of micro-cell type ty
__constant__ int8_t c_mc_dir[6][4][4];
// the 15 stencil directions in the order of the constant-stencil weights
static const int kVarDirs[15][3] = { { 0, 0, 0 },  { -1, 0, 0 }, { 1, 0, 0 },  { 0, -1, 0 }, { 0, 1, 0 },
                                     { 0, 0, -1 }, { 0, 0, 1 },  { -1, 1, 0 }, { 1, -1, 0 }, { -1, 0, 1 },
                                     { 1, 0, -1 }, { 0, -1, 1 }, { 0, 1, -1 }, { 1, -1, 1 }, { -1, 1, -1 } };
__constant__ int8_t c_var_dir[15][3];

__device__ __forceinline__ double ld_any( const double* p ) { return *p; }
__device__ __forceinline__ float  ld_any( const float* p ) { return *p; }
__device__ __forceinline__ float  ld_any( const __half* p ) { return __half2float( *p ); }
__device__ __forceinline__ void   st_any( double* p, double v ) { *p = v; }
__device__ __forceinline__ void   st_any( float* p, float v ) { *p = v; }
__device__ __forceinline__ void   st_any( __half* p, float v ) { *p = __float2half_rn( v ); }

// One parity pass: warp per half-grid row (y, z) of anchors with y = py mod 2, z = pz mod 2, lanes
// over x = px + 2k.  MODE 0 accumulates A src, MODE 1 the diagonal.
// MODE 0: y += K x with K computed on the fly; 1: diagonal of K; 2: compute K and store its upper
// triangle; 3: y += K x with K read from storage; 4: add K into the assembled stencils of the
// cell-array slots of its vertices (kst = stencils, kstride = level size).  Stored entry v of micro-cell (cell c, type ty,
// anchor a) sits at kst[v * kstride + (c * 6 + ty) * tet(n) + cidx(n - 1, a)].
template < typename T, typename A, int MODE >
__global__ void __launch_bounds__( 256 ) k_elem_pass( int n, int nanch, const int* __restrict__ anch, const int64_t* __restrict__ cell_off,
                                                       const CellGeom* __restrict__ geom, Coefficient kc,
                                                       const T* __restrict__ src, A* __restrict__ acc, A* __restrict__ kst,
                                                       int64_t kstride, int64_t level_size, int* err )
{
   const int t = blockIdx.x * blockDim.x + threadIdx.x;  // one micro-cell anchor per thread
   const int c = blockIdx.y;
   if ( t >= nanch ) return;
   const int      a = anch[t];
   const int      x = a & 1023, y = ( a >> 10 ) & 1023, z = a >> 20;
   const CellGeom g  = geom[c];
   const int64_t  base = cell_off[c];
   const A        inv_n = A( 1.0 / double( n ) );
   A              st[3][3];  // computational steps per index direction (coordinateFromIndex)
   for ( int k = 0; k < 3; ++k )
      for ( int d = 0; d < 3; ++d ) st[k][d] = ( A( g.P[k + 1][d] ) - A( g.P[0][d] ) ) * inv_n;
      for ( int ty = 0; ty < 6; ++ty )
      {
         if ( x + y + z > n - 1 - c_mc_shift[ty] ) continue;
         int64_t idx[4];
         A       X[4][3];
         for ( int m = 0; m < 4; ++m )
         {
            const int vx = x + c_mc_off[ty][m][0], vy = y + c_mc_off[ty][m][1], vz = z + c_mc_off[ty][m][2];
            idx[m]       = base + cidx( n, vx, vy, vz );
            for ( int d = 0; d < 3; ++d ) X[m][d] = A( g.P[0][d] ) + st[0][d] * A( vx ) + st[1][d] * A( vy ) + st[2][d] * A( vz );
         }
         A K[4][4];
         const int64_t slot = ( int64_t( c ) * 6 + ty ) * tet_size( n ) + cidx( n - 1, x, y, z );
         // self-check: every node inside the level's vector and every stored slot inside its array;
         // a violation is recorded (error word 2) and the micro-cell skipped
         {
            bool bad = ( MODE == 2 || MODE == 3 ) && ( slot < 0 || slot >= kstride );
            for ( int m = 0; m < 4; ++m ) bad |= idx[m] < 0 || idx[m] >= level_size;
            if ( bad )
            {
               atomicExch( err, 2 );
               continue;
            }
         }
         if constexpr ( MODE == 3 )
         {
            int v = 0;
            for ( int i = 0; i < 4; ++i )
               for ( int j = i; j < 4; ++j, ++v ) K[i][j] = K[j][i] = kst[v * kstride + slot];
            A xl[4];
            for ( int m = 0; m < 4; ++m ) xl[m] = A( ld_any( src + idx[m] ) );
            for ( int i = 0; i < 4; ++i ) acc[idx[i]] += K[i][0] * xl[0] + K[i][1] * xl[1] + K[i][2] * xl[2] + K[i][3] * xl[3];
            continue;
         }
         if ( kc.kind == kCoeffPSPG ) p1_pspg_element( X, K );
         else if ( kc.element == kElemLumpedMassInvK ) p1_lumped_mass_inv_k_element( g, kc, X, K );
         else p1_divkgrad_element( g, kc, X, K );
         if constexpr ( MODE == 2 )
         {
            int v = 0;
            for ( int i = 0; i < 4; ++i )
               for ( int j = i; j < 4; ++j, ++v ) kst[v * kstride + slot] = K[i][j];
         }
         else if constexpr ( MODE == 0 )
         {
            A xl[4];
            for ( int m = 0; m < 4; ++m ) xl[m] = A( ld_any( src + idx[m] ) );
            for ( int i = 0; i < 4; ++i ) acc[idx[i]] += K[i][0] * xl[0] + K[i][1] * xl[1] + K[i][2] * xl[2] + K[i][3] * xl[3];
         }
         else if constexpr ( MODE == 1 )
            for ( int i = 0; i < 4; ++i ) acc[idx[i]] += K[i][i];
         else if constexpr ( MODE == 4 )
            for ( int i = 0; i < 4; ++i )
               for ( int j = 0; j < 4; ++j ) kst[int64_t( c_mc_dir[ty][i][j] ) * kstride + idx[i]] += K[i][j];
      }
}

// ---------------------------------------------------------------------------------------------
// P2 elementwise operators (P2ElementwiseOperator::apply / computeDiagonalOperatorValues,
// elementwiseoperators/P2ElementwiseOperator.cpp:109-318,418-567) with p2_div_k_grad_blending_q4.
// A P2 function on level L is stored on the node set of level L+1: the level-L micro-cell with
// vertices v0..v3 has its ten nodes at 2 v_i (vertices) and v_i + v_j (edge midpoints, edge order
// (2,3), (1,3), (1,2), (0,3), (0,2), (0,1)) in storage coordinates.  Element integrals use the
// degree-4, 11-point Xiao-Gimbutas rule on the tetrahedron, the rule the reference's form is
// generated with; its weights are derived here from exactness for all polynomials of degree <= 4.
// ---------------------------------------------------------------------------------------------
__constant__ double c_xg4_pts[11][3];
__constant__ double c_xg4_w[11];
__constant__ double c_p2_rgrad[11][10][3];  // reference gradients of the ten basis functions per point
__constant__ double c_p2_phi[11][10];       // values of the ten basis functions per point
__constant__ int    c_p2_edge[6][2] = { { 2, 3 }, { 1, 3 }, { 1, 2 }, { 0, 3 }, { 0, 2 }, { 0, 1 } };
// Stored P2 element matrices keep the 55 distinct entries of the symmetric 10x10 matrix in wrapped-
// diagonal order: block 0 (entries 0-9) the diagonal K(i, i); block s = 1..4 (entries 10 s + e) the
// entries K(e, (e + s) mod 10); block 5 (entries 50-54) K(e, e + 5) for e < 5.  Lane i of a ten-lane
// group then finds its row in blocks that the group reads as whole 80-byte runs.  c_p2_wrap maps the
// upper-triangle index r * 10 - r (r - 1) / 2 + (c - r) of (r, c), r <= c, to this order.
__constant__ int    c_p2_wrap[55];

static void p2_wrap_table( int w[55] )
{
   for ( int r = 0; r < 10; ++r )
      for ( int c = r; c < 10; ++c )
      {
         const int ut = r * 10 - r * ( r - 1 ) / 2 + ( c - r ), d = c - r;
         w[ut]        = d == 0 ? r : d <= 4 ? 10 * d + r : d == 5 ? 50 + r : 10 * ( 10 - d ) + c;
      }
}

// barycentric coordinates (l0, l1, l2, l3) of the rule's points (kept identical to the reference's
// generated form: the element integrals must agree); reference coordinates are (l1, l2, l3)
static const double kXG4Bary[11][4] = {
    { 0.17469405869723054, 0.04049050672759043, 0.01356070187980288, 0.7712547326953761 },
    { 0.08140491840285922, 0.752508507009655, 0.06809937093820666, 0.09798720364927911 },
    { 0.3044484024344971, 0.2402766649280726, 0.126801725915392, 0.3284732067220384 },
    { 0.7412288820936226, 0.0672232948933834, 0.03518392977359872, 0.1563638932393953 },
    { 0.053341239535745266, 0.419266313879513, 0.04778143555908666, 0.4796110110256551 },
    { 0.4329534904813558, 0.4507658760912768, 0.05945661629943383, 0.05682401712793367 },
    { 0.5380072039161857, 0.1294113737889104, 0.3301904148374645, 0.002391007457439365 },
    { 0.008991260093335729, 0.1215419913339278, 0.3064939884296903, 0.5629727601430461 },
    { 0.10660417256199362, 0.09720464458758327, 0.68439041545304, 0.1118007673973831 },
    { 0.3292329597426468, 0.02956949520647961, 0.3179035602133946, 0.323293984837479 },
    { 0.10384411641099309, 0.4327102390477686, 0.3538232392092971, 0.1096224053319412 } };

// weights w solving sum_q w_q xi_q^a = a1! a2! a3! / (|a|+3)! for all |a| <= 4 in the least-squares
// sense (Householder QR of the 35 x 11 moment matrix; exact for a degree-4 rule)
static void xg4_weights( double w[11] )
{
   const int           m = 35, n = 11;
   std::vector< double > A( m * n ), b( m );
   auto fact = []( int k ) {
      double f = 1;
      for ( int i = 2; i <= k; ++i ) f *= i;
      return f;
   };
   int row = 0;
   for ( int a = 0; a <= 4; ++a )
      for ( int bb = 0; bb <= 4 - a; ++bb )
         for ( int c = 0; c <= 4 - a - bb; ++c, ++row )
         {
            for ( int q = 0; q < n; ++q )
               A[row * n + q] = std::pow( kXG4Bary[q][1], a ) * std::pow( kXG4Bary[q][2], bb ) * std::pow( kXG4Bary[q][3], c );
            b[row] = fact( a ) * fact( bb ) * fact( c ) / fact( a + bb + c + 3 );
         }
   for ( int k = 0; k < n; ++k )
   {
      double nrm = 0;
      for ( int i = k; i < m; ++i ) nrm += A[i * n + k] * A[i * n + k];
      nrm = std::sqrt( nrm );
      const double alpha = A[k * n + k] > 0 ? -nrm : nrm;
      std::vector< double > v( m, 0.0 );
      for ( int i = k; i < m; ++i ) v[i] = A[i * n + k];
      v[k] -= alpha;
      double vv = 0;
      for ( int i = k; i < m; ++i ) vv += v[i] * v[i];
      if ( vv == 0 ) continue;
      for ( int j = k; j < n; ++j )
      {
         double d = 0;
         for ( int i = k; i < m; ++i ) d += v[i] * A[i * n + j];
         for ( int i = k; i < m; ++i ) A[i * n + j] -= 2 * d / vv * v[i];
      }
      double d = 0;
      for ( int i = k; i < m; ++i ) d += v[i] * b[i];
      for ( int i = k; i < m; ++i ) b[i] -= 2 * d / vv * v[i];
   }
   for ( int k = n - 1; k >= 0; --k )
   {
      double s = b[k];
      for ( int j = k + 1; j < n; ++j ) s -= A[k * n + j] * w[j];
      w[k] = s / A[k * n + k];
   }
}

void ensure_p2_constants()
{
   static PerDeviceOnce once;
   once.run( [] {
      double pts[11][3], w[11], g[11][10][3];
      xg4_weights( w );
      const double lg[4][3] = { { -1, -1, -1 }, { 1, 0, 0 }, { 0, 1, 0 }, { 0, 0, 1 } };
      const int    ed[6][2] = { { 2, 3 }, { 1, 3 }, { 1, 2 }, { 0, 3 }, { 0, 2 }, { 0, 1 } };
      for ( int q = 0; q < 11; ++q )
      {
         for ( int d = 0; d < 3; ++d ) pts[q][d] = kXG4Bary[q][d + 1];
         const double lam[4] = { 1.0 - pts[q][0] - pts[q][1] - pts[q][2], pts[q][0], pts[q][1], pts[q][2] };
         for ( int i = 0; i < 4; ++i )
            for ( int d = 0; d < 3; ++d ) g[q][i][d] = ( 4.0 * lam[i] - 1.0 ) * lg[i][d];
         for ( int e = 0; e < 6; ++e )
            for ( int d = 0; d < 3; ++d )
               g[q][4 + e][d] = 4.0 * ( lam[ed[e][0]] * lg[ed[e][1]][d] + lam[ed[e][1]] * lg[ed[e][0]][d] );
      }
      check_cuda( cudaMemcpyToSymbol( c_xg4_pts, pts, sizeof( pts ) ), "P2 constants (points)" );
      check_cuda( cudaMemcpyToSymbol( c_xg4_w, w, sizeof( w ) ), "P2 constants (weights)" );
      check_cuda( cudaMemcpyToSymbol( c_p2_rgrad, g, sizeof( g ) ), "P2 constants (gradients)" );
      double phi[11][10];
      for ( int q = 0; q < 11; ++q )
      {
         const double lam[4] = { 1.0 - pts[q][0] - pts[q][1] - pts[q][2], pts[q][0], pts[q][1], pts[q][2] };
         for ( int i = 0; i < 4; ++i ) phi[q][i] = lam[i] * ( 2.0 * lam[i] - 1.0 );
         for ( int e = 0; e < 6; ++e ) phi[q][4 + e] = 4.0 * lam[ed[e][0]] * lam[ed[e][1]];
      }
      check_cuda( cudaMemcpyToSymbol( c_p2_phi, phi, sizeof( phi ) ), "P2 constants (basis values)" );
      int wrap[55];
      p2_wrap_table( wrap );
      check_cuda( cudaMemcpyToSymbol( c_p2_wrap, wrap, sizeof( wrap ) ), "P2 constants (stored order)" );
   } );
}

// mapped quantities of quadrature point q of a micro-cell: Mi = (DF J)^-1 and s = w k |det(DF J)|
// kl: the coefficient's values at the ten nodes (a coefficient stored as a P2 function), or nullptr
// for the closed form at the blended point
template < typename A >
__device__ __forceinline__ void p2_point( const CellGeom& g, const Coefficient& kc, const A X0[3], const A J[3][3], int q, A Mi[3][3],
                                          A& s, const A* kl )
{
   A Xq[3];
   for ( int r = 0; r < 3; ++r )
      Xq[r] = X0[r] + J[r][0] * A( c_xg4_pts[q][0] ) + J[r][1] * A( c_xg4_pts[q][1] ) + J[r][2] * A( c_xg4_pts[q][2] );
   A M[3][3], Fq[3];
   if ( g.blend == 1 )
   {
      A DF[3][3];
      shell_map( g, Xq, Fq, DF );
      for ( int r = 0; r < 3; ++r )
         for ( int c = 0; c < 3; ++c ) M[r][c] = DF[r][0] * J[0][c] + DF[r][1] * J[1][c] + DF[r][2] * J[2][c];
   }
   else
      for ( int r = 0; r < 3; ++r )
      {
         Fq[r] = Xq[r];
         for ( int c = 0; c < 3; ++c ) M[r][c] = J[r][c];
      }
   const A c00 = M[1][1] * M[2][2] - M[1][2] * M[2][1];
   const A c01 = M[1][2] * M[2][0] - M[1][0] * M[2][2];
   const A c02 = M[1][0] * M[2][1] - M[1][1] * M[2][0];
   const A det = M[0][0] * c00 + M[0][1] * c01 + M[0][2] * c02;
   const A id  = A( 1 ) / det;
   Mi[0][0]    = c00 * id;
   Mi[1][0]    = c01 * id;
   Mi[2][0]    = c02 * id;
   Mi[0][1]    = ( M[0][2] * M[2][1] - M[0][1] * M[2][2] ) * id;
   Mi[1][1]    = ( M[0][0] * M[2][2] - M[0][2] * M[2][0] ) * id;
   Mi[2][1]    = ( M[0][1] * M[2][0] - M[0][0] * M[2][1] ) * id;
   Mi[0][2]    = ( M[0][1] * M[1][2] - M[0][2] * M[1][1] ) * id;
   Mi[1][2]    = ( M[0][2] * M[1][0] - M[0][0] * M[1][2] ) * id;
   Mi[2][2]    = ( M[0][0] * M[1][1] - M[0][1] * M[1][0] ) * id;
   A kq;
   if ( kl )
   {
      kq = A( 0 );
      for ( int i = 0; i < 10; ++i ) kq += A( c_p2_phi[q][i] ) * kl[i];
   }
   else
      kq = coeff_eval( kc, Fq );
   s = A( c_xg4_w[q] ) * kq * fabs( det );
}

// physical gradient of basis function i at point q: row (reference gradient) times Mi
template < typename A >
__device__ __forceinline__ void p2_grad( int q, int i, const A Mi[3][3], A G[3] )
{
   for ( int d = 0; d < 3; ++d )
      G[d] = A( c_p2_rgrad[q][i][0] ) * Mi[0][d] + A( c_p2_rgrad[q][i][1] ) * Mi[1][d] + A( c_p2_rgrad[q][i][2] ) * Mi[2][d];
}

// One parity pass over the level-L micro-cells (anchors of parity (px, py, pz); ne = 2^L), nodes
// on storage level L+1.  MODE 0: y += K x computed matrix-free (per point the gradient of the local
// solution, then its pairing with every basis gradient); 1: diagonal of K; 2: store the 55 distinct
// entries of K (wrapped-diagonal order, c_p2_wrap); 3: y += K x from the stored entries.  Stored entry
// v of micro-cell (cell c, type ty, anchor t of the pass's parity class p) sits at
// kst[55 * (6 nC aoff[p] + (c * 6 + ty) * nanch + t) + v] (kbase = 6 nC aoff[p]): the 55 entries of
// a micro-cell are contiguous, so the lanes that read one micro-cell's rows share its 440 bytes.
template < typename T, typename A, int MODE >
__global__ void __launch_bounds__( 256, 2 ) k_p2_pass( int ne, int nanch, const int* __restrict__ anch, const int64_t* __restrict__ cell_off,
                                                     const CellGeom* __restrict__ geom, Coefficient kc,
                                                     const T* __restrict__ src, A* __restrict__ acc, A* __restrict__ kst,
                                                     int64_t kstride, int64_t kbase, int64_t level_size, int* err,
                                                     const double* __restrict__ kn )
{
   const int t = blockIdx.x * blockDim.x + threadIdx.x;  // one micro-cell anchor per thread
   const int c = blockIdx.y;
   if ( t >= nanch ) return;
   const int      a = anch[t];
   const int      x = a & 1023, y = ( a >> 10 ) & 1023, z = a >> 20, ns = 2 * ne;
   const CellGeom g    = geom[c];
   const int64_t  base = cell_off[c];
   const A        inv_n = A( 1.0 / double( ne ) );
   A              st[3][3];
   for ( int k = 0; k < 3; ++k )
      for ( int d = 0; d < 3; ++d ) st[k][d] = ( A( g.P[k + 1][d] ) - A( g.P[0][d] ) ) * inv_n;
      for ( int ty = 0; ty < 6; ++ty )
      {
         if ( x + y + z > ne - 1 - c_mc_shift[ty] ) continue;
         int V[4][3];
         for ( int m = 0; m < 4; ++m )
         {
            V[m][0] = x + c_mc_off[ty][m][0];
            V[m][1] = y + c_mc_off[ty][m][1];
            V[m][2] = z + c_mc_off[ty][m][2];
         }
         int64_t idx[10];
         for ( int m = 0; m < 4; ++m ) idx[m] = base + cidx( ns, 2 * V[m][0], 2 * V[m][1], 2 * V[m][2] );
         for ( int e = 0; e < 6; ++e )
         {
            const int a = c_p2_edge[e][0], b = c_p2_edge[e][1];
            idx[4 + e]  = base + cidx( ns, V[a][0] + V[b][0], V[a][1] + V[b][1], V[a][2] + V[b][2] );
         }
         const int64_t slot = kbase + ( int64_t( c ) * 6 + ty ) * nanch + t;
         {
            // self-check: nodes inside the level's vector, stored slot inside its array
            bool bad = ( MODE >= 2 ) && ( slot < 0 || slot >= kstride );
            for ( int m = 0; m < 10; ++m ) bad |= idx[m] < 0 || idx[m] >= level_size;
            if ( bad )
            {
               atomicExch( err, 2 );
               continue;
            }
         }
         A xl[10], yl[10], kl[10];
         if constexpr ( MODE == 0 || MODE == 3 )
            for ( int m = 0; m < 10; ++m ) xl[m] = A( ld_any( src + idx[m] ) );
         if constexpr ( MODE != 3 )
            if ( kn )
               for ( int m = 0; m < 10; ++m ) kl[m] = A( kn[idx[m]] );
         for ( int m = 0; m < 10; ++m ) yl[m] = A( 0 );
         if constexpr ( MODE == 3 )
         {
            int v = 0;
            for ( int i = 0; i < 10; ++i )
               for ( int j = i; j < 10; ++j, ++v )
               {
                  const A k = kst[slot * 55 + c_p2_wrap[v]];
                  yl[i] += k * xl[j];
                  if ( j != i ) yl[j] += k * xl[i];
               }
         }
         else
         {
            A X0[3], J[3][3];
            for ( int d = 0; d < 3; ++d )
            {
               X0[d] = A( g.P[0][d] ) + st[0][d] * A( V[0][0] ) + st[1][d] * A( V[0][1] ) + st[2][d] * A( V[0][2] );
               for ( int k = 0; k < 3; ++k )
                  J[d][k] = st[0][d] * A( V[k + 1][0] - V[0][0] ) + st[1][d] * A( V[k + 1][1] - V[0][1] ) +
                            st[2][d] * A( V[k + 1][2] - V[0][2] );
            }
            A K[MODE == 2 ? 55 : 1];
            if constexpr ( MODE == 2 )
               for ( int v = 0; v < 55; ++v ) K[v] = A( 0 );
#pragma unroll 1
            for ( int q = 0; q < 11; ++q )
            {
               A Mi[3][3], s;
               p2_point( g, kc, X0, J, q, Mi, s, kn ? kl : static_cast< const A* >( nullptr ) );
               if constexpr ( MODE == 0 )
               {
                  A gs[3] = { A( 0 ), A( 0 ), A( 0 ) };
                  for ( int j = 0; j < 10; ++j )
                     for ( int d = 0; d < 3; ++d ) gs[d] += xl[j] * A( c_p2_rgrad[q][j][d] );
                  A gp[3], h[3];
                  for ( int d = 0; d < 3; ++d ) gp[d] = gs[0] * Mi[0][d] + gs[1] * Mi[1][d] + gs[2] * Mi[2][d];
                  for ( int r2 = 0; r2 < 3; ++r2 ) h[r2] = s * ( Mi[r2][0] * gp[0] + Mi[r2][1] * gp[1] + Mi[r2][2] * gp[2] );
                  for ( int i = 0; i < 10; ++i )
                     yl[i] += A( c_p2_rgrad[q][i][0] ) * h[0] + A( c_p2_rgrad[q][i][1] ) * h[1] + A( c_p2_rgrad[q][i][2] ) * h[2];
               }
               else if constexpr ( MODE == 1 )
                  for ( int i = 0; i < 10; ++i )
                  {
                     A G[3];
                     p2_grad( q, i, Mi, G );
                     yl[i] += s * ( G[0] * G[0] + G[1] * G[1] + G[2] * G[2] );
                  }
               else
               {
                  A G[10][3];
                  for ( int i = 0; i < 10; ++i ) p2_grad( q, i, Mi, G[i] );
                  int v = 0;
                  for ( int i = 0; i < 10; ++i )
                     for ( int j = i; j < 10; ++j, ++v ) K[v] += s * ( G[i][0] * G[j][0] + G[i][1] * G[j][1] + G[i][2] * G[j][2] );
               }
            }
            if constexpr ( MODE == 2 )
            {
               for ( int v = 0; v < 55; ++v ) kst[slot * 55 + c_p2_wrap[v]] = K[v];
               continue;
            }
         }
         for ( int i = 0; i < 10; ++i ) acc[idx[i]] += yl[i];
      }
}

// Combine: cell interior points take s = acc, face/edge/vertex owners the sum of their copies in
// the neighbouring cells; then the operation's epilogue (the constant-stencil kernels' semantics).
template < typename T, typename A, int OP >
__device__ __forceinline__ A epilogue_value( int64_t i, A s, A invd, const T* src, const T* v1, T* v2, A a0, A a1, A* second )
{
   if constexpr ( OP == OP_APPLY || OP == OP_APPLY_ADD ) return s;
   else if constexpr ( OP == OP_RESID ) return A( ld_any( v1 + i ) ) - s;
   else if constexpr ( OP == OP_JAC ) return A( ld_any( src + i ) ) + a0 * ( invd * ( A( ld_any( v1 + i ) ) - s ) );
   else if constexpr ( OP == OP_CHEB0 ) return invd * ( A( ld_any( v1 + i ) ) - s );
   else if constexpr ( OP == OP_CHEBI )
   {
      *second = A( ld_any( v2 + i ) ) + a0 * A( ld_any( src + i ) );
      return invd * s;
   }
   else if constexpr ( OP == OP_CHEBL ) return ( A( ld_any( v2 + i ) ) + a0 * A( ld_any( src + i ) ) ) + a1 * ( invd * s );
   else if constexpr ( OP == OP_DINV_APPLY ) return invd * s;
   return s;
}

template < typename T, typename A, int OP >
__global__ void __launch_bounds__( 256 ) k_cell_acc( int n, int nrows, const int2* __restrict__ rows, const int64_t* __restrict__ cell_off,
                                                      const uint8_t* __restrict__ cell_bc, uint32_t flag, const A* __restrict__ acc,
                                                      const A* __restrict__ invd, const T* src, const T* v1, T* v2, T* dst, A a0, A a1 )
{
   const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
   const int r    = blockIdx.x * 8 + warp;
   const int c    = blockIdx.y;
   if ( r >= nrows || !( cell_bc[c] & flag ) ) return;
   const int2    yz   = rows[r];
   const int64_t base = cell_off[c] + cidx( n, 0, yz.x, yz.y );
   for ( int x = 1 + lane; x <= n - 1 - yz.x - yz.y; x += 32 )
   {
      const int64_t i = base + x;
      A             second;
      const A       val = epilogue_value< T, A, OP >( i, acc[i], invd ? invd[i] : A( 1 ), src, v1, v2, a0, a1, &second );
      if constexpr ( OP == OP_CHEBL ) st_any( v2 + i, val );
      else if constexpr ( OP == OP_APPLY_ADD ) st_any( dst + i, A( ld_any( dst + i ) ) + val );
      else
      {
         st_any( dst + i, val );
         if constexpr ( OP == OP_CHEBI ) st_any( v2 + i, second );
      }
   }
}

// cell-array slot of the copy of task tk's point in incidence I
__device__ __forceinline__ int64_t inc_slot( int n, const int4& tk, const Incidence& I, const int64_t* __restrict__ cell_off )
{
   const int x = n * I.o[0] + tk.y * I.e1[0] + tk.z * I.e2[0];
   const int y = n * I.o[1] + tk.y * I.e1[1] + tk.z * I.e2[1];
   const int z = n * I.o[2] + tk.y * I.e1[2] + tk.z * I.e2[2];
   return __ldg( cell_off + I.cell ) + cidx( n, x, y, z );
}

// owner and copies take val; the incidences are read four at a time ahead of their stores, so a
// vertex with many cells does not wait on one incidence read per copy
template < typename T, typename A >
__device__ __forceinline__ void wt_store( int n, const int4& tk, int64_t owner, const int* __restrict__ inc_begin,
                                          const Incidence* __restrict__ inc, const int64_t* __restrict__ cell_off, T* vec, A val )
{
   st_any( vec + owner, val );
   const int q1 = __ldg( inc_begin + tk.x + 1 );
   for ( int q = __ldg( inc_begin + tk.x ); q < q1; q += 4 )
   {
      int64_t sl[4];
#pragma unroll
      for ( int u = 0; u < 4; ++u ) sl[u] = q + u < q1 ? inc_slot( n, tk, inc[q + u], cell_off ) : -1;
#pragma unroll
      for ( int u = 0; u < 4; ++u )
         if ( sl[u] >= 0 ) st_any( vec + sl[u], val );
   }
}

// sum over the incidences q0..q1-1 of f(incidence), in incidence order, four incidences in flight
template < typename A, int U = 4, typename F >
__device__ __forceinline__ A inc_sum( int q0, int q1, const Incidence* __restrict__ inc, F f )
{
   A s = A( 0 );
   for ( int q = q0; q < q1; q += U )
   {
      A v[U];
#pragma unroll
      for ( int u = 0; u < U; ++u ) v[u] = q + u < q1 ? f( inc[q + u] ) : A( 0 );
#pragma unroll
      for ( int u = 0; u < U; ++u )
         if ( q + u < q1 ) s += v[u];
   }
   return s;
}

// Owners of face/edge/vertex DoFs: sum of the cell copies, epilogue, write-through.  G lanes per task
// (G = 1 on fine levels, where face points with two cells dominate; G = 8 on the coarsest levels,
// where a macro-vertex has 20-30 cells): the lanes of a task take every G-th incidence and combine
// their partial sums by a butterfly, which leaves the same bits in every lane of the group.
template < typename T, typename A, int OP, int G >
__global__ void __launch_bounds__( 256 ) k_bnd_acc( int n, int ntasks, const int4* __restrict__ tasks, const int64_t* __restrict__ off,
                                                     const int64_t* __restrict__ cell_off, const int8_t* __restrict__ bkind,
                                                     const uint8_t* __restrict__ bc, const int* __restrict__ inc_begin,
                                                     const Incidence* __restrict__ inc, uint32_t flag, int copy_unflagged,
                                                     const A* __restrict__ acc, const A* __restrict__ invd, A* invd_out, const T* src,
                                                     const T* v1, T* v2, T* dst, A a0, A a1 )
{
   static_assert( G == 1 || G == 2 || G == 4 || G == 8 || G == 16 || G == 32, "G divides the warp" );
   const int gt = blockIdx.x * blockDim.x + threadIdx.x;
   const int t  = gt / G, sub = gt % G;
   if ( t >= ntasks ) return;  // a group's lanes share t: whole groups leave
   const int4    tk    = tasks[t];
   const int     b     = tk.x;
   const int     k     = bkind[b];
   const int64_t owner = off[b] + ( k == 0 ? 0 : ( k == 1 ? int64_t( tk.y ) : fidx( n, tk.y, tk.z ) ) );
   const int     q0 = __ldg( inc_begin + b ), q1 = __ldg( inc_begin + b + 1 );
   const unsigned gmask = G == 32 ? 0xffffffffu : ( ( 1u << G ) - 1u ) << ( ( threadIdx.x & 31 ) & ~( G - 1 ) );
   // this lane's share of the write-through (G = 1: the owner and every copy)
   auto store = [&]( T* vec, A val ) {
      if constexpr ( G == 1 ) wt_store< T, A >( n, tk, owner, inc_begin, inc, cell_off, vec, val );
      else
      {
         if ( sub == 0 ) st_any( vec + owner, val );
         for ( int q = q0 + sub; q < q1; q += G ) st_any( vec + inc_slot( n, tk, inc[q], cell_off ), val );
      }
   };
   if ( !( bc[b] & flag ) )
   {
      if ( !copy_unflagged ) return;
      if constexpr ( OP == OP_JAC || OP == OP_CHEB0 ) store( dst, A( ld_any( src + owner ) ) );
      else if constexpr ( OP == OP_CHEBI ) store( dst, A( ld_any( v2 + owner ) ) );
      return;
   }
   A s;
   if constexpr ( G == 1 )
      s = inc_sum< A >( q0, q1, inc, [&]( const Incidence& I ) { return acc[inc_slot( n, tk, I, cell_off )]; } );
   else
   {
      s = A( 0 );
      for ( int q = q0 + sub; q < q1; q += G ) s += acc[inc_slot( n, tk, inc[q], cell_off )];
#pragma unroll
      for ( int o = G / 2; o > 0; o >>= 1 ) s += __shfl_xor_sync( gmask, s, o, G );
   }
   if ( invd_out )  // diagonal setup: store 1/diag at the owner
   {
      if ( sub == 0 ) invd_out[owner] = A( 1 ) / s;
      return;
   }
   A       second;
   A       val = epilogue_value< T, A, OP >( owner, s, invd ? invd[owner] : A( 1 ), src, v1, v2, a0, a1, &second );
   if constexpr ( OP == OP_APPLY_ADD ) val = A( ld_any( dst + owner ) ) + val;
   // every lane of the group has read the owner's values before any lane stores
   if constexpr ( G > 1 ) __syncwarp( gmask );
   if constexpr ( OP == OP_CHEBL || OP == OP_APPLY_ADD ) store( OP == OP_CHEBL ? v2 : dst, val );
   else
   {
      store( dst, val );
      if constexpr ( OP == OP_CHEBI ) store( v2, second );
   }
}

// launch of the owner combine over the level's tasks, lanes per task by level size
template < typename T, typename A, int OP >
static void launch_bnd_acc( cudaStream_t st, const P1Level& P, uint32_t flag, int copy_unflagged, const A* acc, const A* invd, A* invd_out,
                            const T* src, const T* v1, T* v2, T* dst, A a0, A a1 )
{
   const int nt = int( P.tasks.size() );
   if ( nt <= 0 ) return;
   if ( P.n <= 4 )
      k_bnd_acc< T, A, OP, 8 ><<< ( 8 * nt + 255 ) / 256, 256, 0, st >>>( P.n, nt, P.d_tasks, P.d_off, P.d_off + P.nB, P.d_bkind, P.d_bc,
                                                                          P.d_inc_begin, P.d_inc, flag, copy_unflagged, acc, invd, invd_out,
                                                                          src, v1, v2, dst, a0, a1 );
   else
      k_bnd_acc< T, A, OP, 1 ><<< ( nt + 255 ) / 256, 256, 0, st >>>( P.n, nt, P.d_tasks, P.d_off, P.d_off + P.nB, P.d_bkind, P.d_bc,
                                                                      P.d_inc_begin, P.d_inc, flag, copy_unflagged, acc, invd, invd_out, src,
                                                                      v1, v2, dst, a0, a1 );
}

// ---------------------------------------------------------------------------------------------
// Assembled stencils (P1 operators with stored matrices): A src at cell-local (x, y, z) of a cell is
// sum_d S_d(slot) src(x + dir_d), S_d the sum of the element-matrix entries of the cell's micro-cells
// that couple the point with its neighbour in direction d (the same sum the elementwise apply forms,
// P1ElementwiseOperator.cpp:169-260, taken once at setup instead of every apply).  One read of 15
// weights per point replaces the 6 micro-cells x 10 entries an elementwise sweep reads.
// ---------------------------------------------------------------------------------------------
template < typename T, typename A, bool INTERIOR >
__device__ __forceinline__ A var_apply( const A* __restrict__ S, int64_t ssize, const T* __restrict__ src, int64_t base, int n, int x,
                                        int y, int z )
{
   const int64_t slot = base + cidx( n, x, y, z );
   A             acc  = A( 0 );
#pragma unroll
   for ( int d = 0; d < 15; ++d )
   {
      const int dx = c_var_dir[d][0], dy = c_var_dir[d][1], dz = c_var_dir[d][2];
      const int xx = x + dx, yy = y + dy, zz = z + dz;
      if ( !INTERIOR && ( xx < 0 || yy < 0 || zz < 0 || xx + yy + zz > n ) ) continue;
      acc += S[d * ssize + slot] * A( ld_any( src + base + cidx( n, xx, yy, zz ) ) );
   }
   return acc;
}

template < typename T, typename A, int OP >
__global__ void __launch_bounds__( 256 ) k_var_cell( int n, int nrows, const int2* __restrict__ rows, const int64_t* __restrict__ cell_off,
                                                      const uint8_t* __restrict__ cell_bc, uint32_t flag, const A* __restrict__ S,
                                                      int64_t ssize, const A* __restrict__ invd, const T* src, const T* v1, T* v2, T* dst,
                                                      A a0, A a1 )
{
   const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
   const int r    = blockIdx.x * 8 + warp;
   const int c    = blockIdx.y;
   if ( r >= nrows || !( cell_bc[c] & flag ) ) return;
   const int2    yz   = rows[r];
   const int64_t cb   = cell_off[c];
   const int64_t base = cb + cidx( n, 0, yz.x, yz.y );
   for ( int x = 1 + lane; x <= n - 1 - yz.x - yz.y; x += 32 )
   {
      const int64_t i = base + x;
      A             second;
      const A       s   = var_apply< T, A, true >( S, ssize, src, cb, n, x, yz.x, yz.y );
      const A       val = epilogue_value< T, A, OP >( i, s, invd[i], src, v1, v2, a0, a1, &second );
      if constexpr ( OP == OP_CHEBL ) st_any( v2 + i, val );
      else if constexpr ( OP == OP_APPLY_ADD ) st_any( dst + i, A( ld_any( dst + i ) ) + val );
      else
      {
         st_any( dst + i, val );
         if constexpr ( OP == OP_CHEBI ) st_any( v2 + i, second );
      }
   }
}

template < typename T, typename A, int OP >
__global__ void __launch_bounds__( 256 ) k_var_bnd( int n, int ntasks, const int4* __restrict__ tasks, const int64_t* __restrict__ off,
                                                     const int64_t* __restrict__ cell_off, const int8_t* __restrict__ bkind,
                                                     const uint8_t* __restrict__ bc, const int* __restrict__ inc_begin,
                                                     const Incidence* __restrict__ inc, uint32_t flag, int copy_unflagged,
                                                     const A* __restrict__ S, int64_t ssize, const A* __restrict__ invd, const T* src,
                                                     const T* v1, T* v2, T* dst, A a0, A a1 )
{
   const int t = blockIdx.x * blockDim.x + threadIdx.x;
   if ( t >= ntasks ) return;
   const int4    tk    = tasks[t];
   const int     b     = tk.x;
   const int     k     = bkind[b];
   const int64_t owner = off[b] + ( k == 0 ? 0 : ( k == 1 ? int64_t( tk.y ) : fidx( n, tk.y, tk.z ) ) );
   if ( !( bc[b] & flag ) )
   {
      if ( !copy_unflagged ) return;
      if constexpr ( OP == OP_JAC || OP == OP_CHEB0 )
         wt_store< T, A >( n, tk, owner, inc_begin, inc, cell_off, dst, A( ld_any( src + owner ) ) );
      else if constexpr ( OP == OP_CHEBI ) wt_store< T, A >( n, tk, owner, inc_begin, inc, cell_off, dst, A( ld_any( v2 + owner ) ) );
      return;
   }
   const A s = inc_sum< A, 2 >( __ldg( inc_begin + b ), __ldg( inc_begin + b + 1 ), inc, [&]( const Incidence& I ) {
      const int x = n * I.o[0] + tk.y * I.e1[0] + tk.z * I.e2[0];
      const int y = n * I.o[1] + tk.y * I.e1[1] + tk.z * I.e2[1];
      const int z = n * I.o[2] + tk.y * I.e1[2] + tk.z * I.e2[2];
      return var_apply< T, A, false >( S, ssize, src, __ldg( cell_off + I.cell ), n, x, y, z );
   } );
   A       second;
   const A val = epilogue_value< T, A, OP >( owner, s, invd[owner], src, v1, v2, a0, a1, &second );
   if constexpr ( OP == OP_CHEBL ) wt_store< T, A >( n, tk, owner, inc_begin, inc, cell_off, v2, val );
   else if constexpr ( OP == OP_APPLY_ADD )
      wt_store< T, A >( n, tk, owner, inc_begin, inc, cell_off, dst, A( ld_any( dst + owner ) ) + val );
   else
   {
      wt_store< T, A >( n, tk, owner, inc_begin, inc, cell_off, dst, val );
      if constexpr ( OP == OP_CHEBI ) wt_store< T, A >( n, tk, owner, inc_begin, inc, cell_off, v2, second );
   }
}

template < typename A >
__global__ void k_cell_invert( int n, int nrows, const int2* __restrict__ rows, const int64_t* __restrict__ cell_off, const A* acc,
                               A* invd )
{
   const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
   const int r    = blockIdx.x * 8 + warp;
   const int c    = blockIdx.y;
   if ( r >= nrows ) return;
   const int2    yz   = rows[r];
   const int64_t base = cell_off[c] + cidx( n, 0, yz.x, yz.y );
   for ( int x = 1 + lane; x <= n - 1 - yz.x - yz.y; x += 32 ) invd[base + x] = A( 1 ) / acc[base + x];
}

// ---------------------------------------------------------------------------------------------
// P2 apply from stored element matrices: ten lanes per micro-cell anchor (three anchors per warp,
// lanes 30-31 idle).  Lane i owns element node i: it loads its node value, gathers the other nine
// with shuffles, reads row i of the symmetric matrix (55 distinct entries per micro-cell in
// wrapped-diagonal order, so each of the ten loads of a group covers one 80-byte run) and adds row i
// times x into its node.  The ten nodes of a micro-cell are distinct, the six
// micro-cells of an anchor are taken in turn by the same lanes, and anchors of one parity class
// share no node, so the read-modify-writes are race-free.  One lane per anchor (the recomputing
// pass) left most of a block idle on these levels: 10 x more lanes in flight per pass.
// ---------------------------------------------------------------------------------------------
template < typename T, typename A >
__global__ void __launch_bounds__( 256 ) k_p2_stored_pass( int ne, int nanch, const int* __restrict__ anch,
                                                            const int64_t* __restrict__ cell_off, const T* __restrict__ src,
                                                            A* __restrict__ acc, const A* __restrict__ kst, int64_t kstride, int64_t kbase,
                                                            int64_t level_size, int* err )
{
   const int lane = threadIdx.x & 31, grp = lane / 10, i = lane - 10 * grp;  // grp 3: lanes 30, 31
   const int t    = ( blockIdx.x * ( blockDim.x >> 5 ) + ( threadIdx.x >> 5 ) ) * 3 + grp;
   const int c    = blockIdx.y;
   const bool live = grp < 3 && t < nanch;
   const int  g0   = 10 * grp;  // first lane of the group
   int        x = 0, y = 0, z = 0;
   if ( live )
   {
      const int a = anch[t];
      x = a & 1023, y = ( a >> 10 ) & 1023, z = a >> 20;
   }
   const int     ns   = 2 * ne;
   const int64_t base = cell_off[c];
   // row i of the symmetric matrix in the wrapped-diagonal order: term t multiplies stored entry
   // koff[t] with the node value of lane xsrc[t] of the group (t = 0: K(i, i); t = 2s-1, 2s:
   // K(i, i+s), K(i, i-s) from block s; t = 9: K(i, i+5) from block 5)
   int koff[10], xsrc[10];
   koff[0] = i;
   xsrc[0] = i;
#pragma unroll
   for ( int d = 1; d <= 4; ++d )
   {
      koff[2 * d - 1] = 10 * d + i;
      xsrc[2 * d - 1] = ( i + d ) % 10;
      koff[2 * d]     = 10 * d + ( i + 10 - d ) % 10;
      xsrc[2 * d]     = ( i + 10 - d ) % 10;
   }
   koff[9] = 50 + i % 5;
   xsrc[9] = ( i + 5 ) % 10;
   // node index, stored slot and the self-check of micro-cell type ty (all lanes of the warp take
   // part: the check is a warp vote)
   auto prep = [&]( int ty, int64_t& idx, int64_t& slot, bool& go ) {
      const bool cell = live && x + y + z <= ne - 1 - c_mc_shift[ty];
      // node i of the micro-cell: vertex i (i < 4) at 2 V_i, edge (a, b) at V_a + V_b
      idx = 0;
      if ( cell )
      {
         int P[3];
         if ( i < 4 )
            for ( int d = 0; d < 3; ++d ) P[d] = 2 * ( ( d == 0 ? x : d == 1 ? y : z ) + c_mc_off[ty][i][d] );
         else
         {
            const int ea = c_p2_edge[i - 4][0], eb = c_p2_edge[i - 4][1];
            for ( int d = 0; d < 3; ++d )
               P[d] = 2 * ( d == 0 ? x : d == 1 ? y : z ) + c_mc_off[ty][ea][d] + c_mc_off[ty][eb][d];
         }
         idx = base + cidx( ns, P[0], P[1], P[2] );
      }
      slot = kbase + ( int64_t( c ) * 6 + ty ) * nanch + ( cell ? t : 0 );
      // self-check: every node inside the level's vector and the stored slot inside its array; a
      // violation in any lane of the group skips the micro-cell and records error word 2
      const bool     bad  = cell && ( idx < 0 || idx >= level_size || slot < 0 || slot >= kstride );
      const unsigned bmsk = __ballot_sync( 0xffffffffu, bad );
      const bool     gbad = grp < 3 && ( ( bmsk >> g0 ) & 0x3ffu ) != 0u;
      if ( bad ) atomicExch( err, 2 );
      go = cell && !gbad;
   };
   // software pipeline over the six micro-cell types: the node value and matrix row of type ty+1
   // are loaded before type ty's product and read-modify-write, which are the only steps that must
   // stay in order (micro-cells of one anchor share nodes)
   int64_t idx0, slot0;
   bool    go0;
   prep( 0, idx0, slot0, go0 );
   A x0 = go0 ? A( ld_any( src + idx0 ) ) : A( 0 );
   A k0[10];
#pragma unroll
   for ( int j = 0; j < 10; ++j ) k0[j] = go0 ? __ldg( kst + slot0 * 55 + koff[j] ) : A( 0 );
#pragma unroll 1
   for ( int ty = 0; ty < 6; ++ty )
   {
      int64_t idx1 = 0, slot1 = 0;
      bool    go1 = false;
      A       x1  = A( 0 ), k1[10];
      if ( ty < 5 ) prep( ty + 1, idx1, slot1, go1 );
      if ( go1 ) x1 = A( ld_any( src + idx1 ) );
#pragma unroll
      for ( int j = 0; j < 10; ++j ) k1[j] = go1 ? __ldg( kst + slot1 * 55 + koff[j] ) : A( 0 );
      A yi = A( 0 );
#pragma unroll
      for ( int j = 0; j < 10; ++j )
      {
         const A xj = __shfl_sync( 0xffffffffu, x0, grp < 3 ? g0 + xsrc[j] : lane );
         if ( go0 ) yi += k0[j] * xj;
      }
      if ( go0 ) acc[idx0] += yi;
      idx0 = idx1;
      go0  = go1;
      x0   = x1;
#pragma unroll
      for ( int j = 0; j < 10; ++j ) k0[j] = k1[j];
   }
}

// ---------------------------------------------------------------------------------------------
// Stokes coupling blocks (P2P1ElementwiseBlendingStokesOperator, P2P1ElementwiseBlendingStokesOperator.hpp:
// 113-116): div = P2ToP1ElementwiseBlendingDiv{x,y,z} (forms p2_to_p1_div_{0,1,2}_blending_q2) maps a
// P2 velocity of level l to a P1 pressure of level l, divT (p1_to_p2_divt_{0,1,2}_blending_q2) is its
// transpose.  Element matrix of component k: B_k[i][j] = -int psi_i d(phi_j)/dx_k over the blended
// micro-cell, psi P1 and phi P2, with the 4-point degree-2 rule (a = (5 - sqrt 5)/20,
// b = (5 + 3 sqrt 5)/20, weights 1/24).  Applied matrix-free: div forms the divergence of the local
// velocity at each point; divT pairs the local pressure with every basis gradient.  The P1 nodes are
// the micro-cell's vertices on level l, the P2 nodes the ten nodes on storage level l+1; anchors of
// one parity class share neither, so the passes are race-free.
// ---------------------------------------------------------------------------------------------
__constant__ double c_q2_pts[4][3];
__constant__ double c_q2_rgrad[4][10][3];

void ensure_stokes_constants()
{
   static PerDeviceOnce once;
   once.run( [] {
      const double a = ( 5.0 - std::sqrt( 5.0 ) ) / 20.0, b = ( 5.0 + 3.0 * std::sqrt( 5.0 ) ) / 20.0;
      const double pts[4][3] = { { a, a, a }, { b, a, a }, { a, b, a }, { a, a, b } };
      const double lg[4][3]  = { { -1, -1, -1 }, { 1, 0, 0 }, { 0, 1, 0 }, { 0, 0, 1 } };
      const int    ed[6][2]  = { { 2, 3 }, { 1, 3 }, { 1, 2 }, { 0, 3 }, { 0, 2 }, { 0, 1 } };
      double       g[4][10][3];
      for ( int q = 0; q < 4; ++q )
      {
         const double lam[4] = { 1.0 - pts[q][0] - pts[q][1] - pts[q][2], pts[q][0], pts[q][1], pts[q][2] };
         for ( int i = 0; i < 4; ++i )
            for ( int d = 0; d < 3; ++d ) g[q][i][d] = ( 4.0 * lam[i] - 1.0 ) * lg[i][d];
         for ( int e = 0; e < 6; ++e )
            for ( int d = 0; d < 3; ++d )
               g[q][4 + e][d] = 4.0 * ( lam[ed[e][0]] * lg[ed[e][1]][d] + lam[ed[e][1]] * lg[ed[e][0]][d] );
      }
      check_cuda( cudaMemcpyToSymbol( c_q2_pts, pts, sizeof( pts ) ), "Stokes constants (points)" );
      check_cuda( cudaMemcpyToSymbol( c_q2_rgrad, g, sizeof( g ) ), "Stokes constants (gradients)" );
   } );
}

// inverse of the blended Jacobian M = DF J at reference point xi and |det M|
// (Fq, when given, receives the blended point)
template < typename A >
__device__ __forceinline__ void mapped_point( const CellGeom& g, const A X0[3], const A J[3][3], const double* xi, A Mi[3][3], A& adet,
                                              A* Fq = nullptr )
{
   A Xq[3];
   for ( int r = 0; r < 3; ++r ) Xq[r] = X0[r] + J[r][0] * A( xi[0] ) + J[r][1] * A( xi[1] ) + J[r][2] * A( xi[2] );
   A M[3][3];
   if ( g.blend == 1 )
   {
      A DF[3][3], Fl[3];
      shell_map( g, Xq, Fl, DF );
      for ( int r = 0; r < 3; ++r )
         for ( int c = 0; c < 3; ++c ) M[r][c] = DF[r][0] * J[0][c] + DF[r][1] * J[1][c] + DF[r][2] * J[2][c];
      if ( Fq )
         for ( int r = 0; r < 3; ++r ) Fq[r] = Fl[r];
   }
   else
   {
      for ( int r = 0; r < 3; ++r )
         for ( int c = 0; c < 3; ++c ) M[r][c] = J[r][c];
      if ( Fq )
         for ( int r = 0; r < 3; ++r ) Fq[r] = Xq[r];
   }
   const A c00 = M[1][1] * M[2][2] - M[1][2] * M[2][1];
   const A c01 = M[1][2] * M[2][0] - M[1][0] * M[2][2];
   const A c02 = M[1][0] * M[2][1] - M[1][1] * M[2][0];
   const A det = M[0][0] * c00 + M[0][1] * c01 + M[0][2] * c02;
   const A id  = A( 1 ) / det;
   Mi[0][0]    = c00 * id;
   Mi[1][0]    = c01 * id;
   Mi[2][0]    = c02 * id;
   Mi[0][1]    = ( M[0][2] * M[2][1] - M[0][1] * M[2][2] ) * id;
   Mi[1][1]    = ( M[0][0] * M[2][2] - M[0][2] * M[2][0] ) * id;
   Mi[2][1]    = ( M[0][1] * M[2][0] - M[0][0] * M[2][1] ) * id;
   Mi[0][2]    = ( M[0][1] * M[1][2] - M[0][2] * M[1][1] ) * id;
   Mi[1][2]    = ( M[0][2] * M[1][0] - M[0][0] * M[1][2] ) * id;
   Mi[2][2]    = ( M[0][0] * M[1][1] - M[0][1] * M[1][0] ) * id;
   adet        = fabs( det );
}

// DIVT 0: p_acc[vertex i] += sum_k sum_j B_k[i][j] u_k[j];  DIVT 1: u_acc_k[node j] += sum_i B_k[i][j] p[i]
template < typename T, typename A, int DIVT >
__global__ void __launch_bounds__( 256 ) k_stokes_div_pass( int ne, int nanch, const int* __restrict__ anch,
                                                             const int64_t* __restrict__ off_p, const int64_t* __restrict__ off_u,
                                                             const CellGeom* __restrict__ geom, const T* __restrict__ u0,
                                                             const T* __restrict__ u1, const T* __restrict__ u2,
                                                             const T* __restrict__ p, A* accp, A* acc0, A* acc1, A* acc2,
                                                             int64_t size_p, int64_t size_u, int* err )
{
   const int t = blockIdx.x * blockDim.x + threadIdx.x;
   const int c = blockIdx.y;
   if ( t >= nanch ) return;
   const int      a = anch[t];
   const int      x = a & 1023, y = ( a >> 10 ) & 1023, z = a >> 20, ns = 2 * ne;
   const CellGeom g = geom[c];
   const int64_t  bp = off_p[c], bu = off_u[c];
   const A        inv_n = A( 1.0 / double( ne ) );
   A              st[3][3];
   for ( int k = 0; k < 3; ++k )
      for ( int d = 0; d < 3; ++d ) st[k][d] = ( A( g.P[k + 1][d] ) - A( g.P[0][d] ) ) * inv_n;
   for ( int ty = 0; ty < 6; ++ty )
   {
      if ( x + y + z > ne - 1 - c_mc_shift[ty] ) continue;
      int V[4][3];
      for ( int m = 0; m < 4; ++m )
         for ( int d = 0; d < 3; ++d ) V[m][d] = ( d == 0 ? x : d == 1 ? y : z ) + c_mc_off[ty][m][d];
      int64_t ip[4], iu[10];
      for ( int m = 0; m < 4; ++m )
      {
         ip[m] = bp + cidx( ne, V[m][0], V[m][1], V[m][2] );
         iu[m] = bu + cidx( ns, 2 * V[m][0], 2 * V[m][1], 2 * V[m][2] );
      }
      for ( int e = 0; e < 6; ++e )
      {
         const int ea = c_p2_edge[e][0], eb = c_p2_edge[e][1];
         iu[4 + e]    = bu + cidx( ns, V[ea][0] + V[eb][0], V[ea][1] + V[eb][1], V[ea][2] + V[eb][2] );
      }
      {
         bool bad = false;
         for ( int m = 0; m < 4; ++m ) bad |= ip[m] < 0 || ip[m] >= size_p;
         for ( int m = 0; m < 10; ++m ) bad |= iu[m] < 0 || iu[m] >= size_u;
         if ( bad )
         {
            atomicExch( err, 2 );
            continue;
         }
      }
      A X0[3], J[3][3];
      for ( int d = 0; d < 3; ++d )
      {
         X0[d] = A( g.P[0][d] ) + st[0][d] * A( V[0][0] ) + st[1][d] * A( V[0][1] ) + st[2][d] * A( V[0][2] );
         for ( int k = 0; k < 3; ++k )
            J[d][k] = st[0][d] * A( V[k + 1][0] - V[0][0] ) + st[1][d] * A( V[k + 1][1] - V[0][1] ) + st[2][d] * A( V[k + 1][2] - V[0][2] );
      }
      if constexpr ( DIVT == 0 )
      {
         A ul[3][10];
         for ( int j = 0; j < 10; ++j )
         {
            ul[0][j] = A( ld_any( u0 + iu[j] ) );
            ul[1][j] = A( ld_any( u1 + iu[j] ) );
            ul[2][j] = A( ld_any( u2 + iu[j] ) );
         }
         A yl[4] = { A( 0 ), A( 0 ), A( 0 ), A( 0 ) };
         for ( int q = 0; q < 4; ++q )
         {
            A Mi[3][3], adet;
            mapped_point( g, X0, J, c_q2_pts[q], Mi, adet );
            // divergence of the local velocity: sum_k sum_j u_k[j] (grad_ref phi_j . Mi)_k
            A dv = A( 0 );
            for ( int j = 0; j < 10; ++j )
               for ( int k = 0; k < 3; ++k )
                  dv += ul[k][j] * ( A( c_q2_rgrad[q][j][0] ) * Mi[0][k] + A( c_q2_rgrad[q][j][1] ) * Mi[1][k] +
                                     A( c_q2_rgrad[q][j][2] ) * Mi[2][k] );
            const A f      = -A( 1.0 / 24.0 ) * adet * dv;
            const A lam[4] = { A( 1.0 - c_q2_pts[q][0] - c_q2_pts[q][1] - c_q2_pts[q][2] ), A( c_q2_pts[q][0] ), A( c_q2_pts[q][1] ),
                               A( c_q2_pts[q][2] ) };
            for ( int i = 0; i < 4; ++i ) yl[i] += f * lam[i];
         }
         for ( int i = 0; i < 4; ++i ) accp[ip[i]] += yl[i];
      }
      else
      {
         A pl[4];
         for ( int i = 0; i < 4; ++i ) pl[i] = A( ld_any( p + ip[i] ) );
         A yl[3][10];
         for ( int k = 0; k < 3; ++k )
            for ( int j = 0; j < 10; ++j ) yl[k][j] = A( 0 );
         for ( int q = 0; q < 4; ++q )
         {
            A Mi[3][3], adet;
            mapped_point( g, X0, J, c_q2_pts[q], Mi, adet );
            const A pq = pl[0] * A( 1.0 - c_q2_pts[q][0] - c_q2_pts[q][1] - c_q2_pts[q][2] ) + pl[1] * A( c_q2_pts[q][0] ) +
                         pl[2] * A( c_q2_pts[q][1] ) + pl[3] * A( c_q2_pts[q][2] );
            const A f = -A( 1.0 / 24.0 ) * adet * pq;
            for ( int j = 0; j < 10; ++j )
               for ( int k = 0; k < 3; ++k )
                  yl[k][j] += f * ( A( c_q2_rgrad[q][j][0] ) * Mi[0][k] + A( c_q2_rgrad[q][j][1] ) * Mi[1][k] +
                                    A( c_q2_rgrad[q][j][2] ) * Mi[2][k] );
         }
         for ( int j = 0; j < 10; ++j )
         {
            acc0[iu[j]] += yl[0][j];
            acc1[iu[j]] += yl[1][j];
            acc2[iu[j]] += yl[2][j];
         }
      }
   }
}

// ---------------------------------------------------------------------------------------------
// host launch
// ---------------------------------------------------------------------------------------------
template < typename A >
static A* acc_buffer( Operator* op, int L, int64_t size )
{
   ElemLevel& e   = op->el[L];
   const int  adt = sizeof( A ) == 8 ? F64 : F32;
   if ( e.d_acc && e.acc_dtype != adt && adt == F64 )
   {
      check_cuda( cudaFree( e.d_acc ), "cudaFree(acc)" );
      e.d_acc = nullptr;
   }
   if ( !e.d_acc )
   {
      check_cuda( cudaMalloc( &e.d_acc, size * sizeof( double ) ), "cudaMalloc(elementwise scratch)" );
      e.acc_dtype = F64;
   }
   return reinterpret_cast< A* >( e.d_acc );
}

// stencil direction of every vertex pair of every micro-cell type (vertex offsets as c_mc_off)
static void ensure_var_tables()
{
   static PerDeviceOnce once;
   once.run( [] {
      static const int off[6][4][3] = {
          { { 0, 0, 0 }, { 1, 0, 0 }, { 0, 1, 0 }, { 0, 0, 1 } }, { { 1, 0, 0 }, { 1, 1, 0 }, { 0, 1, 0 }, { 1, 0, 1 } },
          { { 1, 0, 0 }, { 0, 1, 0 }, { 1, 0, 1 }, { 0, 0, 1 } }, { { 1, 1, 0 }, { 1, 1, 1 }, { 0, 1, 1 }, { 1, 0, 1 } },
          { { 1, 0, 1 }, { 0, 1, 1 }, { 0, 0, 1 }, { 0, 1, 0 } }, { { 0, 1, 0 }, { 1, 1, 0 }, { 1, 0, 1 }, { 0, 1, 1 } } };
      int8_t dir[6][4][4], vd[15][3];
      for ( int d = 0; d < 15; ++d )
         for ( int k = 0; k < 3; ++k ) vd[d][k] = int8_t( kVarDirs[d][k] );
      for ( int t = 0; t < 6; ++t )
         for ( int i = 0; i < 4; ++i )
            for ( int j = 0; j < 4; ++j )
            {
               int found = -1;
               for ( int d = 0; d < 15; ++d )
                  if ( off[t][j][0] - off[t][i][0] == kVarDirs[d][0] && off[t][j][1] - off[t][i][1] == kVarDirs[d][1] &&
                       off[t][j][2] - off[t][i][2] == kVarDirs[d][2] )
                     found = d;
               if ( found < 0 ) throw std::runtime_error( "micro-cell edge outside the 15-point stencil" );
               dir[t][i][j] = int8_t( found );
            }
      check_cuda( cudaMemcpyToSymbol( c_mc_dir, dir, sizeof( dir ) ), "upload stencil directions" );
      check_cuda( cudaMemcpyToSymbol( c_var_dir, vd, sizeof( vd ) ), "upload stencil directions" );
   } );
}

template < typename A >
static A* assembled_stencils( Operator* op, int L ) { return reinterpret_cast< A* >( op->el[L].d_S[sizeof( A ) == 8 ? 0 : 1] ); }

// micro-cells per macro-edge of the elements living on storage level L (P2 elements of level L-1
// have their nodes on storage level L)
static int element_n( const Operator* op, int L ) { return op->order == 2 ? ( 1 << ( L - 1 ) ) : ( 1 << L ); }
static int element_values( const Operator* op ) { return op->order == 2 ? 55 : 10; }

// micro-cell anchors (x, y, z), x + y + z <= n - 1, grouped by coordinate parity: the micro-cells of
// anchors of one parity class share no vertex (nor, for P2, any node), so a pass over one class
// updates its nodes without conflicts
static void ensure_rows( Operator* op, int L )
{
   ElemLevel& e = op->el[L];
   if ( e.d_anch ) return;
   const int          n = element_n( op, L );
   std::vector< int > anch;
   for ( int p = 0; p < 8; ++p )
   {
      e.aoff[p]    = int( anch.size() );
      const int px = p & 1, py = ( p >> 1 ) & 1, pz = p >> 2;
      for ( int z = pz; z <= n - 1; z += 2 )
         for ( int y = py; y + z <= n - 1; y += 2 )
            for ( int x = px; x + y + z <= n - 1; x += 2 ) anch.push_back( x | ( y << 10 ) | ( z << 20 ) );
   }
   e.aoff[8] = int( anch.size() );
   check_cuda( cudaMalloc( &e.d_anch, std::max< size_t >( anch.size(), 1 ) * sizeof( int ) ), "cudaMalloc(anchors)" );
   if ( !anch.empty() )
      check_cuda( cudaMemcpy( e.d_anch, anch.data(), anch.size() * sizeof( int ), cudaMemcpyHostToDevice ), "upload anchors" );
}

// entries per stored value: every (cell, micro-cell type, anchor) slot of the level
static int64_t kstride( Mesh* m, const Operator* op, int L ) { return int64_t( m->topo.nC ) * 6 * tet_size( int64_t( element_n( op, L ) ) ); }

template < typename A >
static A* stored_matrices( Operator* op, int L ) { return reinterpret_cast< A* >( op->el[L].d_K[sizeof( A ) == 8 ? 0 : 1] ); }

// threads per block of a pass over na anchors per cell (grid: blocks x cells): whole warps, at most
// maxb, so that the small levels (a few anchors per cell) do not launch mostly idle blocks
static int pass_block( int na, int maxb ) { return std::min( maxb, ( na + 31 ) / 32 * 32 ); }

template < typename T, typename A, int MODE >
static void run_passes( Context* ctx, Mesh* m, Operator* op, int L, const T* src, A* acc )
{
   P1Level&   P = m->level( L );
   ElemLevel& e = op->el[L];
   if ( MODE != 2 && MODE != 4 ) check_cuda( cudaMemsetAsync( acc, 0, P.size * sizeof( A ), ctx->stream ), "cudaMemset(acc)" );
   A*            kst = MODE == 4 ? assembled_stencils< A >( op, L ) : stored_matrices< A >( op, L );
   const int64_t ks  = MODE == 4 ? P.size : kstride( m, op, L );
   const int nC = m->topo.nC;
   for ( int p = 0; p < 8; ++p )
   {
      const int na = e.aoff[p + 1] - e.aoff[p];
      if ( na <= 0 ) continue;
      // P2 stored matrices are grouped by parity class, then cell, micro-cell type and anchor, so the
      // anchors of one pass read consecutive slots
      const int64_t kbase = int64_t( 6 ) * nC * e.aoff[p];
      const int bs = pass_block( na, 256 );
      dim3      grid( ( na + bs - 1 ) / bs, nC );
      if ( op->order == 2 && MODE == 3 )
      {
         // three anchors per warp (ten lanes each), at most 8 warps per block
         const int  wb = std::min( 8, ( na + 2 ) / 3 );
         const dim3 g3( ( na + 3 * wb - 1 ) / ( 3 * wb ), nC );
         k_p2_stored_pass< T, A ><<< g3, 32 * wb, 0, ctx->stream >>>( element_n( op, L ), na, e.d_anch + e.aoff[p], P.d_off + P.nB, src,
                                                                      acc, kst, ks, kbase, P.size, ctx->d_error );
      }
      else if ( op->order == 2 )
         k_p2_pass< T, A, MODE ><<< grid, bs, 0, ctx->stream >>>( element_n( op, L ), na, e.d_anch + e.aoff[p], P.d_off + P.nB,
                                                                   op->d_geom, op->coeff, src, acc, kst, ks, kbase, P.size,
                                                                   ctx->d_error, op->nodal_k ? e.d_kn : nullptr );
      else
         k_elem_pass< T, A, MODE ><<< grid, bs, 0, ctx->stream >>>( P.n, na, e.d_anch + e.aoff[p], P.d_off + P.nB, op->d_geom,
                                                                     op->coeff, src, acc, kst, ks, P.size, ctx->d_error );
      ++ctx->launches;
   }
   check_cuda( cudaGetLastError(), "elementwise pass launch" );
}

// A coefficient stored as a P2 function (the hyteg-operators P2ElementwiseDivKGrad operators take k
// as a P2Function interpolated at the nodes): its closed form at every cell-array node of storage
// level ns, at the node's blended position.  Block (z, cell), threads over the rows y of slice z.
__global__ void __launch_bounds__( 128 ) k_p2_nodal_coeff( int ns, const int64_t* __restrict__ cell_off, const CellGeom* __restrict__ geom,
                                                            Coefficient kc, double* kn )
{
   const int      z = blockIdx.x, c = blockIdx.y;
   const CellGeom g = geom[c];
   for ( int y = threadIdx.x; y + z <= ns; y += blockDim.x )
      for ( int x = 0; x + y + z <= ns; ++x )
      {
         double X[3], F[3], DF[3][3];
         for ( int d = 0; d < 3; ++d )
            X[d] = g.P[0][d] + ( ( g.P[1][d] - g.P[0][d] ) * x + ( g.P[2][d] - g.P[0][d] ) * y + ( g.P[3][d] - g.P[0][d] ) * z ) / double( ns );
         if ( g.blend == 1 ) shell_map( g, X, F, DF );
         else
            for ( int d = 0; d < 3; ++d ) F[d] = X[d];
         kn[cell_off[c] + cidx( ns, x, y, z )] = coeff_eval( kc, F );
      }
}

static void upload_geometry( Operator* op )
{
   if ( op->d_geom ) return;
   check_cuda( cudaMalloc( &op->d_geom, op->geom.size() * sizeof( CellGeom ) ), "cudaMalloc(geometry)" );
   check_cuda( cudaMemcpy( op->d_geom, op->geom.data(), op->geom.size() * sizeof( CellGeom ), cudaMemcpyHostToDevice ), "upload geometry" );
}

void set_p2_nodal_coefficient( Context* ctx, Operator* op, int Ls, const double* src )
{
   Mesh*    m = op->mesh;
   P1Level& P = m->level( Ls );
   ensure_device( m, P );
   upload_geometry( op );
   ElemLevel& e = op->el[Ls];
   if ( !e.d_kn ) check_cuda( cudaMalloc( &e.d_kn, P.size * sizeof( double ) ), "cudaMalloc(nodal coefficient)" );
   check_cuda( cudaMemsetAsync( e.d_kn, 0, P.size * sizeof( double ), ctx->stream ), "cudaMemset(nodal coefficient)" );
   if ( src )
      check_cuda( cudaMemcpyAsync( e.d_kn, src, P.size * sizeof( double ), cudaMemcpyDeviceToDevice, ctx->stream ), "copy nodal coefficient" );
   else
   {
      const dim3 grid( P.n + 1, m->topo.nC );
      k_p2_nodal_coeff<<< grid, 128, 0, ctx->stream >>>( P.n, P.d_off + P.nB, op->d_geom, op->coeff, e.d_kn );
      ++ctx->launches;
      check_cuda( cudaGetLastError(), "nodal coefficient launch" );
   }
}

template < typename T, typename A >
static void ensure_level_t( Context* ctx, Operator* op, int L, int dtype )
{
   Mesh*    m = op->mesh;
   P1Level& P = m->level( L );
   ensure_device( m, P );
   upload_geometry( op );
   ensure_rows( op, L );
   ElemLevel& e = op->el[L];
   A*         acc = acc_buffer< A >( op, L, P.size );
   void*&     K   = e.d_K[sizeof( A ) == 8 ? 0 : 1];
   if ( op->store_matrices && op->order == 1 )
   {
      // P1: the stored matrices are kept assembled, summed in double once and rounded for float
      ensure_var_tables();
      const int64_t cnt = int64_t( 15 ) * P.size;
      if ( !e.d_S[0] )
      {
         check_cuda( cudaMalloc( &e.d_S[0], cnt * sizeof( double ) ), "cudaMalloc(assembled stencils)" );
         check_cuda( cudaMemsetAsync( e.d_S[0], 0, cnt * sizeof( double ), ctx->stream ), "cudaMemset" );
         run_passes< double, double, 4 >( ctx, m, op, L, nullptr, nullptr );
      }
      if ( sizeof( A ) == 4 && !e.d_S[1] )
      {
         check_cuda( cudaMalloc( &e.d_S[1], cnt * sizeof( float ) ), "cudaMalloc(assembled stencils)" );
         launch_convert( ctx, cnt, F32, e.d_S[1], F64, e.d_S[0] );
      }
   }
   else if ( op->store_matrices && !K )
   {
      check_cuda( cudaMalloc( &K, size_t( element_values( op ) ) * size_t( kstride( m, op, L ) ) * sizeof( A ) ),
                  "cudaMalloc(element matrices)" );
      run_passes< T, A, 2 >( ctx, m, op, L, nullptr, acc );
   }
   if ( e.d_invd[dtype] ) return;
   A* invd = nullptr;
   check_cuda( cudaMalloc( &invd, P.size * sizeof( A ) ), "cudaMalloc(inverse diagonal)" );
   check_cuda( cudaMemsetAsync( invd, 0, P.size * sizeof( A ), ctx->stream ), "cudaMemset" );
   e.d_invd[dtype] = invd;
   // diagonal: sum of element-matrix diagonals, owners summing their cell copies
   run_passes< T, A, 1 >( ctx, m, op, L, nullptr, acc );
   const int nrows = int( P.rows.size() );
   if ( nrows > 0 )
   {
      dim3 grid( ( nrows + 7 ) / 8, m->topo.nC );
      k_cell_invert< A ><<< grid, 256, 0, ctx->stream >>>( P.n, nrows, P.d_rows, P.d_off + P.nB, acc, invd );
   }
   if ( !P.tasks.empty() )
      launch_bnd_acc< T, A, OP_APPLY >( ctx->stream, P, kAll, 0, acc, nullptr, invd, nullptr, nullptr, nullptr, nullptr, A( 0 ), A( 0 ) );
   check_cuda( cudaGetLastError(), "diagonal launch" );
}

void ensure_elementwise_level( Context* ctx, Operator* op, int L, int dtype )
{
   if ( dtype == F64 ) ensure_level_t< double, double >( ctx, op, L, dtype );
   else if ( dtype == F32 ) ensure_level_t< float, float >( ctx, op, L, dtype );
   else ensure_level_t< __half, float >( ctx, op, L, dtype );
}

template < typename T, typename A, int OP >
static void run_var( Context* ctx, Mesh* m, Operator* op, int L, int dtype, const StencilArgs& a )
{
   P1Level& P = m->level( L );
   const A* S   = assembled_stencils< A >( op, L );
   const A* inv = reinterpret_cast< const A* >( op->el[L].d_invd[dtype] );
   struct Join
   {
      Context* c;
      ~Join()
      {
         cudaEventRecord( c->ev_join, c->aux );
         cudaStreamWaitEvent( c->stream, c->ev_join, 0 );
      }
   };
   check_cuda( cudaEventRecord( ctx->ev_fork, ctx->stream ), "fork" );
   check_cuda( cudaStreamWaitEvent( ctx->aux, ctx->ev_fork, 0 ), "fork" );
   Join      j{ ctx };
   const int nrows = int( P.rows.size() );
   if ( nrows > 0 )
   {
      dim3 grid( ( nrows + 7 ) / 8, m->topo.nC );
      k_var_cell< T, A, OP ><<< grid, 256, 0, ctx->stream >>>( P.n, nrows, P.d_rows, P.d_off + P.nB, P.d_bc + P.nB, a.flag, S, P.size, inv,
                                                                (const T*) a.src, (const T*) a.v1, (T*) a.v2, (T*) a.dst, A( a.a0 ),
                                                                A( a.a1 ) );
      ++ctx->launches;
   }
   if ( !P.tasks.empty() )
   {
      k_var_bnd< T, A, OP ><<< ( int( P.tasks.size() ) + 255 ) / 256, 256, 0, ctx->aux >>>(
          P.n, int( P.tasks.size() ), P.d_tasks, P.d_off, P.d_off + P.nB, P.d_bkind, P.d_bc, P.d_inc_begin, P.d_inc, a.flag,
          a.copy_unflagged, S, P.size, inv, (const T*) a.src, (const T*) a.v1, (T*) a.v2, (T*) a.dst, A( a.a0 ), A( a.a1 ) );
      ++ctx->launches;
   }
   check_cuda( cudaGetLastError(), "assembled stencil launch" );
}

template < typename T, typename A, int OP >
static void run_elem( Context* ctx, Mesh* m, Operator* op, int L, int dtype, const StencilArgs& a )
{
   if ( op->order == 1 && assembled_stencils< A >( op, L ) ) return run_var< T, A, OP >( ctx, m, op, L, dtype, a );
   P1Level& P   = m->level( L );
   A*       acc = acc_buffer< A >( op, L, P.size );
   const A* inv = reinterpret_cast< const A* >( op->el[L].d_invd[dtype] );
   if ( stored_matrices< A >( op, L ) ) run_passes< T, A, 3 >( ctx, m, op, L, (const T*) a.src, acc );
   else run_passes< T, A, 0 >( ctx, m, op, L, (const T*) a.src, acc );
   const int nrows = int( P.rows.size() );
   {
      struct Join
      {
         Context* c;
         ~Join()
         {
            cudaEventRecord( c->ev_join, c->aux );
            cudaStreamWaitEvent( c->stream, c->ev_join, 0 );
         }
      };
      check_cuda( cudaEventRecord( ctx->ev_fork, ctx->stream ), "fork" );
      check_cuda( cudaStreamWaitEvent( ctx->aux, ctx->ev_fork, 0 ), "fork" );
      Join j{ ctx };
      if ( nrows > 0 )
      {
         dim3 grid( ( nrows + 7 ) / 8, m->topo.nC );
         k_cell_acc< T, A, OP ><<< grid, 256, 0, ctx->stream >>>( P.n, nrows, P.d_rows, P.d_off + P.nB, P.d_bc + P.nB, a.flag, acc, inv,
                                                                   (const T*) a.src, (const T*) a.v1, (T*) a.v2, (T*) a.dst, A( a.a0 ),
                                                                   A( a.a1 ) );
         ++ctx->launches;
      }
      if ( !P.tasks.empty() )
      {
         launch_bnd_acc< T, A, OP >( ctx->aux, P, a.flag, a.copy_unflagged, acc, inv, nullptr, (const T*) a.src, (const T*) a.v1,
                                     (T*) a.v2, (T*) a.dst, A( a.a0 ), A( a.a1 ) );
         ++ctx->launches;
      }
   }
   check_cuda( cudaGetLastError(), "elementwise combine launch" );
}

template < typename T, typename A >
static void dispatch_elem( Context* ctx, Mesh* m, Operator* op, int L, int dtype, const StencilArgs& a )
{
   switch ( a.op )
   {
   case OP_APPLY: run_elem< T, A, OP_APPLY >( ctx, m, op, L, dtype, a ); break;
   case OP_APPLY_ADD: run_elem< T, A, OP_APPLY_ADD >( ctx, m, op, L, dtype, a ); break;
   case OP_RESID: run_elem< T, A, OP_RESID >( ctx, m, op, L, dtype, a ); break;
   case OP_JAC: run_elem< T, A, OP_JAC >( ctx, m, op, L, dtype, a ); break;
   case OP_CHEB0: run_elem< T, A, OP_CHEB0 >( ctx, m, op, L, dtype, a ); break;
   case OP_CHEBI: run_elem< T, A, OP_CHEBI >( ctx, m, op, L, dtype, a ); break;
   case OP_CHEBL: run_elem< T, A, OP_CHEBL >( ctx, m, op, L, dtype, a ); break;
   case OP_DINV_APPLY: run_elem< T, A, OP_DINV_APPLY >( ctx, m, op, L, dtype, a ); break;
   default: throw std::invalid_argument( "unknown operation" );
   }
}

// owner/copy combine of an accumulation array (cell-array slots) into dst with the apply epilogue:
// cell interiors on the main stream, face/edge/vertex owners (sum of their cell copies, written
// through) on the second stream
template < typename T, typename A, int OP >
static void combine_acc( Context* ctx, Mesh* m, int L, const A* acc, uint32_t flag, T* dst )
{
   P1Level& P = m->level( L );
   struct Join
   {
      Context* c;
      ~Join()
      {
         cudaEventRecord( c->ev_join, c->aux );
         cudaStreamWaitEvent( c->stream, c->ev_join, 0 );
      }
   };
   check_cuda( cudaEventRecord( ctx->ev_fork, ctx->stream ), "fork" );
   check_cuda( cudaStreamWaitEvent( ctx->aux, ctx->ev_fork, 0 ), "fork" );
   Join      j{ ctx };
   const int nrows = int( P.rows.size() );
   if ( nrows > 0 )
   {
      dim3 grid( ( nrows + 7 ) / 8, m->topo.nC );
      k_cell_acc< T, A, OP ><<< grid, 256, 0, ctx->stream >>>( P.n, nrows, P.d_rows, P.d_off + P.nB, P.d_bc + P.nB, flag, acc, nullptr,
                                                                nullptr, nullptr, nullptr, dst, A( 0 ), A( 0 ) );
      ++ctx->launches;
   }
   if ( !P.tasks.empty() )
   {
      launch_bnd_acc< T, A, OP >( ctx->aux, P, flag, 0, acc, nullptr, nullptr, nullptr, nullptr, nullptr, dst, A( 0 ), A( 0 ) );
      ++ctx->launches;
   }
   check_cuda( cudaGetLastError(), "combine launch" );
}

template < typename T, typename A >
static void run_stokes( Context* ctx, Operator* op, int Lp, int divt, const void* const* u, const void* p, void* const* dst_u, void* dst_p,
                        uint32_t flag, int add )
{
   Mesh*      m  = op->mesh;
   const int  Ls = Lp + 1;
   P1Level&   PP = m->level( Lp );
   P1Level&   PU = m->level( Ls );
   ensure_device( m, PP );
   ensure_device( m, PU );
   ensure_stokes_constants();
   if ( !op->d_geom )
   {
      check_cuda( cudaMalloc( &op->d_geom, op->geom.size() * sizeof( CellGeom ) ), "cudaMalloc(geometry)" );
      check_cuda( cudaMemcpy( op->d_geom, op->geom.data(), op->geom.size() * sizeof( CellGeom ), cudaMemcpyHostToDevice ),
                  "upload geometry" );
   }
   ensure_rows( op, Ls );
   ElemLevel& e = op->el[Ls];
   if ( !e.d_sacc )
      check_cuda( cudaMalloc( &e.d_sacc, size_t( 3 * PU.size + PP.size ) * sizeof( double ) ), "cudaMalloc(Stokes scratch)" );
   A* acc_u = reinterpret_cast< A* >( e.d_sacc );
   A* acc_p = acc_u + 3 * PU.size;
   if ( divt ) check_cuda( cudaMemsetAsync( acc_u, 0, size_t( 3 * PU.size ) * sizeof( A ), ctx->stream ), "cudaMemset" );
   else check_cuda( cudaMemsetAsync( acc_p, 0, size_t( PP.size ) * sizeof( A ), ctx->stream ), "cudaMemset" );
   const int nC = m->topo.nC;
   for ( int pc = 0; pc < 8; ++pc )
   {
      const int na = e.aoff[pc + 1] - e.aoff[pc];
      if ( na <= 0 ) continue;
      const int bs = pass_block( na, 256 );
      dim3      grid( ( na + bs - 1 ) / bs, nC );
      const T* u0 = u ? (const T*) u[0] : nullptr;
      const T* u1 = u ? (const T*) u[1] : nullptr;
      const T* u2 = u ? (const T*) u[2] : nullptr;
      if ( divt )
         k_stokes_div_pass< T, A, 1 ><<< grid, bs, 0, ctx->stream >>>( 1 << Lp, na, e.d_anch + e.aoff[pc], PP.d_off + PP.nB,
                                                                         PU.d_off + PU.nB, op->d_geom, u0, u1, u2, (const T*) p, acc_p,
                                                                         acc_u, acc_u + PU.size, acc_u + 2 * PU.size, PP.size, PU.size,
                                                                         ctx->d_error );
      else
         k_stokes_div_pass< T, A, 0 ><<< grid, bs, 0, ctx->stream >>>( 1 << Lp, na, e.d_anch + e.aoff[pc], PP.d_off + PP.nB,
                                                                         PU.d_off + PU.nB, op->d_geom, u0, u1, u2, (const T*) p, acc_p,
                                                                         acc_u, acc_u + PU.size, acc_u + 2 * PU.size, PP.size, PU.size,
                                                                         ctx->d_error );
      ++ctx->launches;
   }
   check_cuda( cudaGetLastError(), "Stokes pass launch" );
   if ( divt )
      for ( int k = 0; k < 3; ++k )
      {
         if ( add ) combine_acc< T, A, OP_APPLY_ADD >( ctx, m, Ls, acc_u + k * PU.size, flag, (T*) dst_u[k] );
         else combine_acc< T, A, OP_APPLY >( ctx, m, Ls, acc_u + k * PU.size, flag, (T*) dst_u[k] );
      }
   else if ( add ) combine_acc< T, A, OP_APPLY_ADD >( ctx, m, Lp, acc_p, flag, (T*) dst_p );
   else combine_acc< T, A, OP_APPLY >( ctx, m, Lp, acc_p, flag, (T*) dst_p );
}

void launch_stokes_div( Context* ctx, Operator* op, int Lp, int dtype, int divt, const void* const* u, const void* p, void* const* dst_u,
                        void* dst_p, uint32_t flag, int add )
{
   if ( dtype == F64 ) run_stokes< double, double >( ctx, op, Lp, divt, u, p, dst_u, dst_p, flag, add );
   else if ( dtype == F32 ) run_stokes< float, float >( ctx, op, Lp, divt, u, p, dst_u, dst_p, flag, add );
   else run_stokes< __half, float >( ctx, op, Lp, divt, u, p, dst_u, dst_p, flag, add );
}

// ---------------------------------------------------------------------------------------------
// Full viscous velocity block (P2ElementwiseBlendingFullViscousOperator.hpp:34-68): block (i, j) is
// the form p2_full_stokesvar_{i}_{j}_blending_q3, int 2 mu eps(u) : eps(v) - (2/3) mu div u div v
// with mu evaluated at the blended point, Yu's 5-point degree-3 rule.  Applied matrix-free per
// micro-cell: at each point the velocity gradient g (g_ik = d u_i / d x_k) of the ten local nodes
// gives the stress s = w mu |det| (g + g^T - (2/3) tr(g) I), and node a of component i receives
// grad phi_a . s_i.  The diagonal pass sums w mu |det| (|grad phi_a|^2 + (1/3) (d_i phi_a)^2).  Same
// parity passes as the coupling blocks (anchors of one class share no P2 node).
// ---------------------------------------------------------------------------------------------
__constant__ double c_yu5_rgrad[5][10][3];

static void ensure_visc_constants()
{
   static PerDeviceOnce once;
   once.run( [] {
      const double lg[4][3] = { { -1, -1, -1 }, { 1, 0, 0 }, { 0, 1, 0 }, { 0, 0, 1 } };
      const int    ed[6][2] = { { 2, 3 }, { 1, 3 }, { 1, 2 }, { 0, 3 }, { 0, 2 }, { 0, 1 } };
      const double pts[5][3] = { { 0.25, 0.25, 0.25 },
                                 { 1.0 / 6.0, 1.0 / 6.0, 1.0 / 6.0 },
                                 { 0.5, 1.0 / 6.0, 1.0 / 6.0 },
                                 { 1.0 / 6.0, 0.5, 1.0 / 6.0 },
                                 { 1.0 / 6.0, 1.0 / 6.0, 0.5 } };
      double g[5][10][3];
      for ( int q = 0; q < 5; ++q )
      {
         const double lam[4] = { 1.0 - pts[q][0] - pts[q][1] - pts[q][2], pts[q][0], pts[q][1], pts[q][2] };
         for ( int i = 0; i < 4; ++i )
            for ( int d = 0; d < 3; ++d ) g[q][i][d] = ( 4.0 * lam[i] - 1.0 ) * lg[i][d];
         for ( int e = 0; e < 6; ++e )
            for ( int d = 0; d < 3; ++d )
               g[q][4 + e][d] = 4.0 * ( lam[ed[e][0]] * lg[ed[e][1]][d] + lam[ed[e][1]] * lg[ed[e][0]][d] );
      }
      check_cuda( cudaMemcpyToSymbol( c_yu5_rgrad, g, sizeof( g ) ), "viscous block constants" );
   } );
}

template < typename T, typename A, int MODE >
__global__ void __launch_bounds__( 128 ) k_visc_pass( int ne, int nanch, const int* __restrict__ anch, const int64_t* __restrict__ off_u,
                                                       const CellGeom* __restrict__ geom, Coefficient kc, const T* __restrict__ u0,
                                                       const T* __restrict__ u1, const T* __restrict__ u2, A* acc0, A* acc1, A* acc2,
                                                       int64_t size_u, int* err )
{
   const int t = blockIdx.x * blockDim.x + threadIdx.x;
   const int c = blockIdx.y;
   if ( t >= nanch ) return;
   const int      a  = anch[t];
   const int      x = a & 1023, y = ( a >> 10 ) & 1023, z = a >> 20, ns = 2 * ne;
   const CellGeom g  = geom[c];
   const int64_t  bu = off_u[c];
   const A        inv_n = A( 1.0 / double( ne ) );
   A              st[3][3];
   for ( int k = 0; k < 3; ++k )
      for ( int d = 0; d < 3; ++d ) st[k][d] = ( A( g.P[k + 1][d] ) - A( g.P[0][d] ) ) * inv_n;
   for ( int ty = 0; ty < 6; ++ty )
   {
      if ( x + y + z > ne - 1 - c_mc_shift[ty] ) continue;
      int V[4][3];
      for ( int m = 0; m < 4; ++m )
         for ( int d = 0; d < 3; ++d ) V[m][d] = ( d == 0 ? x : d == 1 ? y : z ) + c_mc_off[ty][m][d];
      int64_t iu[10];
      for ( int m = 0; m < 4; ++m ) iu[m] = bu + cidx( ns, 2 * V[m][0], 2 * V[m][1], 2 * V[m][2] );
      for ( int e = 0; e < 6; ++e )
      {
         const int ea = c_p2_edge[e][0], eb = c_p2_edge[e][1];
         iu[4 + e]    = bu + cidx( ns, V[ea][0] + V[eb][0], V[ea][1] + V[eb][1], V[ea][2] + V[eb][2] );
      }
      {
         bool bad = false;
         for ( int m = 0; m < 10; ++m ) bad |= iu[m] < 0 || iu[m] >= size_u;
         if ( bad )
         {
            atomicExch( err, 2 );
            continue;
         }
      }
      A X0[3], J[3][3];
      for ( int d = 0; d < 3; ++d )
      {
         X0[d] = A( g.P[0][d] ) + st[0][d] * A( V[0][0] ) + st[1][d] * A( V[0][1] ) + st[2][d] * A( V[0][2] );
         for ( int k = 0; k < 3; ++k )
            J[d][k] = st[0][d] * A( V[k + 1][0] - V[0][0] ) + st[1][d] * A( V[k + 1][1] - V[0][1] ) + st[2][d] * A( V[k + 1][2] - V[0][2] );
      }
      A ul[3][10];
      if constexpr ( MODE == 0 )
         for ( int j = 0; j < 10; ++j )
         {
            ul[0][j] = A( ld_any( u0 + iu[j] ) );
            ul[1][j] = A( ld_any( u1 + iu[j] ) );
            ul[2][j] = A( ld_any( u2 + iu[j] ) );
         }
      A yl[3][10];
      for ( int k = 0; k < 3; ++k )
         for ( int j = 0; j < 10; ++j ) yl[k][j] = A( 0 );
      for ( int q = 0; q < 5; ++q )
      {
         A Mi[3][3], adet, Fq[3];
         mapped_point( g, X0, J, c_yu5_pts[q], Mi, adet, Fq );
         const A s = A( c_yu5_w[q] ) * coeff_eval( kc, Fq ) * adet;
         if constexpr ( MODE == 0 )
         {
            A gr[3][3];
            for ( int i = 0; i < 3; ++i )
               for ( int k = 0; k < 3; ++k ) gr[i][k] = A( 0 );
            for ( int b = 0; b < 10; ++b )
            {
               A G[3];
               for ( int k = 0; k < 3; ++k )
                  G[k] = A( c_yu5_rgrad[q][b][0] ) * Mi[0][k] + A( c_yu5_rgrad[q][b][1] ) * Mi[1][k] + A( c_yu5_rgrad[q][b][2] ) * Mi[2][k];
               for ( int i = 0; i < 3; ++i )
                  for ( int k = 0; k < 3; ++k ) gr[i][k] += ul[i][b] * G[k];
            }
            const A tr3 = A( 2.0 / 3.0 ) * ( gr[0][0] + gr[1][1] + gr[2][2] );
            A       sg[3][3];
            for ( int i = 0; i < 3; ++i )
               for ( int k = 0; k < 3; ++k ) sg[i][k] = s * ( ( gr[i][k] + gr[k][i] ) - ( i == k ? tr3 : A( 0 ) ) );
            for ( int b = 0; b < 10; ++b )
            {
               A G[3];
               for ( int k = 0; k < 3; ++k )
                  G[k] = A( c_yu5_rgrad[q][b][0] ) * Mi[0][k] + A( c_yu5_rgrad[q][b][1] ) * Mi[1][k] + A( c_yu5_rgrad[q][b][2] ) * Mi[2][k];
               for ( int i = 0; i < 3; ++i ) yl[i][b] += G[0] * sg[i][0] + G[1] * sg[i][1] + G[2] * sg[i][2];
            }
         }
         else
            for ( int b = 0; b < 10; ++b )
            {
               A G[3];
               for ( int k = 0; k < 3; ++k )
                  G[k] = A( c_yu5_rgrad[q][b][0] ) * Mi[0][k] + A( c_yu5_rgrad[q][b][1] ) * Mi[1][k] + A( c_yu5_rgrad[q][b][2] ) * Mi[2][k];
               const A gg = G[0] * G[0] + G[1] * G[1] + G[2] * G[2];
               for ( int i = 0; i < 3; ++i ) yl[i][b] += s * ( gg + A( 1.0 / 3.0 ) * G[i] * G[i] );
            }
      }
      for ( int j = 0; j < 10; ++j )
      {
         acc0[iu[j]] += yl[0][j];
         acc1[iu[j]] += yl[1][j];
         acc2[iu[j]] += yl[2][j];
      }
   }
}

template < typename T, typename A >
static void run_visc( Context* ctx, Operator* op, int Lp, int mode, const void* const* u, void* const* dst, uint32_t flag, int add )
{
   Mesh*     m  = op->mesh;
   const int Ls = Lp + 1;
   P1Level&  PU = m->level( Ls );
   ensure_device( m, PU );
   ensure_visc_constants();
   if ( !op->d_geom )
   {
      check_cuda( cudaMalloc( &op->d_geom, op->geom.size() * sizeof( CellGeom ) ), "cudaMalloc(geometry)" );
      check_cuda( cudaMemcpy( op->d_geom, op->geom.data(), op->geom.size() * sizeof( CellGeom ), cudaMemcpyHostToDevice ),
                  "upload geometry" );
   }
   ensure_rows( op, Ls );
   ElemLevel& e = op->el[Ls];
   if ( !e.d_sacc ) check_cuda( cudaMalloc( &e.d_sacc, size_t( 3 * PU.size ) * sizeof( double ) ), "cudaMalloc(viscous block scratch)" );
   A* acc = reinterpret_cast< A* >( e.d_sacc );
   check_cuda( cudaMemsetAsync( acc, 0, size_t( 3 * PU.size ) * sizeof( A ), ctx->stream ), "cudaMemset" );
   const int nC = m->topo.nC;
   const T*  u0 = u ? (const T*) u[0] : nullptr;
   const T*  u1 = u ? (const T*) u[1] : nullptr;
   const T*  u2 = u ? (const T*) u[2] : nullptr;
   for ( int pc = 0; pc < 8; ++pc )
   {
      const int na = e.aoff[pc + 1] - e.aoff[pc];
      if ( na <= 0 ) continue;
      const int bs = pass_block( na, 128 );
      dim3      grid( ( na + bs - 1 ) / bs, nC );
      if ( mode == 0 )
         k_visc_pass< T, A, 0 ><<< grid, bs, 0, ctx->stream >>>( 1 << Lp, na, e.d_anch + e.aoff[pc], PU.d_off + PU.nB, op->d_geom, op->coeff,
                                                                 u0, u1, u2, acc, acc + PU.size, acc + 2 * PU.size, PU.size,
                                                                 ctx->d_error );
      else
         k_visc_pass< T, A, 1 ><<< grid, bs, 0, ctx->stream >>>( 1 << Lp, na, e.d_anch + e.aoff[pc], PU.d_off + PU.nB, op->d_geom, op->coeff,
                                                                 u0, u1, u2, acc, acc + PU.size, acc + 2 * PU.size, PU.size,
                                                                 ctx->d_error );
      ++ctx->launches;
   }
   check_cuda( cudaGetLastError(), "viscous block pass launch" );
   if ( mode == 0 )
   {
      for ( int k = 0; k < 3; ++k )
      {
         if ( add ) combine_acc< T, A, OP_APPLY_ADD >( ctx, m, Ls, acc + k * PU.size, flag, (T*) dst[k] );
         else combine_acc< T, A, OP_APPLY >( ctx, m, Ls, acc + k * PU.size, flag, (T*) dst[k] );
      }
      return;
   }
   // diagonal: owners sum their copies, then 1/diag on every owned node (dst: three A arrays)
   const int nrows = int( PU.rows.size() );
   for ( int k = 0; k < 3; ++k )
   {
      A* invd = reinterpret_cast< A* >( dst[k] );
      check_cuda( cudaMemsetAsync( invd, 0, size_t( PU.size ) * sizeof( A ), ctx->stream ), "cudaMemset" );
      if ( nrows > 0 )
      {
         dim3 grid( ( nrows + 7 ) / 8, nC );
         k_cell_invert< A ><<< grid, 256, 0, ctx->stream >>>( PU.n, nrows, PU.d_rows, PU.d_off + PU.nB, acc + k * PU.size, invd );
      }
      if ( !PU.tasks.empty() )
         launch_bnd_acc< T, A, OP_APPLY >( ctx->stream, PU, kAll, 0, acc + k * PU.size, nullptr, invd, nullptr, nullptr, nullptr, nullptr,
                                           A( 0 ), A( 0 ) );
   }
   check_cuda( cudaGetLastError(), "viscous block diagonal launch" );
}

void launch_full_viscous( Context* ctx, Operator* op, int Lp, int dtype, int mode, const void* const* u, void* const* dst, uint32_t flag,
                          int add )
{
   if ( dtype == F64 ) run_visc< double, double >( ctx, op, Lp, mode, u, dst, flag, add );
   else if ( dtype == F32 ) run_visc< float, float >( ctx, op, Lp, mode, u, dst, flag, add );
   else run_visc< __half, float >( ctx, op, Lp, mode, u, dst, flag, add );
}

void launch_elementwise( Context* ctx, Mesh* m, Operator* op, int L, int dtype, const StencilArgs& a )
{
   ensure_elementwise_level( ctx, op, L, dtype );
   if ( dtype == F64 ) dispatch_elem< double, double >( ctx, m, op, L, dtype, a );
   else if ( dtype == F32 ) dispatch_elem< float, float >( ctx, m, op, L, dtype, a );
   else dispatch_elem< __half, float >( ctx, m, op, L, dtype, a );
}

}  // namespace hyb
