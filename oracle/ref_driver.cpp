// C entry points around the reference's own generated P1 kernels and FEniCS P1 diffusion form,
// compiled from the reference sources in place (see oracle/Makefile).  TEST INFRASTRUCTURE ONLY:
// used by tests/ to pin the oracle and by bench.py's CPU baseline, never by the product.
//
// Wrapped reference code:
//   src/constant_stencil_operator/P1generatedKernels/apply_3D_macrocell_vertexdof_to_vertexdof_replace.cpp
//   src/hyteg/gridtransferoperators/generatedKernels/restrict_3D_macrocell_P1_pull_additive.cpp
//   src/hyteg/gridtransferoperators/generatedKernels/prolongate_3D_macrocell_P1_push_additive.cpp
//   src/hyteg/forms/form_fenics_generated/p1_tet_diffusion.h (tabulate_tensor)
#include <map>
#include <omp.h>
#include <cmath>
#include <memory>

#include "apply_3D_macrocell_vertexdof_to_vertexdof_replace.hpp"
#include "hyteg/forms/form_fenics_generated/p1_tet_diffusion.h"
#include "prolongate_3D_macrocell_P1_push_additive.hpp"
#include "restrict_3D_macrocell_P1_pull_additive.hpp"

using hyteg::indexing::Index;

// stencil order: centre, W E S N B T NW SE TW BE TS BN TSE BNW
static const int kDirs[15][3] = { { 0, 0, 0 },  { -1, 0, 0 }, { 1, 0, 0 },  { 0, -1, 0 }, { 0, 1, 0 },
                                  { 0, 0, -1 }, { 0, 0, 1 },  { -1, 1, 0 }, { 1, -1, 0 }, { -1, 0, 1 },
                                  { 1, 0, -1 }, { 0, -1, 1 }, { 0, 1, -1 }, { 1, -1, 1 }, { -1, 1, -1 } };

static std::map< Index, double > stencil_map( const double* s )
{
   std::map< Index, double > m;
   for ( int d = 0; d < 15; ++d ) m[Index( kDirs[d][0], kDirs[d][1], kDirs[d][2] )] = s[d];
   return m;
}

extern "C" {

void ref_cell_apply( double* dst, const double* src, int level, const double* stencil15 )
{
   auto m = stencil_map( stencil15 );
   hyteg::vertexdof::macrocell::generated::apply_3D_macrocell_vertexdof_to_vertexdof_replace< double >( dst, src, level, m );
}

// one macro-cell per OpenMP thread, like one MPI rank per macro-cell
void ref_cell_apply_many( int ncells, double* const* dst, const double* const* src, int level, const double* stencils,
                          int threads )
{
#pragma omp parallel for num_threads( threads ) schedule( static, 1 )
   for ( int c = 0; c < ncells; ++c )
      ref_cell_apply( dst[c], src[c], level, stencils + 15 * c );
}

void ref_restrict( double* coarse, const double* fine, int coarse_level, const double* nc14 )
{
   // nc14: edges 0-5, faces 0-3, vertices 0-3 (number of macro-cells around each)
   hyteg::vertexdof::macrocell::generated::restrict_3D_macrocell_P1_pull_additive< double >(
       coarse, fine, coarse_level, nc14[0], nc14[1], nc14[2], nc14[3], nc14[4], nc14[5], nc14[6], nc14[7], nc14[8], nc14[9],
       nc14[10], nc14[11], nc14[12], nc14[13] );
}

void ref_prolongate( const double* coarse, double* fine, int coarse_level, const double* nc14 )
{
   hyteg::vertexdof::macrocell::generated::prolongate_3D_macrocell_P1_push_additive< double >(
       coarse, fine, coarse_level, nc14[0], nc14[1], nc14[2], nc14[3], nc14[4], nc14[5], nc14[6], nc14[7], nc14[8], nc14[9],
       nc14[10], nc14[11], nc14[12], nc14[13] );
}

void ref_p1_diffusion_element( const double* coords12, double* A16 )
{
   p1_tet_diffusion_cell_integral_0_otherwise form;
   form.tabulate_tensor( A16, nullptr, coords12, 0 );
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// HyTeG-generated P1 variable-coefficient diffusion form with blending
// (src/hyteg/forms/form_hyteg_generated/p1/p1_div_k_grad_blending_q3.cpp)
// ---------------------------------------------------------------------------------------------
#include "hyteg/forms/form_hyteg_generated/p1/p1_div_k_grad_blending_q3.hpp"

namespace {
// test blending maps: 0 identity; 1 F(x) = x (1 + a x0 x1) (a smooth non-affine map of the tests)
struct TestMap : public hyteg::GeometryMap
{
   int    kind = 0;
   double a    = 0;
   void   evalF( const hyteg::Point3D& x, hyteg::Point3D& F ) const override
   {
      const double s = kind == 1 ? 1.0 + a * x[0] * x[1] : 1.0;
      F              = hyteg::Point3D( x[0] * s, x[1] * s, x[2] * s );
   }
   double evalDF( const hyteg::Point3D& x, hyteg::Matrix3r& D ) const override
   {
      const double s    = kind == 1 ? 1.0 + a * x[0] * x[1] : 1.0;
      const double g[3] = { kind == 1 ? a * x[1] : 0.0, kind == 1 ? a * x[0] : 0.0, 0.0 };
      for ( int i = 0; i < 3; ++i )
         for ( int j = 0; j < 3; ++j ) D( i, j ) = ( i == j ? s : 0.0 ) + x[i] * g[j];
      return D( 0, 0 ) * ( D( 1, 1 ) * D( 2, 2 ) - D( 1, 2 ) * D( 2, 1 ) ) - D( 0, 1 ) * ( D( 1, 0 ) * D( 2, 2 ) - D( 1, 2 ) * D( 2, 0 ) ) +
             D( 0, 2 ) * ( D( 1, 0 ) * D( 2, 1 ) - D( 1, 1 ) * D( 2, 0 ) );
   }
};
}  // namespace

extern "C" void ref_p1_divkgrad_blending_element( const double* coords12, int map_kind, double map_a, double k_amp,
                                                   const double* k_phase3, double* A16 )
{
   auto   map   = std::make_shared< TestMap >();
   map->kind    = map_kind;
   map->a       = map_a;
   const double amp = k_amp;
   const double ph[3] = { k_phase3[0], k_phase3[1], k_phase3[2] };
   auto k3 = [amp, ph]( const hyteg::Point3D& p ) {
      const double tp = 2.0 * 3.14159265358979323846;
      return std::exp( amp * std::sin( tp * ( p[0] + ph[0] ) ) * std::cos( tp * ( p[1] + ph[1] ) ) * std::sin( tp * ( p[2] + ph[2] ) ) );
   };
   auto                                   k2 = []( const hyteg::Point3D& ) { return 1.0; };
   hyteg::forms::p1_div_k_grad_blending_q3 form( k3, k2 );
   form.setGeometryMap( map );
   std::array< hyteg::Point3D, 4 > c;
   for ( int v = 0; v < 4; ++v ) c[v] = hyteg::Point3D( coords12[3 * v], coords12[3 * v + 1], coords12[3 * v + 2] );
   hyteg::Matrix< double, 4, 4 > M;
   form.integrateAll( c, M );
   for ( int i = 0; i < 16; ++i ) A16[i] = M.a[i];
}

// ---------------------------------------------------------------------------------------------
// HyTeG-generated P2 variable-coefficient diffusion form with blending
// (src/hyteg/forms/form_hyteg_generated/p2/p2_div_k_grad_blending_q4.cpp), same test maps and
// coefficient as the P1 form above.  Element DoFs: 4 vertices, then the edges (2,3), (1,3), (1,2),
// (0,3), (0,2), (0,1).
// ---------------------------------------------------------------------------------------------
#include "hyteg/forms/form_hyteg_generated/p2/p2_div_k_grad_blending_q4.hpp"

extern "C" void ref_p2_divkgrad_blending_element( const double* coords12, int map_kind, double map_a, double k_amp,
                                                   const double* k_phase3, double* A100 )
{
   auto map  = std::make_shared< TestMap >();
   map->kind = map_kind;
   map->a    = map_a;
   const double amp   = k_amp;
   const double ph[3] = { k_phase3[0], k_phase3[1], k_phase3[2] };
   auto k3 = [amp, ph]( const hyteg::Point3D& p ) {
      const double tp = 2.0 * 3.14159265358979323846;
      return std::exp( amp * std::sin( tp * ( p[0] + ph[0] ) ) * std::cos( tp * ( p[1] + ph[1] ) ) * std::sin( tp * ( p[2] + ph[2] ) ) );
   };
   auto                                   k2 = []( const hyteg::Point3D& ) { return 1.0; };
   hyteg::forms::p2_div_k_grad_blending_q4 form( k2, k3 );  // (2D callback, 3D callback)
   form.setGeometryMap( map );
   std::array< hyteg::Point3D, 4 > c;
   for ( int v = 0; v < 4; ++v ) c[v] = hyteg::Point3D( coords12[3 * v], coords12[3 * v + 1], coords12[3 * v + 2] );
   hyteg::Matrix< double, 10, 10 > M;
   form.integrateAll( c, M );
   for ( int i = 0; i < 100; ++i ) A100[i] = M.a[i];
}

// CPU timing of the reference's per-micro-cell work in P2ElementwiseOperator::apply
// (P2ElementwiseOperator.cpp:203-220: integrateAll of p2_div_k_grad_blending_q4, then y += K x on the
// ten element DoFs) over `ncells` micro-cells of a refined tetrahedron, with the smooth test blending
// map standing in for the shell map, OpenMP over micro-cells.  Returns the wall-clock seconds.
#include <chrono>
#include <omp.h>
extern "C" double ref_p2_elem_apply_bench( long ncells, int threads, double k_amp )
{
   const double ph[3] = { 0.13, 0.27, 0.41 };
   auto         t0    = std::chrono::steady_clock::now();
   double       sink  = 0;
#pragma omp parallel num_threads( threads ) reduction( + : sink )
   {
      auto map  = std::make_shared< TestMap >();
      map->kind = 1;
      map->a    = 0.1;
      auto k3   = [k_amp, &ph]( const hyteg::Point3D& p ) {
         const double tp = 2.0 * 3.14159265358979323846;
         return std::exp( k_amp * std::sin( tp * ( p[0] + ph[0] ) ) * std::cos( tp * ( p[1] + ph[1] ) ) * std::sin( tp * ( p[2] + ph[2] ) ) );
      };
      auto                                   k2 = []( const hyteg::Point3D& ) { return 1.0; };
      hyteg::forms::p2_div_k_grad_blending_q4 form( k2, k3 );
      form.setGeometryMap( map );
      double x[10], y[10] = {};
      for ( int i = 0; i < 10; ++i ) x[i] = 0.1 * ( i + 1 );
      const double h = 1.0 / 64.0;
#pragma omp for schedule( static )
      for ( long c = 0; c < ncells; ++c )
      {
         const double o[3] = { h * double( c % 61 ), h * double( ( c / 61 ) % 59 ), h * double( ( c / 3599 ) % 53 ) };
         std::array< hyteg::Point3D, 4 > v = { hyteg::Point3D( o[0], o[1], o[2] ), hyteg::Point3D( o[0] + h, o[1], o[2] ),
                                               hyteg::Point3D( o[0], o[1] + h, o[2] ), hyteg::Point3D( o[0], o[1], o[2] + h ) };
         hyteg::Matrix< double, 10, 10 > K;
         form.integrateAll( v, K );
         for ( int i = 0; i < 10; ++i )
            for ( int j = 0; j < 10; ++j ) y[i] += K( i, j ) * x[j];
      }
      for ( int i = 0; i < 10; ++i ) sink += y[i];
   }
   const double s = std::chrono::duration< double >( std::chrono::steady_clock::now() - t0 ).count();
   return sink == 12345.678 ? -s : s;  // keep the work observable
}

// ---------------------------------------------------------------------------------------------
// Stokes blocks (P2P1ElementwiseBlendingStokesOperator: div P2ToP1ElementwiseBlendingDiv{x,y,z}
// with p2_to_p1_div_{0,1,2}_blending_q2, divT P1ToP2ElementwiseBlendingDivT{x,y,z} with
// p1_to_p2_divt_{0,1,2}_blending_q2) and the PSPG element matrix whose inverted diagonal is the
// Uzawa pressure scaling (P1PSPGInvDiagOperator, P1ConstantOperator.hpp:205-210, form
// p1_tet_pspg_tet.h).  Row-major element matrices.
// ---------------------------------------------------------------------------------------------
#include "hyteg/forms/form_hyteg_generated/p2_to_p1/p2_to_p1_div_blending_q2.hpp"
#include "hyteg/forms/form_hyteg_generated/p1_to_p2/p1_to_p2_divt_blending_q2.hpp"
#include "hyteg/forms/form_fenics_generated/p1_tet_pspg_tet.h"

extern "C" void ref_p2p1_div_element( const double* coords12, int map_kind, double map_a, int comp, double* A40 )
{
   auto map  = std::make_shared< TestMap >();
   map->kind = map_kind;
   map->a    = map_a;
   std::array< hyteg::Point3D, 4 > c;
   for ( int v = 0; v < 4; ++v ) c[v] = hyteg::Point3D( coords12[3 * v], coords12[3 * v + 1], coords12[3 * v + 2] );
   hyteg::Matrix< double, 4, 10 > M;
   if ( comp == 0 )
   {
      hyteg::forms::p2_to_p1_div_0_blending_q2 f;
      f.setGeometryMap( map );
      f.integrateAll( c, M );
   }
   else if ( comp == 1 )
   {
      hyteg::forms::p2_to_p1_div_1_blending_q2 f;
      f.setGeometryMap( map );
      f.integrateAll( c, M );
   }
   else
   {
      hyteg::forms::p2_to_p1_div_2_blending_q2 f;
      f.setGeometryMap( map );
      f.integrateAll( c, M );
   }
   for ( int i = 0; i < 40; ++i ) A40[i] = M.a[i];
}

extern "C" void ref_p1p2_divt_element( const double* coords12, int map_kind, double map_a, int comp, double* A40 )
{
   auto map  = std::make_shared< TestMap >();
   map->kind = map_kind;
   map->a    = map_a;
   std::array< hyteg::Point3D, 4 > c;
   for ( int v = 0; v < 4; ++v ) c[v] = hyteg::Point3D( coords12[3 * v], coords12[3 * v + 1], coords12[3 * v + 2] );
   hyteg::Matrix< double, 10, 4 > M;
   if ( comp == 0 )
   {
      hyteg::forms::p1_to_p2_divt_0_blending_q2 f;
      f.setGeometryMap( map );
      f.integrateAll( c, M );
   }
   else if ( comp == 1 )
   {
      hyteg::forms::p1_to_p2_divt_1_blending_q2 f;
      f.setGeometryMap( map );
      f.integrateAll( c, M );
   }
   else
   {
      hyteg::forms::p1_to_p2_divt_2_blending_q2 f;
      f.setGeometryMap( map );
      f.integrateAll( c, M );
   }
   for ( int i = 0; i < 40; ++i ) A40[i] = M.a[i];
}

extern "C" void ref_p1_pspg_element( const double* coords12, double* A16 )
{
   p1_tet_pspg_tet_cell_integral_0_otherwise form;
   form.tabulate_tensor( A16, nullptr, coords12, 0 );
}

// ---------------------------------------------------------------------------------------------
// Full viscous velocity block (P2ElementwiseBlendingFullViscousOperator, .hpp:34-68): block (i, j)
// is p2_full_stokesvar_{i}_{j}_blending_q3 with the variable viscosity mu (the exp-sin test
// coefficient here), 2 mu eps(u) : eps(v) - (2/3) mu div u div v.  Row-major 10x10 element matrix.
// ---------------------------------------------------------------------------------------------
#include "hyteg/forms/form_hyteg_generated/p2/p2_full_stokesvar_blending_q3.hpp"

extern "C" void ref_p2_full_viscous_element( const double* coords12, int map_kind, double map_a, int bi, int bj, double k_amp,
                                              const double* k_phase3, double* A100 )
{
   auto map  = std::make_shared< TestMap >();
   map->kind = map_kind;
   map->a    = map_a;
   const double amp   = k_amp;
   const double ph[3] = { k_phase3[0], k_phase3[1], k_phase3[2] };
   std::function< double( const hyteg::Point3D& ) > mu = [amp, ph]( const hyteg::Point3D& p ) {
      const double tp = 2.0 * 3.14159265358979323846;
      return std::exp( amp * std::sin( tp * ( p[0] + ph[0] ) ) * std::cos( tp * ( p[1] + ph[1] ) ) * std::sin( tp * ( p[2] + ph[2] ) ) );
   };
   std::array< hyteg::Point3D, 4 > c;
   for ( int v = 0; v < 4; ++v ) c[v] = hyteg::Point3D( coords12[3 * v], coords12[3 * v + 1], coords12[3 * v + 2] );
   hyteg::Matrix< double, 10, 10 > M;
   auto run = [&]( auto&& f ) {
      f.setGeometryMap( map );
      f.integrateAll( c, M );
   };
   using namespace hyteg::forms;
   const int b = 3 * bi + bj;
   if ( b == 0 ) run( p2_full_stokesvar_0_0_blending_q3( mu, mu ) );
   else if ( b == 1 ) run( p2_full_stokesvar_0_1_blending_q3( mu, mu ) );
   else if ( b == 2 ) run( p2_full_stokesvar_0_2_blending_q3( mu ) );
   else if ( b == 3 ) run( p2_full_stokesvar_1_0_blending_q3( mu, mu ) );
   else if ( b == 4 ) run( p2_full_stokesvar_1_1_blending_q3( mu, mu ) );
   else if ( b == 5 ) run( p2_full_stokesvar_1_2_blending_q3( mu ) );
   else if ( b == 6 ) run( p2_full_stokesvar_2_0_blending_q3( mu ) );
   else if ( b == 7 ) run( p2_full_stokesvar_2_1_blending_q3( mu ) );
   else run( p2_full_stokesvar_2_2_blending_q3( mu ) );
   for ( int i = 0; i < 100; ++i ) A100[i] = M.a[i];
}
