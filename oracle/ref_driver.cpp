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
