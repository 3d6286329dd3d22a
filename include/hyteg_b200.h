/*
 * hyteg_b200 — C ABI of the B200 matrix-free multigrid path for HyTeG-style hybrid
 * tetrahedral grids.
 *
 * Every entry point returns an int status (HYB_OK on success) and never throws.  On failure
 * hyb_last_error() returns a message for the calling thread.  All handles are opaque; every
 * create has a matching destroy.  Device work is issued on the context's CUDA stream; entry
 * points that return host values (dot products, residual histories, downloads) synchronise that
 * stream, the others are asynchronous.
 *
 * The reference interface each group replaces is cited per declaration (paths relative to the
 * hyteg source tree).
 */
#ifndef HYTEG_B200_H
#define HYTEG_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes (reference: WALBERLA_ABORT / WALBERLA_CHECK abort the process, e.g.
 * src/hyteg/operators/Operator.hpp:80; here they become return codes) */
#define HYB_OK 0
#define HYB_EINVAL 1
#define HYB_ENOMEM 2
#define HYB_EDEVICE 3
#define HYB_ETIMEOUT 4
#define HYB_EINTERNAL 5

/* value types of function storage (FunctionMemory<ValueType>, src/hyteg/memory/FunctionMemory.hpp:47-130) */
#define HYB_F64 0
#define HYB_F32 1
#define HYB_F16 2

/* DoFType bits (src/hyteg/types/types.hpp:29-43) */
#define HYB_INNER 1u
#define HYB_DIRICHLET 2u
#define HYB_NEUMANN 4u
#define HYB_FREESLIP 8u
#define HYB_ALL 15u

/* UpdateType (src/hyteg/types/types.hpp:88-92) */
#define HYB_REPLACE 0
#define HYB_ADD 1

/* operator kinds */
#define HYB_P1_CONST_LAPLACE 1 /* P1ConstantLaplaceOperator, constant_stencil_operator/P1ConstantOperator.hpp:167 */
#define HYB_P1_CONST_MASS 2    /* P1ConstantMassOperator, same file */

#define HYB_P1_ELEM_DIVKGRAD 3 /* P1ElementwiseBlendingDivKGradOperator (elementwiseoperators/P1ElementwiseOperator.hpp:329-373)
                                  with the form p1_div_k_grad_blending_q3 */
#define HYB_P2_ELEM_DIVKGRAD 4 /* P2ElementwiseBlendingDivKGradOperator (elementwiseoperators/P2ElementwiseOperator.hpp:475) */
#define HYB_P2P1_DIV 5 /* P2ToP1ElementwiseBlendingDivOperator / P1ToP2ElementwiseBlendingDivTOperator (P2P1ElementwiseBlendingStokesOperator.hpp:113-116) */
#define HYB_P1_PSPG 6  /* P1PSPGOperator; its inverted diagonal is P1PSPGInvDiagOperator (P1ConstantOperator.hpp:200-210) */
#define HYB_P2_FULL_VISCOUS 7 /* P2ElementwiseBlendingFullViscousOperator (elementwiseoperators/P2ElementwiseBlendingFullViscousOperator.hpp:34-68) */
#define HYB_P2_CONST_LAPLACE 8 /* P2ConstantLaplaceOperator: P2ConstantOperator (constant_stencil_operator/P2ConstantOperator.cpp:100-114), levels are P2 levels */

/* blending maps (geometry/) */
#define HYB_BLEND_NONE 0
#define HYB_BLEND_SHELL 1 /* IcosahedralShellMap (geometry/IcosahedralShellMap.hpp) */

/* coefficient families k(x) */
#define HYB_COEFF_CONSTANT 0 /* k = value */
#define HYB_COEFF_EXPSIN 1   /* k = exp(amp sin(2 pi f (x+p0)) cos(2 pi f (y+p1)) sin(2 pi f (z+p2))) */
#define HYB_COEFF_RADIAL_EXP 2 /* k = exp(amp (value - |x|) / freq): radial viscosity profile, e.g. amp 2.99, value 1, freq 0.45 */

typedef struct hyb_coeff
{
   int    kind;
   double value;
   double amp;
   double freq;
   double phase[3];
} hyb_coeff;

/* smoother kinds */
#define HYB_SMOOTHER_JACOBI 0    /* solvers/WeightedJacobiSmoother.hpp:46-66 */
#define HYB_SMOOTHER_CHEBYSHEV 1 /* solvers/ChebyshevSmoother.hpp:112-240 */
#define HYB_SMOOTHER_GAUSS_SEIDEL 2 /* solvers/GaussSeidelSmoother.hpp:31-60: smooth_gs (SOR with relax 1) */
#define HYB_SMOOTHER_SOR 3          /* solvers/SORSmoother.hpp: smooth_sor with relax = jacobi_relax */

#define HYB_VCYCLE 0 /* CycleType::VCYCLE, solvers/GeometricMultigridSolver.hpp */
#define HYB_WCYCLE 1

typedef struct hyb_ctx  hyb_ctx;
typedef struct hyb_mesh hyb_mesh;
typedef struct hyb_fn   hyb_fn;
typedef struct hyb_op   hyb_op;
typedef struct hyb_gmg  hyb_gmg;

/* ---------------------------------------------------------------- context and errors */
const char* hyb_version( void );
/* message of the last failed call on this thread */
const char* hyb_last_error( void );
/* device: CUDA ordinal; stream: a cudaStream_t to issue work on, or NULL for a private stream */
int hyb_ctx_create( int device, void* stream, hyb_ctx** out );
int hyb_ctx_destroy( hyb_ctx* ctx );
int hyb_ctx_synchronize( hyb_ctx* ctx );
/* number of kernels this library launched through ctx so far */
int hyb_ctx_launch_count( const hyb_ctx* ctx, int64_t* out );
/* the context's stream (cudaStream_t) */
int hyb_ctx_stream( const hyb_ctx* ctx, void** stream );
/* bytes of device scratch the context holds (reduction partials, smoother scratch, transfer staging,
 * buffers kept for captured graphs); no counterpart in the reference */
int hyb_ctx_scratch_bytes( const hyb_ctx* ctx, int64_t* out );

/* ---------------------------------------------------------------- macro mesh and primitive storage
 * Replaces MeshInfo (src/hyteg/mesh/MeshInfo.hpp:221,512,562) + SetupPrimitiveStorage
 * (src/hyteg/primitivestorage/SetupPrimitiveStorage.hpp:45) + PrimitiveStorage
 * (src/hyteg/primitivestorage/PrimitiveStorage.hpp:116).  Primitive ids and local orientations
 * follow the reference; boundary flags default to setMeshBoundaryFlagsOnBoundary(1, 0, true) and
 * flag -> DoFType to BoundaryCondition::create0123BC (0 Inner, 1 Dirichlet, 2 Neumann, 3 Freeslip). */
int hyb_mesh_create( hyb_ctx* ctx, int nverts, const double* coords /* 3*nverts */, int ntets, const int* tets /* 4*ntets */,
                     hyb_mesh** out );
/* MeshInfo::meshCuboid (src/hyteg/mesh/MeshGenCuboid.cpp:35-172) */
int hyb_mesh_create_cuboid( hyb_ctx* ctx, const double* lo, const double* hi, int nx, int ny, int nz, hyb_mesh** out );
/* MeshInfo::meshSphericalShell(ntan, nrad, rmin, rmax) with the default SHELLMESH_CLASSIC flavour
 * (src/hyteg/mesh/MeshGenSphericalShell.cpp:642-765); ntan-1 must be a power of two */
int hyb_mesh_create_spherical_shell( hyb_ctx* ctx, int ntan, int nrad, double rmin, double rmax, hyb_mesh** out );
/* MeshInfo::fromGmshFile, MSH 2.2 and 4.1 tetrahedral meshes (src/hyteg/mesh/GmshReaderForMSH22.hpp) */
int hyb_mesh_create_gmsh( hyb_ctx* ctx, const char* path, hyb_mesh** out );
int hyb_mesh_destroy( hyb_mesh* mesh );
/* SetupPrimitiveStorage::setMeshBoundaryFlagsOnBoundary (SetupPrimitiveStorage.cpp:977-988) */
int hyb_mesh_set_boundary_flags_on_boundary( hyb_mesh* mesh, int on_boundary, int inner );
/* BoundaryCondition: DoFType of primitives carrying mesh boundary flag `flag` */
int hyb_mesh_set_bc_type( hyb_mesh* mesh, int flag, uint32_t dof_type );
/* counts[4] = macro vertices, edges, faces, cells */
int hyb_mesh_counts( const hyb_mesh* mesh, int* counts );
/* kind 0 vertex, 1 edge, 2 face, 3 cell: vertex ids of primitive `id` in its local order (-1 padded) */
int hyb_mesh_primitive_vertices( const hyb_mesh* mesh, int kind, int id, int* out4 );
/* coordinates of all macro-vertices in id order (3 doubles each) */
int hyb_mesh_vertex_coords( const hyb_mesh* mesh, double* out );
/* mesh boundary flag of a primitive */
int hyb_mesh_primitive_flag( const hyb_mesh* mesh, int kind, int id, int* flag );

/* ---------------------------------------------------------------- vertex-DoF layout
 * Packed HyTeG layout of one level: every primitive's FunctionMemory array
 * (p1functionspace/VertexDoFMemory.hpp:39-60: vertex 1+nEdges, edge (n+1)+nFaces*n+nCells*(n-1),
 * face tri(n+1)+nCells*tri(n), cell tet(n+1)) concatenated in id order vertices, edges, faces, cells. */
int hyb_layout_packed_size( hyb_mesh* mesh, int level, int64_t* size );
/* packed offsets and sizes of all primitives (nV+nE+nF+nC entries each; either may be NULL) */
int hyb_layout_primitive_offsets( hyb_mesh* mesh, int level, int64_t* offsets, int64_t* sizes );
/* linearMacroCellIndex / linearMacroFaceIndex (indexing/MacroCellIndexing.hpp:45-52, MacroFaceIndexing.hpp:45-50) */
int64_t hyb_layout_cell_index( int level, int x, int y, int z );
int64_t hyb_layout_face_index( int level, int i, int j );

/* ---------------------------------------------------------------- functions
 * P1Function<ValueType> (p1functionspace/P1Function.hpp, VertexDoFFunction.hpp). */
int hyb_fn_create( hyb_ctx* ctx, hyb_mesh* mesh, int dtype, int min_level, int max_level, hyb_fn** out );
/* P2Function<T>(name, storage, minLevel, maxLevel) (p2functionspace/P2Function.hpp:35-429): quadratic
 * Lagrange DoFs (micro-vertices and micro-edge midpoints of level l).  Stored on the node set of level
 * l+1, so every hyb_fn_* / hyb_op_* / solver call takes the P2 level and packed uploads and downloads
 * use the vertex-DoF layout of level l+1 (hyb_layout_packed_size( mesh, l+1 ) values). */
int hyb_fn_create_p2( hyb_ctx* ctx, hyb_mesh* mesh, int dtype, int min_level, int max_level, hyb_fn** out );
/* A P2 function of level l in the reference's own memory layout (P2Function = VertexDoFFunction +
 * EdgeDoFFunction, p2functionspace/P2Function.hpp:35-60): first the vertex-DoF arrays of level l in
 * the packed order of hyb_layout_* (`vertex_part` values), then the edge-DoF array of every primitive
 * in the order vertices, edges, faces, cells (`edge_part` values; per-primitive sizes
 * edgeDoFMacro{Vertex,Edge,Face,Cell}FunctionMemorySize, edgedofspace/EdgeDoFFunction.cpp:1642-1690).
 * Inside a primitive's edge-DoF array the own DoFs come first in the reference's order
 * (edgedof::macroedge::index, macroface::index blocks X, XY, Y, macrocell::xIndex ... xyzIndex,
 * edgedofspace/EdgeDoFIndexing.hpp:361-366,579-594,922-980); the ghost layers that follow (and a
 * vertex's whole edge-DoF array) are communication buffers: download writes them as zero and upload
 * ignores them.  Upload then refreshes every copy of an owned DoF from its owner. */
int hyb_p2_layout_sizes( hyb_mesh* mesh, int level, int64_t* vertex_part, int64_t* edge_part );
int hyb_p2_fn_download_reference( hyb_fn* fn, int level, double* out );
int hyb_p2_fn_upload_reference( hyb_fn* fn, int level, const double* in );
int hyb_fn_destroy( hyb_fn* fn );
/* host <-> device in the packed layout; host values are doubles.  Upload refreshes every copy of
 * an owned DoF from its owner (communicate). */
int hyb_fn_upload( hyb_fn* fn, int level, const double* host_packed );
int hyb_fn_download( hyb_fn* fn, int level, double* host_packed );
/* the same transfers queued on the function's context stream without waiting (no counterpart in the
 * reference): the host buffer must stay valid (pinned memory for full bandwidth) until
 * hyb_ctx_synchronize; each function has its own staging, so transfers of functions on different
 * contexts overlap each other and kernels */
int hyb_fn_upload_async( hyb_fn* fn, int level, const double* host_packed );
int hyb_fn_download_async( hyb_fn* fn, int level, double* host_packed );
/* interpolate(constant, level, flag) (VertexDoFFunction.cpp:384) */
int hyb_fn_interpolate_const( hyb_fn* fn, double value, int level, uint32_t flag );
/* interpolate(std::function<real_t(const Point3D&)>, level, flag) (VertexDoFFunction.cpp:384-470) */
int hyb_fn_interpolate_callback( hyb_fn* fn, double ( *f )( const double* xyz, void* user ), void* user, int level,
                                 uint32_t flag );
/* assign(scalars, functions, level, flag): dst = sum_k scalars[k] * srcs[k], n <= 3 (VertexDoFFunction.cpp:1131) */
int hyb_fn_assign( hyb_fn* dst, int n, const double* scalars, hyb_fn* const* srcs, int level, uint32_t flag );
/* add(scalars, functions, level, flag): dst += sum_k scalars[k] * srcs[k] (VertexDoFFunction.cpp:1224) */
int hyb_fn_add( hyb_fn* dst, int n, const double* scalars, hyb_fn* const* srcs, int level, uint32_t flag );
/* multElementwise({a, b}, level, flag) (VertexDoFFunction.cpp:1487) */
int hyb_fn_mult_elementwise( hyb_fn* dst, hyb_fn* a, hyb_fn* b, int level, uint32_t flag );
/* invertElementwise(level, flag) (VertexDoFFunction.cpp:1566) */
int hyb_fn_invert_elementwise( hyb_fn* fn, int level, uint32_t flag );
/* dotGlobal(other, level, flag) (VertexDoFFunction.cpp:1710-1790); deterministic */
int hyb_fn_dot( hyb_fn* a, hyb_fn* b, int level, uint32_t flag, double* out );
/* Allocation-free hyb_fn_dot (no counterpart in the reference): the same deterministic kernels and
 * result, with the per-block partial sums in a fixed file-scope device array (65536 partials, 512 KiB)
 * instead of a buffer grown with cudaMalloc, for callers whose device memory is reserved up front by
 * their own allocator.  The array's address is resolved by the library's per-device set-up, which
 * the first operation of any kind on a device runs; before that this entry point returns HYB_EINVAL
 * rather than load anything.  The level's index tables must already be on the device (any earlier
 * operation on that level puts them there).  Levels needing more partials return HYB_EINVAL.  The
 * array is shared per device: overlapping calls race and must be serialised by the caller. */
int hyb_fn_dot_noalloc( hyb_fn* a, hyb_fn* b, int level, uint32_t flag, double* out );
/* copyFrom between value types (VertexDoFFunction.hpp:150-151) */
int hyb_fn_copy_from( hyb_fn* dst, hyb_fn* src, int level );
/* swap(other, level) */
int hyb_fn_swap( hyb_fn* a, hyb_fn* b, int level );
/* device pointer and slot count of one level (padded device layout) */
int hyb_fn_device_ptr( hyb_fn* fn, int level, void** ptr, int64_t* nslots );
/* order (1: P1Function, 2: P2Function), value type and level range of a function (any may be NULL) */
int hyb_fn_info( const hyb_fn* fn, int* order, int* dtype, int* min_level, int* max_level );

/* ---------------------------------------------------------------- operators
 * Operator<Src,Dst>::apply(src, dst, level, flag, updateType) (operators/Operator.hpp:74-81),
 * P1Operator::apply (p1functionspace/P1Operator.hpp:192-320). */
int hyb_op_create( hyb_ctx* ctx, hyb_mesh* mesh, int kind, int min_level, int max_level, hyb_op** out );
/* elementwise -div(k grad u) with the coefficient k (NULL: k = 1) and optional blending; every micro-cell's
 * element matrix comes from 5-point degree-3 quadrature (p1_div_k_grad_blending_q3); smoothers use the
 * assembled inverse diagonal (P1ElementwiseOperator::computeInverseDiagonalOperatorValues) */
int hyb_op_create_divkgrad( hyb_ctx* ctx, hyb_mesh* mesh, int min_level, int max_level, const hyb_coeff* k, int blending,
                            hyb_op** out );
/* P1ElementwiseOperator::computeAndStoreLocalElementMatrices (elementwiseoperators/P1ElementwiseOperator.hpp:138):
 * from now on every level's element matrices are computed once (when the level is first used) and read back
 * by every later apply instead of being recomputed; 80 bytes per micro-cell per level in FP64 (40 in FP32).
 * Call it before capturing any graph that applies the operator. */
/* P2ElementwiseBlendingDivKGradOperator (elementwiseoperators/P2ElementwiseOperator.hpp:475) with the form
 * p2_div_k_grad_blending_q4 (11-point degree-4 quadrature) on P2 functions (hyb_fn_create_p2); with k = NULL
 * and no blending it is the P2 Laplacian (the matrix of P2ConstantLaplaceOperator).  hyb_restrict and
 * hyb_prolongate on P2 functions are the quadratic transfers (P2toP2QuadraticRestriction /
 * P2toP2QuadraticProlongation), used by the multigrid solver for P2 operators. */
int hyb_op_create_p2_divkgrad( hyb_ctx* ctx, hyb_mesh* mesh, int min_level, int max_level, const hyb_coeff* k, int blending,
                               hyb_op** out );
/* The hyteg-operators form of the same operator, operatorgeneration::P2ElementwiseDivKGrad and
 * P2ElementwiseDivKGradIcosahedralShellMap (generated code in the hyteg_operators submodule, absent from the
 * reference tree; call sites tests/hyteg/convergence/ElementwiseDivKGradCGConvergenceTest.cpp:38-39,85-92):
 * the coefficient is a P2 function k_h and enters each quadrature point as sum_i k_h(node_i) phi_i(point)
 * instead of its closed form.  _nodal interpolates the closed form k at the (blended) nodes of every level,
 * as kFunction.interpolate(k, level) does there; _fn copies a caller's FP64 P2 function (levels
 * min_level..max_level) at creation. */
int hyb_op_create_p2_divkgrad_nodal( hyb_ctx* ctx, hyb_mesh* mesh, int min_level, int max_level, const hyb_coeff* k, int blending,
                                     hyb_op** out );
int hyb_op_create_p2_divkgrad_fn( hyb_ctx* ctx, hyb_mesh* mesh, int min_level, int max_level, hyb_fn* k, int blending, hyb_op** out );
int hyb_op_store_element_matrices( hyb_op* op );
int hyb_op_destroy( hyb_op* op );
int hyb_op_apply( hyb_op* op, hyb_fn* src, hyb_fn* dst, int level, uint32_t flag, int update );
/* WeightedJacobiSmoothable::smooth_jac(dst, rhs, src, relax, level, flag) (solvers/Smoothables.hpp:33-40,
 * P1Operator.hpp:429-447): dst = src + relax * D^-1 (rhs - A src) on flagged DoFs */
/* P1Operator::smooth_sor / smooth_gs / smooth_sor_backwards (p1functionspace/P1Operator.hpp:322-420)
 * for constant-stencil operators: dst <- dst + relax D^-1 (rhs - A dst) point by point on the flagged
 * DoFs, in place.  The sweep keeps the reference's primitive order (macro-vertices, -edges, -faces,
 * -cells; reversed when backwards) with colour sets inside each class (edge DoFs by index parity,
 * face DoFs by (i + 2j) mod 3, cell interiors by (x + 2y + 3z) mod 4) instead of the lexicographic
 * order inside a primitive, so iterates differ from the reference's in order, not in kind. */
int hyb_op_smooth_sor( hyb_op* op, hyb_fn* dst, hyb_fn* rhs, double relax, int level, uint32_t flag, int backwards );
int hyb_op_smooth_jac( hyb_op* op, hyb_fn* dst, hyb_fn* rhs, hyb_fn* src, double relax, int level, uint32_t flag );
/* OperatorWithInverseDiagonal::getInverseDiagonalValues (solvers/Smoothables.hpp:109-119) written into out */
int hyb_op_inverse_diagonal( hyb_op* op, hyb_fn* out, int level, uint32_t flag );
/* stencil of cell `cell`, position class cls (0 interior, 1-4 faces, 5-10 edges, 11-14 vertices), 15 weights:
 * centre, then directions W E S N B T NW SE TW BE TS BN TSE BNW (P1Elements.hpp:466-529) */
int hyb_op_stencil( hyb_op* op, int level, int cell, int cls, double* out15 );

/* ---------------------------------------------------------------- grid transfer
 * P1toP1LinearRestriction::restrict (gridtransferoperators/P1toP1LinearRestriction.cpp:169-346) and
 * P1toP1LinearProlongation::prolongate / prolongateAndAdd (P1toP1LinearProlongation.hpp:35-55). */
int hyb_restrict( hyb_fn* fn, int source_level, uint32_t flag );
int hyb_prolongate( hyb_fn* fn, int source_level, uint32_t flag, int update );

/* ---------------------------------------------------------------- solvers */
typedef struct hyb_gmg_params
{
   int    min_level, max_level;
   int    pre_smooth, post_smooth, smooth_increment; /* GeometricMultigridSolver.hpp:61-75 */
   int    cycle;                                     /* HYB_VCYCLE | HYB_WCYCLE */
   int    smoother;                                  /* HYB_SMOOTHER_* */
   double jacobi_relax;                              /* WeightedJacobiSmoother relax; the SOR smoother's relax */
   int    cheb_order;                                /* ChebyshevSmoother::setupCoefficients order */
   double cheb_upper_factor, cheb_lower_factor;      /* 1.2, 0.3 */
   int    cheb_power_iterations;                     /* chebyshev::estimateRadius iterations per level */
   int    coarse_max_iter;                           /* CGSolver(maxIter, relTol, absTol), CGSolver.hpp:44-75 */
   double coarse_rtol, coarse_atol;
   int    use_graph;                                 /* capture each cycle in a CUDA graph */
   int    coarse_fp64;                               /* FP32/FP16 hierarchies: coarse-grid CG in FP64 */
} hyb_gmg_params;

int hyb_gmg_params_default( hyb_gmg_params* p );
/* GeometricMultigridSolver (solvers/GeometricMultigridSolver.hpp:61-162) with its smoother and a CG
 * coarse solver on the device.  For Chebyshev smoothing the spectral radius of D^-1 A is estimated per
 * level by power iteration (chebyshev::estimateRadius, ChebyshevSmoother.hpp:656) from a seeded
 * start vector unless set explicitly. */
int hyb_gmg_create( hyb_ctx* ctx, hyb_op* op, const hyb_gmg_params* params, hyb_gmg** out );
int hyb_gmg_destroy( hyb_gmg* gmg );
/* per-level spectral radii (max_level-min_level+1 values); recomputes Chebyshev coefficients */
int hyb_gmg_set_radii( hyb_gmg* gmg, const double* radii );
int hyb_gmg_get_radii( hyb_gmg* gmg, double* radii );
/* Solver::solve(A, x, b, level) (solvers/Solver.hpp:31-35): one multigrid cycle */
int hyb_gmg_solve( hyb_gmg* gmg, hyb_fn* x, hyb_fn* b, int level );
/* the solver's smoother alone on one level above the coarsest: `iterations` applications of
 * ChebyshevSmoother::solve (solvers/ChebyshevSmoother.hpp:112-240), WeightedJacobiSmoother::solve
 * (WeightedJacobiSmoother.hpp:46-66) or the Gauss-Seidel / SOR smoother, with the solver's
 * coefficients for that level */
int hyb_gmg_smooth( hyb_gmg* gmg, hyb_fn* x, hyb_fn* b, int level, int iterations );
/* up to max_cycles cycles until ||r||/||r0|| < rtol (discrete L2 over non-Dirichlet DoFs);
 * res_history receives ||r_0|| .. ||r_k|| (max_cycles+1 entries) */
int hyb_gmg_solve_cycles( hyb_gmg* gmg, hyb_fn* x, hyb_fn* b, int level, int max_cycles, double rtol, double* res_history,
                          int* cycles_done );
/* chebyshev::estimateRadius (ChebyshevSmoother.hpp:656-676): power iteration on D^-1 A, flag All */
int hyb_estimate_radius( hyb_op* op, hyb_fn* x, hyb_fn* tmp, int level, int iterations, double* radius );
/* ChebyshevSmoother::setupCoefficientsInternal (ChebyshevSmoother.hpp:329-555) */
int hyb_chebyshev_coefficients( int order, double lower, double upper, double* out );
/* CGSolver::solve (solvers/CGSolver.hpp:94-206), identity preconditioner, flag Inner|Neumann|Freeslip */
int hyb_cg_solve( hyb_op* op, hyb_fn* x, hyb_fn* b, int level, int max_iter, double rtol, double atol, int* iterations );
/* Mixed-precision iterative refinement (defect correction) after
 * tests/hyteg/mixedPrecision/mixedPrecisionIterativeRefinement.cpp:163-173: x and b are FP64; each outer
 * step forms r = b - A x in FP64, scales r to unit RMS and stores it in the value type of `inner` (FP32 or
 * FP16, fixed by `inner_dtype`), runs `inner_cycles` multigrid cycles of `inner` from a zero guess (coarse
 * solve in FP64) and adds the rescaled correction to x in FP64.  Stops when ||r||/||r_0|| < rtol or after
 * max_outer steps; res_history receives ||r_0|| .. ||r_k|| (max_outer+1 entries). */
int hyb_mixed_solve( hyb_gmg* inner, int inner_dtype, hyb_op* op, hyb_fn* x, hyb_fn* b, int level, int inner_cycles,
                     int max_outer, double rtol, double* res_history, int* outer_iters );
/* fill every DoF of one level with seeded uniform values in [-1, 1] (device-side, reproducible) */
int hyb_fn_fill_random( hyb_fn* fn, int level, uint64_t seed );
/* discrete L2 norm of b - A x over the flagged DoFs */
int hyb_residual_norm( hyb_op* op, hyb_fn* x, hyb_fn* b, hyb_fn* tmp, int level, uint32_t flag, double* out );

/* ---------------------------------------------------------------- serving
 * Continuous admission of solve requests (no counterpart in the reference, which solves one problem per
 * run): requests wait in a FIFO queue and are admitted into resident multigrid "slots" keyed by (mesh,
 * operator, coefficient, blending, level, precision) as slots and the HBM budget allow; idle slots are
 * reused (no setup, the captured graph is replayed) or evicted least-recently-used; every slot runs on
 * its own stream, so solves overlap on the device.  Chebyshev(3) V(pre,post) cycles with a CG coarse
 * solve; mixed requests run FP64 defect correction around cycles in `inner_dtype`. */
typedef struct hyb_serve hyb_serve;
typedef struct hyb_serve_params
{
   int    max_slots;
   double hbm_budget_bytes; /* 0: 80 % of the free device memory at creation */
   int    inner_dtype;      /* HYB_F32 or HYB_F16 for mixed requests */
   int    pre_smooth, post_smooth;
   int    power_iterations; /* spectral-radius estimate per level when a slot is created */
   int    batch_width;      /* > 1: FP64 P1 requests of one key share batch slots of this many solves,
                               whose multigrid runs on batch_width disjoint copies of the mesh, so that
                               every kernel launch of a cycle serves all of them (P2 and mixed requests
                               keep one-solve slots); 1: one solve per slot */
} hyb_serve_params;
typedef struct hyb_request
{
   hyb_mesh*     mesh;
   int           op_kind;  /* HYB_P1_CONST_LAPLACE, HYB_P1_ELEM_DIVKGRAD, HYB_P2_ELEM_DIVKGRAD or HYB_P2_CONST_LAPLACE (P2:
                              level = P2 level, rhs / x_out in the P2 packed layout, FP64 only) */
   hyb_coeff     coeff;    /* HYB_P1_ELEM_DIVKGRAD only */
   int           blending; /* HYB_P1_ELEM_DIVKGRAD only */
   int           level;
   const double* rhs;      /* packed level layout, or NULL for seeded uniform values */
   uint64_t      seed;
   double        rtol;     /* stop when ||r||/||r_0|| < rtol */
   int           max_cycles;
   int           mixed;        /* 0 plain FP64 cycles, 1 mixed-precision defect correction */
   double        arrival_time; /* seconds on the server clock (hyb_serve_now); < 0: now */
   double*       x_out;        /* packed solution on completion, or NULL */
} hyb_request;
int    hyb_serve_params_default( hyb_serve_params* p );
int    hyb_serve_create( hyb_ctx* ctx, const hyb_serve_params* params, hyb_serve** out );
int    hyb_serve_destroy( hyb_serve* s );
double hyb_serve_now( hyb_serve* s );
/* HYB_ENOMEM if the request could never fit the budget */
int hyb_serve_submit( hyb_serve* s, const hyb_request* r, int64_t* id );
/* one scheduler pass: retire finished solves, launch next cycles, admit queued requests */
int hyb_serve_step( hyb_serve* s, int* running, int* queued );
/* state: 0 queued, 1 running, 2 converged, 3 stopped without converging */
int hyb_serve_status( hyb_serve* s, int64_t id, int* state, double* t_arrival, double* t_admit, double* t_done, int* cycles,
                      double* rel_res );
const char* hyb_serve_last_error( void );

/* ---------------------------------------------------------------------------------------------
 * P2-P1 Taylor-Hood Stokes (P2P1ElementwiseBlendingStokesOperator, elementwiseoperators/
 * P2P1ElementwiseBlendingStokesOperator.hpp:36-122, with the velocity block -div(eta grad) of each
 * component, UzawaSmoother solvers/UzawaSmoother.hpp:321-441).  Velocity: three P2 functions
 * (hyb_fn_create_p2); pressure: one P1 function of the same level whose every DoF is free (the
 * reference's all-inner pressure boundary condition), so pressure calls use HYB_ALL.
 * --------------------------------------------------------------------------------------------- */
/* the coupling blocks on P2 level l / P1 level l: div (P2ToP1ElementwiseBlendingDiv{x,y,z}Operator,
 * forms p2_to_p1_div_{0,1,2}_blending_q2) and divT (P1ToP2ElementwiseBlendingDivT{x,y,z}Operator,
 * forms p1_to_p2_divt_{0,1,2}_blending_q2, the transpose) */
int hyb_op_create_p2p1_div( hyb_ctx* ctx, hyb_mesh* mesh, int min_level, int max_level, int blending, hyb_op** out );
/* p (update)= div u (u: three P2 functions) */
int hyb_p2p1_div_apply( hyb_op* div, hyb_fn* const* u3, hyb_fn* p, int level, uint32_t flag, int update );
/* u_k (update)= divT_k p */
int hyb_p1p2_divt_apply( hyb_op* div, hyb_fn* p, hyb_fn* const* u3, int level, uint32_t flag, int update );
/* P1PSPGOperator on the affine macro geometry; hyb_op_inverse_diagonal gives P1PSPGInvDiagOperator's values */
int hyb_op_create_p1_pspg( hyb_ctx* ctx, hyb_mesh* mesh, int min_level, int max_level, hyb_op** out );

/* P2ElementwiseBlendingFullViscousOperator (elementwiseoperators/P2ElementwiseBlendingFullViscousOperator.hpp:
 * 34-68): the velocity block 2 mu eps(u) : eps(v) - (2/3) mu div u div v coupling the three P2
 * components, block (i, j) the form p2_full_stokesvar_{i}_{j}_blending_q3 (Yu's 5-point rule, mu at
 * the blended point); applied matrix-free.  VectorToVectorOperator::apply (mixed_operator/
 * VectorToVectorOperator.hpp) maps to hyb_p2_full_viscous_apply: dst_i (update)= sum_j A_ij src_j on
 * the flagged owned DoFs.  hyb_p2_full_viscous_inverse_diagonal writes 1/diag(A_ii) into out_i
 * (OperatorWithInverseDiagonal::computeInverseDiagonalOperatorValues / getInverseDiagonalValues). */
int hyb_op_create_p2_full_viscous( hyb_ctx* ctx, hyb_mesh* mesh, int min_level, int max_level, const hyb_coeff* viscosity,
                                   int blending, hyb_op** out );
int hyb_p2_full_viscous_apply( hyb_op* op, hyb_fn* const* src3, hyb_fn* const* dst3, int level, uint32_t flag, int update );
int hyb_p2_full_viscous_inverse_diagonal( hyb_op* op, hyb_fn* const* out3, int level );

typedef struct hyb_stokes hyb_stokes;
typedef struct hyb_stokes_params
{
   int    min_level, max_level; /* P2 / P1 levels of the hierarchy */
   int    pre_smooth, post_smooth;
   int    velocity_sweeps;  /* velocity smoother applications per Uzawa step */
   int    cheb_order;       /* Chebyshev order of the velocity smoother (ChebyshevSmoother) */
   int    power_iterations; /* spectral-radius estimate of D^-1 A per level */
   double omega;            /* Uzawa relaxation parameter (UzawaSmoother::setRelaxationParameter) */
   int    coarse_sweeps;    /* Uzawa steps on the coarsest level (the coarse solve; default 30) */
   int    velocity_block;   /* 0: -div(eta grad) per component (block Laplace); 1: the full viscous block
                               P2ElementwiseBlendingFullViscousOperator, Chebyshev on the coupled block */
   int    pressure_scaling; /* scaling S^-1 of the pressure update p += omega S^-1 (b_p - div u):
                               0: the inverted PSPG diagonal (P2P1TaylorHoodStokesOperator's pspg_inv_diag_);
                               1: the inverse lumped pressure mass matrix weighted by 1/eta (blended), the
                               P1LumpedInvMassOperator pattern of tests/hyteg/convergence/
                               P2P1Stokes3DUzawaConvergenceTest.cpp:125-139 with the viscosity that the
                               Schur complement of a variable-viscosity velocity block carries */
} hyb_stokes_params;
int hyb_stokes_params_default( hyb_stokes_params* p );
/* GeometricMultigridSolver< P2P1ElementwiseBlendingStokesOperator > with UzawaSmoother; viscosity:
 * the coefficient of the velocity block (e.g. HYB_COEFF_RADIAL_EXP), NULL for eta = 1 */
int hyb_stokes_create( hyb_ctx* ctx, hyb_mesh* mesh, const hyb_coeff* viscosity, int blending, const hyb_stokes_params* p,
                       hyb_stokes** out );
int hyb_stokes_destroy( hyb_stokes* s );
/* fixes the velocity smoother's spectral radii (max_level - min_level + 1 values, P2 levels) */
int hyb_stokes_set_velocity_radii( hyb_stokes* s, const double* radii );
/* UzawaSmoother::setRelaxationParameter (solvers/UzawaSmoother.hpp): the omega of every later Uzawa step */
int hyb_stokes_set_omega( hyb_stokes* s, double omega );
/* estimateUzawaRelaxationParameter (solvers/UzawaSmoother.hpp:40-97) with
 * P2P1UzawaDampingFactorEstimationOperator (mixed_operator/P2P1UzawaDampingFactorEstimationOperator.hpp):
 * power iteration (iterations steps from a seeded random pressure) for the spectral radius rho of
 * E = |S|^-1 B A~^-1 B^T on one level, A~^-1 being velocity_sweeps applications of the solver's own velocity
 * smoother from zero and |S|^-1 the magnitude of its pressure scaling.  The reference passes the radius
 * of its estimator (lumped mass in place of S) to setRelaxationParameter; for the scaling of this solver
 * omega = 1/rho keeps the Uzawa pressure iteration I - omega |S|^-1 B A~^-1 B^T a contraction. */
int hyb_stokes_estimate_relaxation( hyb_stokes* s, int level, int iterations, int velocity_sweeps, double* rho );
/* P2P1ElementwiseBlendingStokesOperator::apply: du = A u + divT p (velocity flag Inner), dp = div u (all) */
int hyb_stokes_apply( hyb_stokes* s, hyb_fn* const* u3, hyb_fn* p, hyb_fn* const* du3, hyb_fn* dp, int level );
/* one UzawaSmoother::solve step */
int hyb_stokes_uzawa_smooth( hyb_stokes* s, hyb_fn* const* u3, hyb_fn* p, hyb_fn* const* bu3, hyb_fn* bp, int level );
/* sqrt(|b_u - A u - divT p|^2 + |b_p - div u|^2) over the velocity's inner DoFs and all pressure DoFs */
int hyb_stokes_residual_norm( hyb_stokes* s, hyb_fn* const* u3, hyb_fn* p, hyb_fn* const* bu3, hyb_fn* bp, int level, double* out );
/* V-cycles (Uzawa smoothing, quadratic / linear transfers, coarse Uzawa sweeps) until the residual
 * norm drops by rtol or max_cycles; history[0..cycles] the residual norms */
int hyb_stokes_solve( hyb_stokes* s, hyb_fn* const* u3, hyb_fn* p, hyb_fn* const* bu3, hyb_fn* bp, int level, int max_cycles, double rtol,
                      double* history, int* cycles_done );
/* mixed-precision defect correction (mixedPrecisionIterativeRefinement): FP64 residual of `outer`,
 * one V-cycle of `inner` (a second solver of the same mesh and levels) in inner_dtype (HYB_F32; FP16
 * is refused: the inverted PSPG diagonal, of order h^-3, leaves its range) on the scaled residual,
 * FP64 update; u3, p, bu3, bp hold FP64 values */
int hyb_stokes_mixed_solve( hyb_stokes* outer, hyb_stokes* inner, int inner_dtype, hyb_fn* const* u3, hyb_fn* p, hyb_fn* const* bu3,
                            hyb_fn* bp, int level, int max_outer, double rtol, double* history, int* iterations );

/* ---------------------------------------------------------------- data export and checkpoints
 * VTKOutput (dataexport/VTKOutput/VTKOutput.hpp:44-139; VTKOutput( dir, filename, storage,
 * writeFrequency ), add( function ), write( level, timestep ), setParameter( "vtkDataFormat",
 * "ASCII" | "BINARY" )).  write() writes, when timestep % write_frequency == 0, one file per DoF type
 * with added functions: <dir>/<filename>_VertexDoF_level<L>_ts<T>.vtu for P1 functions and
 * <dir>/<filename>_P2_level<L>_ts<T>.vtu for P2 functions (an XML UnstructuredGrid piece: per macro-cell
 * the micro-vertices of level L, for P2 of level L+1, at their positions under the storage's geometry
 * map, the micro-tetrahedra of level L, for P2 as ten-node quadratic tetrahedra, and each function as
 * point data).  Functions are downloaded at write time; they must stay alive while added. */
typedef struct hyb_vtk hyb_vtk;
int hyb_vtk_create( hyb_mesh* mesh, const char* dir, const char* filename, int write_frequency, hyb_vtk** out );
int hyb_vtk_destroy( hyb_vtk* w );
/* the geometry map of the point coordinates (the storage's blending map in the reference):
 * HYB_BLEND_NONE (default) or HYB_BLEND_SHELL */
int hyb_vtk_set_blending( hyb_vtk* w, int blending );
int hyb_vtk_set_parameter( hyb_vtk* w, const char* key, const char* value );
int hyb_vtk_add( hyb_vtk* w, hyb_fn* fn, const char* name );
int hyb_vtk_remove( hyb_vtk* w, hyb_fn* fn );
int hyb_vtk_write( hyb_vtk* w, int level, int timestep );
/* the same file from host data: nfields packed vectors (hyb_fn_download layout) of one order at
 * `level`, written to `path`; dtypes name each field's value type (HYB_F64 -> Float64, else Float32) */
int hyb_vtk_write_packed( hyb_mesh* mesh, const char* path, int level, int order, int blending, int binary, int nfields,
                          const char* const* names, const int* dtypes, const double* const* packed );

/* Checkpoints (checkpointrestore/CheckpointExporter.hpp:26-60: registerFunction( function, minLevel,
 * maxLevel ), storeCheckpoint( filePath, fileName ); ADIOS2/AdiosCheckpointImporter.hpp:97-170:
 * getFunctionDetails(), restoreFunction( function, minLevel, maxLevel )).  ADIOS2 is not used: the
 * checkpoint is <dir>/<filename>.hybckpt in this library's own binary format (the mesh's primitive
 * counts and a hash of its coordinates and cells; per function its name, kind, value type, level range
 * and the packed vector of every level).  Restoring refuses a different mesh, kind or value type and a
 * level range the checkpoint does not hold, as the reference's importer does. */
int hyb_checkpoint_store( const char* dir, const char* filename, int nfn, hyb_fn* const* fns, const char* const* names,
                          const int* min_levels, const int* max_levels );
int hyb_checkpoint_function_count( const char* dir, const char* filename, int* count );
int hyb_checkpoint_function_info( const char* dir, const char* filename, int index, char* name, int name_cap, char* kind, int kind_cap,
                                  char* value_type, int vtype_cap, int* min_level, int* max_level );
int hyb_checkpoint_restore( const char* dir, const char* filename, hyb_fn* fn, const char* name, int min_level, int max_level );

#ifdef __cplusplus
}
#endif

#endif /* HYTEG_B200_H */
