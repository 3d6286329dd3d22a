// Internal declarations of the hyteg_b200 runtime (host C++ and CUDA).
//
// Data model (per function, per level): one device buffer holding every macro-primitive's
// vertex-DoF array in HyTeG's own per-primitive layout (VertexDoFMemory.hpp:39-60 of the
// reference), packed in the order vertices, edges, faces, cells, each primitive array starting
// on a 32-element boundary.  Owned DoFs are the cell interiors, face interiors, edge interiors
// and the macro-vertices.  Cell arrays also hold copies of the face/edge/vertex DoFs on their
// boundary; every kernel that writes a lower-dimensional owner also writes those copies
// ("write-through"), so cell arrays are always consistent and no separate ghost exchange is
// needed before a stencil sweep.
#pragma once

#include <cuda_runtime.h>
#include <cuda_fp16.h>

#include <array>
#include <atomic>
#include <cstdint>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

namespace hyb {

// DoFType bits (types/types.hpp:29-43 of the reference)
enum : uint32_t { kInner = 1, kDirichlet = 2, kNeumann = 4, kFreeslip = 8, kAll = 15 };

enum DType : int { F64 = 0, F32 = 1, F16 = 2 };

inline size_t dtype_size(int dt) { return dt == F64 ? 8 : dt == F32 ? 4 : 2; }

// --------------------------------------------------------------------------------------------
// index math (MacroCellIndexing.hpp:39-52, MacroFaceIndexing.hpp:39-50)
// --------------------------------------------------------------------------------------------
__host__ __device__ inline int64_t tet_size(int64_t w) { return ((w + 2) * (w + 1) * w) / 6; }
__host__ __device__ inline int64_t tri_size(int64_t w) { return ((w + 1) * w) / 2; }

// cell-local (x, y, z) with x+y+z <= n  ->  offset inside the cell array (width n+1)
__host__ __device__ inline int64_t cidx(int n, int x, int y, int z)
{
   const int64_t w  = n + 1;
   const int64_t wz = w - z;
   return tet_size(w) - tet_size(wz) + (int64_t) y * (wz + 1) - ((int64_t) y * (y + 1)) / 2 + x;
}

// face-local (i, j) with i+j <= n  ->  offset inside the face array (width n+1)
__host__ __device__ inline int64_t fidx(int n, int i, int j)
{
   const int64_t w = n + 1;
   return (int64_t) j * (w + 1) - ((int64_t) j * (j + 1)) / 2 + i;
}

// The 15 stencil directions: centre first, then the 14 neighbours of the 3D P1 stencil
// (VertexDoFIndexing.hpp:289-323).
constexpr int kNumDirs = 15;
extern const int kDirs[kNumDirs][3];

// Position classes of a micro-vertex inside a macro-cell: 0 interior, 1..4 cell faces 0..3,
// 5..10 cell edges 0..5, 11..14 cell vertices 0..3.  Cell-local numbering follows
// SetupPrimitiveStorage.cpp:305-315 (faces 012, 013, 023, 123; edges 01, 02, 12, 03, 13, 23).
constexpr int kNumClasses = 15;
// cell faces touched by each position class (bit 0: z = 0, bit 1: y = 0, bit 2: x = 0, bit 3:
// x + y + z = n): interior, faces 012 013 023 123, edges 01 02 12 03 13 23, vertices 0..3
constexpr int kClassFaces[kNumClasses] = { 0, 1, 2, 4, 8, 3, 5, 9, 6, 10, 12, 7, 11, 13, 14 };
// P2 constant-stencil tables: entries of the eight parity classes' stencils (230 in all; every
// class starts on a multiple of four entries, so weights load as 16-byte vectors), then the eight
// interior inverse diagonals; one such block per position class and macro-cell
constexpr int kP2cEntries    = 256;
constexpr int kP2cInterior   = kP2cEntries + 8;
constexpr int kP2cCellStride = kP2cInterior + ( kNumClasses - 1 ) * kP2cEntries;
// bit mask of directions that stay inside the cell for a point of each class
extern const uint16_t kClassDirMask[kNumClasses];
int class_of_point(int n, int x, int y, int z);  // host version

// A face-interior boundary task between two macro-cells, resolved once per level for the boundary
// stencil kernel: the owner slot, the slots of the owner's copies in the two cell arrays (the centres
// of the cells' class stencils), their rows and slices, cells and position classes, the face's
// boundary-primitive index and type.  cell0 < 0 marks any other task.
struct FaceRec {
   int64_t owner;
   int64_t c0, c1;
   int     b;
   int     cell0, cell1;
   int16_t y0, z0, y1, z1;
   int8_t  cls0, cls1;
   uint8_t bc;
   uint8_t pad;
};
static_assert( sizeof( FaceRec ) == 48, "face record layout" );

struct Incidence {
   int   cell;
   int   cls;
   int8_t o[3];   // origin = n * o (cell-local corner of the primitive's vertex 0)
   int8_t e1[3];  // cell-local step per primitive-local i
   int8_t e2[3];  // cell-local step per primitive-local j
   int8_t pad[3];
};

// --------------------------------------------------------------------------------------------
// macro mesh / primitive storage (host)
// --------------------------------------------------------------------------------------------
struct Topology {
   int nV = 0, nE = 0, nF = 0, nC = 0;
   std::vector< std::array< double, 3 > > vx;  // coordinates per vertex (id order)
   std::vector< std::array< int, 2 > >    ev;  // edge vertices (sorted)
   std::vector< std::array< int, 3 > >    fv;  // face vertices (sorted)
   std::vector< std::array< int, 4 > >    cv;  // cell vertices (mesh order)
   std::vector< std::array< int, 6 > >    ce;  // cell local edges
   std::vector< std::array< int, 4 > >    cf;  // cell local faces
   std::vector< std::vector< int > >      v_edges, v_faces, v_cells, e_faces, e_cells, f_cells;
   std::vector< int >                     flag_v, flag_e, flag_f, flag_c;  // mesh boundary flags
   std::map< int, uint32_t >              bc_of_flag{ { 0, kInner }, { 1, kDirichlet }, { 2, kNeumann }, { 3, kFreeslip } };
   // optional blending (0 = affine, 1 = icosahedral shell)
   int    blending = 0;
   double shell_rmin = 0, shell_rmax = 0;

   uint32_t bc(int flag) const
   {
      auto it = bc_of_flag.find( flag );
      return it == bc_of_flag.end() ? kInner : it->second;
   }
   void build( const std::vector< std::array< double, 3 > >& coords, const std::vector< std::array< int, 4 > >& tets );
   void set_boundary_flags_on_boundary( int onBoundary, int inner );
};

// per-level host + device tables of the P1 layout
// units of the cell-interior sweep (k_cell_sweep): kSwR rows by kSwTX x-points (two per lane) over a
// range of slices; a half-width unit (flag kSwUnitHalf on x0) has rows that all end within 32 points
// and runs one point per lane.  Each warp of a launch owns a list of units; a launch has kSwWarps
// warps per block and BPS = 2, 3 or 4 blocks per SM (by value type and operation), one list set per
// BPS.
constexpr int kSwR         = 4;
constexpr int kSwTX        = 64;  // 32 or 64
constexpr int kSwWarps     = 4;
constexpr int kSwUnitHalf  = 1 << 30;
constexpr int kSwUnitXMask = kSwUnitHalf - 1;
constexpr int kSwLists     = 3;  // BPS 2, 3, 4
// tile rows of the rolled-register sweep (k_cell_zstream): 64 x-points (two per lane) by kZTileY rows
constexpr int kZTileY = 8;

struct P1Level {
   int     L = 0, n = 0;
   int64_t size = 0;         // slots incl. padding
   int64_t packed_size = 0;  // slots without padding (HyTeG export)
   std::vector< int64_t > off;         // slot offset of each primitive (v, e, f, c order)
   std::vector< int64_t > packed_off;  // same without padding
   std::vector< int64_t > psize;       // HyTeG array size of each primitive
   // boundary primitives (vertices, edges, faces) in one index space: b = v | nV+e | nV+nE+f
   int                          nB = 0;
   std::vector< int >           inc_begin;  // nB+1
   std::vector< Incidence >     inc;
   std::vector< std::array< int, 4 > > tasks;  // {b, i, j, 0}: owned DoFs of boundary primitives
   std::vector< std::array< int, 2 > > rows;   // (y, z) of cell interior rows
   // y-marching work items of the cell stencil sweep: (z, x0, y_first, y_last); a warp covers
   // x0..x0+31 of slice z and marches over rows y_first..y_last
   std::vector< std::array< int, 4 > > march;
   // rolled-register sweep: units {x0 (| kSwUnitHalf), y0, z_first, z_last} of macro-cell zcell[i];
   // block k runs units zbegin[k]..zbegin[k+1]-1
   std::vector< std::array< int, 4 > > zunits;
   std::vector< int >                  zcell;
   std::vector< int >                  zbegin;
   // cell-interior sweep: units {x0 (| kSwUnitHalf), y0, z_first, z_last} of macro-cell swcell[b][i];
   // warp w of a launch with b + 2 blocks per SM runs units swbegin[b][w]..swbegin[b][w+1]-1
   std::vector< std::array< int, 4 > > swunits[kSwLists];
   std::vector< int >                  swcell[kSwLists];
   std::vector< int >                  swbegin[kSwLists];
   int64_t n_owned_cell = 0;
   // device copies
   int64_t*   d_off       = nullptr;  // all primitives
   int64_t*   d_poff      = nullptr;  // packed offsets of all primitives and the packed size (nP + 1)
   int*       d_inc_begin = nullptr;
   Incidence* d_inc       = nullptr;
   int4*      d_tasks     = nullptr;
   int4*      d_btasks    = nullptr;  // tasks grouped by boundary type (Inner, Dirichlet, Neumann, Freeslip)
   FaceRec*   d_frec      = nullptr;  // per grouped task: its two-cell face record, if it is one
   int        bcount[4]   = {};
   int2*      d_rows      = nullptr;
   int4*      d_march     = nullptr;
   int4*      d_zunits            = nullptr;
   int*       d_zcell             = nullptr;
   int*       d_zbegin            = nullptr;
   int4*      d_swunits[kSwLists]  = {};
   int*       d_swcell[kSwLists]   = {};
   int*       d_swbegin[kSwLists]  = {};
   uint8_t*   d_bc        = nullptr;  // bc type per primitive (v, e, f, c order)
   int8_t*    d_bkind     = nullptr;  // 0 vertex, 1 edge, 2 face per boundary primitive
   float*     d_ncell_cls = nullptr;  // per cell, per class: number of macro-cells around the sub-primitive
};

struct Context;

struct Mesh {
   Context*                                  ctx = nullptr;
   void*                                     handle    = nullptr;  // owning C-ABI handle (reference count)
   void*                                     owner_ctx = nullptr;  // C-ABI context handle the mesh holds
   Topology                                  topo;
   std::map< int, std::unique_ptr< P1Level > > levels;
   P1Level&                                  level( int L );
   ~Mesh();
};

struct Function {
   Mesh*                mesh  = nullptr;
   int                  dtype = F64;
   int                  lshift = 0;  // 1 for P2: user level L is stored on the nodes of storage level L+1
   int                  minL = 0, maxL = 0;
   std::vector< void* > data;  // device buffer per level (index L - minL)
   void*                ptr( int L ) const { return data.at( L - minL ); }
   size_t               bytes( int L ) const;
};

// constant-stencil operator (P1ConstantLaplaceOperator and friends)
// P2 constant-stencil operator, one storage level: per macro-cell and position class the stencil
// weights of every parity class of the level-(l+1) node grid (the interior block is followed by the
// eight interior inverse diagonals), FP64 and an FP32 copy
struct P2cLevel {
   std::vector< double > W;      // [nC][kP2cCellStride]
   std::vector< int4 >   tasks;  // boundary tasks grouped by boundary type, then by primitive and parity class
   double* d_W     = nullptr;
   float*  d_Wf    = nullptr;
   int4*   d_tasks = nullptr;
};

struct OpLevel {
   std::vector< double > W;      // [nC][15 classes][15 dirs]
   std::vector< double > invd_b; // per boundary primitive
   std::vector< double > invd_c; // per cell
   double* d_W = nullptr;
   float*  d_Wf = nullptr;
   double* d_invd_b = nullptr;
   double* d_invd_c = nullptr;
   float*  d_invd_bf = nullptr;
   float*  d_invd_cf = nullptr;
};

// scalar coefficient k(x) of -div(k grad u): constant, or exp(amp sin(2 pi f (x+p0)) cos(2 pi f (y+p1))
// sin(2 pi f (z+p2)))
// coefficient kind that selects the P1 PSPG element matrix instead of -div(k grad)
constexpr int kCoeffPSPG = 3;

// element functions of the P1 elementwise operators besides -div(k grad) and PSPG (kind 3)
constexpr int kElemLumpedMassInvK = 2;  // minus the lumped mass matrix weighted by 1/k (a Schur-complement scaling)

struct Coefficient {
   int    kind  = 0;  // 0 constant, 1 exp-sin-cos-sin, 2 radial exp(amp (value - |x|) / freq), 3 PSPG
   int    element = 0;  // 0: -div(k grad); kElemLumpedMassInvK
   double value = 1.0;
   double amp   = 0.5;
   double freq  = 1.0;
   double phase[3] = { 0, 0, 0 };
};

// per-cell geometry of elementwise operators: computational vertex coordinates and, for the
// icosahedral shell blending, the classified vertices of IcosahedralShellMap
struct CellGeom {
   double P[4][3];
   double ray[3], bxc[3];
   double volT, rad_ray, rad_ref;
   int    blend;
};
// vertices and (blending 1) the IcosahedralShellMap classification of macro-cell c
void cell_geometry( const Topology& t, int c, int blending, CellGeom& g );

struct ElemLevel {
   void* d_acc  = nullptr;  // accumulation buffer (level size, accumulation precision)
   int   acc_dtype = -1;
   void* d_invd[3] = { nullptr, nullptr, nullptr };  // inverse diagonal per DoF, per storage dtype
   int*  d_anch     = nullptr;                         // micro-cell anchors x | y << 10 | z << 20, by parity class
   int   aoff[9]    = {};                              // class p = px | py << 1 | pz << 2 spans aoff[p]..aoff[p+1]-1
   // stored element matrices (computeAndStoreLocalElementMatrices): the 10 upper-triangle entries
   // of every micro-cell's 4x4 matrix, value-major, in double ([0]) and float ([1])
   void* d_K[2] = { nullptr, nullptr };
   // P1 operators with stored matrices keep them assembled: the 15 stencil weights of every
   // cell-array slot (the partial stencil of that cell at copies of face/edge/vertex DoFs),
   // weight-major over the level's slots, in double ([0]) and float ([1])
   void* d_S[2] = { nullptr, nullptr };
   void* d_sacc = nullptr;  // Stokes coupling blocks: three velocity accumulators and one pressure accumulator
   // P2 operators with a stored coefficient function: k at every cell-array node of this storage level
   double* d_kn = nullptr;
};

struct Operator {
   Mesh*                     mesh = nullptr;
   int                       kind = 0;
   int                       minL = 0, maxL = 0;
   std::map< int, OpLevel >  lv;
   // elementwise operators
   bool                      elementwise = false;
   bool                      store_matrices = false;  // element matrices computed once and read back
   // 1: P1 operator; 2: P2 operator whose level L lives on the node set of storage level L+1
   int                       order = 1;
   // P2 elementwise operators whose coefficient is a P2 function (el[L].d_kn), evaluated at the
   // quadrature points through the P2 basis instead of from its closed form
   bool                      nodal_k = false;
   int                       blending    = 0;
   Coefficient               coeff;
   CellGeom*                 d_geom = nullptr;
   std::vector< CellGeom >   geom;
   std::map< int, ElemLevel > el;
   // P2 constant-stencil operators (HYB_P2_CONST_LAPLACE), by storage level
   std::map< int, P2cLevel > p2c;
   ~Operator();
};

struct Context {
   int          device = 0;
   cudaStream_t stream = nullptr;
   bool         own_stream = false;
   cudaStream_t aux     = nullptr;  // second stream for the boundary half of each operation
   cudaEvent_t  ev_fork = nullptr;
   cudaEvent_t  ev_join = nullptr;
   std::string  last_error;
   // scratch for reductions
   double* d_partials = nullptr;
   int     partial_cap = 0;
   double* d_scalars = nullptr;  // small pool of device scalars
   int*    d_error   = nullptr;  // device error word (bounded waits that gave up)
   double* d_stage   = nullptr;  // packed-vector staging for host transfers (grown on demand)
   int64_t stage_cap = 0;
   double* d_sor     = nullptr;  // new owner values of a Gauss-Seidel colour set (one per boundary task)
   int64_t sor_cap   = 0;
   // Buffers replaced by a larger one (partials, SOR scratch).  A CUDA graph captured earlier still
   // holds their addresses, so they stay allocated until the context is destroyed.
   std::vector< void* > retired;
   int64_t              retired_bytes = 0;
   int64_t launches = 0;         // kernel launches issued through this context
};

// --------------------------------------------------------------------------------------------
// kernel launchers (p1_kernels.cu)
// --------------------------------------------------------------------------------------------
enum StencilOp : int {
   OP_APPLY = 0,     // dst = A src
   OP_APPLY_ADD,     // dst += A src
   OP_RESID,         // dst = v1 - A src
   OP_JAC,           // dst = src + a0 * (invd * (v1 - A src)); unflagged: dst = src
   OP_CHEB0,         // dst = invd * (v1 - A src); unflagged: dst = src
   OP_CHEBI,         // dst = invd * (A src); v2 += a0 * src; unflagged: dst = v2
   OP_CHEBL,         // v2 = (v2 + a0 * src) + a1 * (invd * (A src))
   OP_DINV_APPLY,    // dst = invd * (A src)
};

struct StencilArgs {
   int         op;
   uint32_t    flag;
   int         copy_unflagged;
   const void* src;
   const void* v1;
   void*       v2;
   void*       dst;
   double      a0, a1;
};

void launch_stencil( Context* ctx, Mesh* m, Operator* A, int L, int dtype, const StencilArgs& a );
void launch_elementwise( Context* ctx, Mesh* m, Operator* A, int L, int dtype, const StencilArgs& a );
// per-copy dot products and packed transfers on meshes made of disjoint copies of one mesh
// (p1_kernels.cu; the batched solves of the serving loop)
void launch_dot_replicas( Context* ctx, Mesh* m, int L, int dtype, uint32_t flag, const void* a, const void* b, int R, const int4* tasks,
                          int tpad, double* out );
void launch_repack_map( Context* ctx, int64_t count, int np, const int64_t* poff, const int64_t* off, int dtype, int to_padded,
                        double* packed, void* vec );
// P2 constant-stencil operator (p2_constant.cu); Ls is the storage level (P2 level + 1)
void launch_p2_constant( Context* ctx, Mesh* m, Operator* A, int Ls, int dtype, const StencilArgs& a );
void build_p2_constant_level( Operator* A, int Ls );
void ensure_p2_constant_device();
void ensure_p2_constant_tables( P2cLevel& pl );
void p2_constant_inverse_diagonal( const Operator* A, int Ls, uint32_t flag, std::vector< double >& padded );
void ensure_p2_constants();
void launch_p2_restrict( Context* ctx, Mesh* m, int Lf, int dtype, uint32_t flag, const void* fine, void* coarse );
void launch_p2_prolongate( Context* ctx, Mesh* m, int Lc, int dtype, uint32_t flag, const void* coarse, void* fine, int add );
void build_elementwise_operator( Operator* A );  // host tables (cell geometry, shell classification)
void ensure_elementwise_level( Context* ctx, Operator* A, int L, int dtype );  // device buffers + diagonal
// coefficient of a P2 elementwise operator stored as a P2 function on storage level Ls: copied from
// src (a level buffer of the same layout) or, with src NULL, the closed form at the blended nodes
void set_p2_nodal_coefficient( Context* ctx, Operator* A, int Ls, const double* src );
void ensure_stokes_constants();
// Stokes coupling blocks on P1 level Lp / P2 level Lp (storage Lp+1): divt 0 dst_p (+)= div u,
// divt 1 dst_u[k] (+)= divT_k p
void launch_stokes_div( Context* ctx, Operator* op, int Lp, int dtype, int divt, const void* const* u, const void* p, void* const* dst_u,
                        void* dst_p, uint32_t flag, int add );

// full viscous velocity block on P2 level Lp (storage Lp+1): mode 0 dst[k] (+)= sum_j A_kj u[j] on
// flagged owners; mode 1 writes 1/diag(A_kk) into the accumulation-precision arrays dst[k] (u unused)
void launch_full_viscous( Context* ctx, Operator* op, int Lp, int dtype, int mode, const void* const* u, void* const* dst, uint32_t flag,
                          int add );

enum PointOp : int {
   PT_LINCOMB = 0,  // dst = a0*s0 + a1*s1 + a2*s2 (nsrc terms)
   PT_ADD,          // dst += a0*s0 + a1*s1 + a2*s2
   PT_MULT,         // dst = s0 * s1
   PT_INVERT,       // dst = 1 / s0
   PT_SET,          // dst = a0
   PT_CG_XR,        // s0 += alpha*s1 (x += alpha p);  dst -= alpha*s2 (r -= alpha ap)
   PT_CG_P,         // dst = s0 + beta*dst (p = r + beta p)
   PT_SYNC,         // write-through of owners only
};

struct PointArgs {
   int         op;
   uint32_t    flag;
   int         nsrc;
   const void* s0;
   const void* s1;
   const void* s2;
   void*       dst;
   double      a0, a1, a2;
   const double* dev_scalars;  // CG state (alpha at [4], beta at [5], done at [6])
};

void launch_point( Context* ctx, Mesh* m, int L, int dtype, const PointArgs& a );
void launch_flat_lincomb( Context* ctx, int64_t count, int dtype, void* dst, int nsrc, const void* const* srcs, const double* scal );
void launch_convert( Context* ctx, int64_t count, int dst_dtype, void* dst, int src_dtype, const void* src, double scale = 1.0 );
// packed <-> padded level vector on the device: to_padded 1 scatters the packed doubles `packed` into
// the level vector `vec` (value type dtype, padding untouched); 0 gathers vec into packed doubles
void launch_repack( Context* ctx, Mesh* m, int L, int dtype, int to_padded, double* packed, void* vec );
// deterministic dot over owned flagged DoFs -> *out (device)
void launch_dot( Context* ctx, Mesh* m, int L, int dtype, uint32_t flag, const void* a, const void* b, double* out );
void launch_dot_noalloc( Context* ctx, Mesh* m, int L, int dtype, uint32_t flag, const void* a, const void* b, double* host_out );
void launch_restrict( Context* ctx, Mesh* m, int Lfine, int dtype, uint32_t flag, const void* fine, void* coarse );
void launch_prolongate( Context* ctx, Mesh* m, int Lcoarse, int dtype, uint32_t flag, const void* coarse, void* fine, int add );
void launch_axpy_to_f64( Context* ctx, int64_t count, double* x, int src_dtype, const void* c, double a );
void prepare_device( Context* ctx, Mesh* m, Operator* op, int minL, int maxL, int dtype );
// Gauss-Seidel / SOR sweep of a constant-stencil operator on level L (in place in x, flagged DoFs):
// colour sets in the reference's primitive order (vertices, edges, faces, cells), reversed when
// backwards
void launch_sor( Context* ctx, Mesh* m, Operator* op, int L, int dtype, uint32_t flag, void* x, const void* rhs, double relax,
                 int backwards );
void launch_fill_uniform( Context* ctx, int64_t count, int dtype, void* dst, uint64_t seed );
void launch_cg_scalar( Context* ctx, double* state, int stage, double rtol, double atol );

// host helpers
void check_cuda( cudaError_t e, const char* what );

// One-time set-up per CUDA device: __constant__ tables and kernel attributes exist once per device,
// so a process that uses several devices must run each set-up on every one of them.  run(f) calls f
// once for the current device (thread-safe; later calls return at the cost of one atomic load).
class PerDeviceOnce
{
 public:
   template < class F >
   void run( F&& f )
   {
      int dev = 0;
      check_cuda( cudaGetDevice( &dev ), "cudaGetDevice" );
      if ( dev < 0 || dev >= 64 ) throw std::invalid_argument( "device ordinal out of range" );
      const uint64_t bit = uint64_t( 1 ) << dev;
      if ( done_.load( std::memory_order_acquire ) & bit ) return;
      std::lock_guard< std::mutex > lock( mu_ );
      if ( done_.load( std::memory_order_relaxed ) & bit ) return;
      f();
      done_.fetch_or( bit, std::memory_order_release );
   }
   // whether the set-up has run on the current device
   bool done_on_current_device() const
   {
      int dev = 0;
      if ( cudaGetDevice( &dev ) != cudaSuccess || dev < 0 || dev >= 64 ) return false;
      return ( done_.load( std::memory_order_acquire ) >> dev ) & 1u;
   }

 private:
   std::atomic< uint64_t > done_{ 0 };
   std::mutex              mu_;
};
void build_level( Mesh* m, int L );
void ensure_device( Mesh* m, P1Level& P );
// unit lists of the rolled-register sweep for a launch of nblocks blocks
void build_zunits( P1Level& P, int nblocks, int ncells );
// unit lists of the cell-interior sweep for a launch of nwarps warps (list index b)
void build_sweep_units( P1Level& P, int b, int nwarps, int ncells );
void build_operator_level( Operator* A, int L );
void ensure_device_op( OpLevel& ol );

}  // namespace hyb
