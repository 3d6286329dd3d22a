// Device helpers shared by the constant-stencil kernel files (sm_100a): value loads and stores,
// the level view passed to the kernels, write-through of boundary owners, and the mbarrier and
// bulk-copy primitives of the streamed sweeps.  Included by .cu files inside namespace hyb.
#pragma once

#include "hyb_internal.hpp"

#include <cuda_fp16.h>

namespace hyb {

// Cell-interior and boundary-primitive kernels of one operation write disjoint slots, so the
// boundary kernel runs on an auxiliary stream forked from (and joined back into) the context stream.
struct Fork
{
   Context* c;
   explicit Fork( Context* ctx )
   : c( ctx )
   {
      check_cuda( cudaEventRecord( c->ev_fork, c->stream ), "fork record" );
      check_cuda( cudaStreamWaitEvent( c->aux, c->ev_fork, 0 ), "fork wait" );
   }
   cudaStream_t aux() const { return c->aux; }
   ~Fork()
   {
      cudaEventRecord( c->ev_join, c->aux );
      cudaStreamWaitEvent( c->stream, c->ev_join, 0 );
   }
};

template < typename T >
struct AccT
{
   using type = float;
};
template <>
struct AccT< double >
{
   using type = double;
};

__device__ __forceinline__ double ldv( const double* p ) { return __ldg( p ); }
__device__ __forceinline__ float  ldv( const float* p ) { return __ldg( p ); }
__device__ __forceinline__ float  ldv( const __half* p ) { return __half2float( __ldg( p ) ); }
// plain (coherent) loads for vectors that are also written by the same kernel
__device__ __forceinline__ double ldc( const double* p ) { return *p; }
__device__ __forceinline__ float  ldc( const float* p ) { return *p; }
__device__ __forceinline__ float  ldc( const __half* p ) { return __half2float( *p ); }
__device__ __forceinline__ void   stv( double* p, double v ) { *p = v; }
__device__ __forceinline__ void   stv( float* p, float v ) { *p = v; }
__device__ __forceinline__ void   stv( __half* p, float v ) { *p = __float2half_rn( v ); }

// ---------------------------------------------------------------------------------------------
// argument blocks
// ---------------------------------------------------------------------------------------------
struct LevelView
{
   int              n;
   int              nrows;
   const int2*      rows;
   int              ntasks;
   const int4*      tasks;
   const int4*      btasks;      // the same tasks grouped by their primitive's boundary type
   const FaceRec*   frec;        // per grouped task: its two-cell face record (cell0 < 0: none)
   int              bcount[4];   // tasks per group: Inner, Dirichlet, Neumann, Freeslip
   const int64_t*   off;       // all primitives
   const int64_t*   cell_off;  // off + nB
   const int*       inc_begin;
   const Incidence* inc;
   const uint8_t*   bc;       // all primitives
   const uint8_t*   cell_bc;  // bc + nB
   const int8_t*    bkind;
   const float*     ncell_cls;
   int              nmarch;
   const int4*      march;
   int              nzblocks;  // blocks of the rolled sweep and their units (zunits/zcell from zbegin[b])
   const int4*      zunits;
   const int*       zcell;
   const int*       zbegin;
   int              nswarps[kSwLists];  // warps of a cell-sweep launch with 2, 3, 4 blocks per SM
   const int4*      swunits[kSwLists];
   const int*       swcell[kSwLists];
   const int*       swbegin[kSwLists];
};

template < typename A >
struct OpView
{
   const A* W;       // [nC][15][15]
   const A* invd_b;  // per boundary primitive
   const A* invd_c;  // per cell
};

static inline LevelView make_view( Mesh* m, int L )
{
   P1Level& P = m->level( L );
   ensure_device( m, P );
   LevelView v;
   v.n         = P.n;
   v.nrows     = int( P.rows.size() );
   v.rows      = P.d_rows;
   v.ntasks    = int( P.tasks.size() );
   v.tasks     = P.d_tasks;
   v.btasks    = P.d_btasks;
   v.frec      = P.d_frec;
   for ( int g = 0; g < 4; ++g ) v.bcount[g] = P.bcount[g];
   v.off       = P.d_off;
   v.cell_off  = P.d_off + P.nB;
   v.inc_begin = P.d_inc_begin;
   v.inc       = P.d_inc;
   v.bc        = P.d_bc;
   v.cell_bc   = P.d_bc + P.nB;
   v.bkind     = P.d_bkind;
   v.ncell_cls = P.d_ncell_cls;
   v.nmarch     = int( P.march.size() );
   v.march      = P.d_march;
   v.nzblocks = int( P.zbegin.size() ) - 1;
   v.zunits   = P.d_zunits;
   v.zcell    = P.d_zcell;
   v.zbegin   = P.d_zbegin;
   for ( int b = 0; b < kSwLists; ++b )
   {
      v.nswarps[b] = int( P.swbegin[b].size() ) - 1;
      v.swunits[b] = P.d_swunits[b];
      v.swcell[b]  = P.d_swcell[b];
      v.swbegin[b] = P.d_swbegin[b];
   }
   return v;
}

// The contiguous groups of the type-sorted task list a boundary launch covers: every group when
// unflagged owners are copied, else the groups whose boundary type is in `flag`.
struct TaskSegments
{
   int start[4];
   int count[4];
};

static inline TaskSegments task_segments( const LevelView& v, uint32_t flag, int all )
{
   static const uint32_t type_bit[4] = { kInner, kDirichlet, kNeumann, kFreeslip };
   TaskSegments          s{};
   int                   k = 0, at = 0;
   for ( int g = 0; g < 4; ++g )
   {
      if ( v.bcount[g] > 0 && ( all || ( flag & type_bit[g] ) ) )
      {
         s.start[k] = at;
         s.count[k] = v.bcount[g];
         ++k;
      }
      at += v.bcount[g];
   }
   return s;
}

__device__ __forceinline__ int64_t owner_slot( const LevelView& v, int b, int i, int j )
{
   const int k = v.bkind[b];
   return v.off[b] + ( k == 0 ? 0 : ( k == 1 ? int64_t( i ) : fidx( v.n, i, j ) ) );
}

__device__ __forceinline__ void inc_point( const Incidence& I, int n, int i, int j, int& x, int& y, int& z )
{
   x = n * I.o[0] + i * I.e1[0] + j * I.e2[0];
   y = n * I.o[1] + i * I.e1[1] + j * I.e2[1];
   z = n * I.o[2] + i * I.e1[2] + j * I.e2[2];
}

// store val to the owner slot and every copy in the neighbouring cell arrays
template < typename T, typename A >
__device__ __forceinline__ void write_through( const LevelView& v, T* vec, int b, int i, int j, int64_t owner, A val )
{
   stv( vec + owner, val );
   // incidences read four at a time ahead of their stores (a vertex has many cells)
   const int q1 = v.inc_begin[b + 1];
   for ( int q = v.inc_begin[b]; q < q1; q += 4 )
   {
      int64_t sl[4];
#pragma unroll
      for ( int u = 0; u < 4; ++u )
      {
         sl[u] = -1;
         if ( q + u < q1 )
         {
            const Incidence I = v.inc[q + u];
            int             x, y, z;
            inc_point( I, v.n, i, j, x, y, z );
            sl[u] = v.cell_off[I.cell] + cidx( v.n, x, y, z );
         }
      }
#pragma unroll
      for ( int u = 0; u < 4; ++u )
         if ( sl[u] >= 0 ) stv( vec + sl[u], val );
   }
}

__device__ __forceinline__ uint32_t smem_addr( const void* p ) { return uint32_t( __cvta_generic_to_shared( p ) ); }

__device__ __forceinline__ void mbar_init( uint64_t* bar, uint32_t count )
{
   asm volatile( "mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"( smem_addr( bar ) ), "r"( count ) : "memory" );
}

__device__ __forceinline__ void mbar_expect_tx( uint64_t* bar, uint32_t bytes )
{
   asm volatile( "mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"( smem_addr( bar ) ), "r"( bytes ) : "memory" );
}

__device__ __forceinline__ void mbar_arrive( uint64_t* bar )
{
   asm volatile( "mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"( smem_addr( bar ) ) : "memory" );
}

__device__ __forceinline__ bool mbar_try_wait( uint64_t* bar, uint32_t parity )
{
   uint32_t ok;
   asm volatile( "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
                 : "=r"( ok )
                 : "r"( smem_addr( bar ) ), "r"( parity )
                 : "memory" );
   return ok != 0;
}

__device__ __forceinline__ void bulk_copy_g2s( void* dst, const void* src, uint32_t bytes, uint64_t* bar )
{
   asm volatile( "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"( smem_addr( dst ) ),
                 "l"( src ), "r"( bytes ), "r"( smem_addr( bar ) )
                 : "memory" );
}

__device__ __forceinline__ uint64_t global_ns()
{
   uint64_t t;
   asm volatile( "mov.u64 %0, %%globaltimer;" : "=l"( t ) );
   return t;
}

// A healthy wait lasts microseconds; one second means the copy or the partner warps are gone.
constexpr uint64_t kWaitLimitNs = 1000000000ull;

// bounded wait for the completion of phase `parity`; false if it ran out or (when abort_flag is
// given) another warp of the block aborted
__device__ __forceinline__ bool mbar_wait_bounded( uint64_t* bar, uint32_t parity, const volatile int* abort_flag )
{
   if ( mbar_try_wait( bar, parity ) ) return true;
   const uint64_t t0 = global_ns();
   for ( ;; )
   {
      if ( mbar_try_wait( bar, parity ) ) return true;
      if ( abort_flag && *abort_flag ) return false;
      if ( global_ns() - t0 > kWaitLimitNs ) return false;
   }
}

// Ops whose epilogue reads a second vector at the point (b for residual, Jacobi and the first
// Chebyshev step, the running update for the later ones, dst itself for apply-add) stage that
// vector's tile rows (no halo) in the same stage, so no step waits on a global load.
template < int OP >
__host__ __device__ constexpr bool sweep_aux()
{
   return OP == OP_APPLY_ADD || OP == OP_RESID || OP == OP_JAC || OP == OP_CHEB0 || OP == OP_CHEBI || OP == OP_CHEBL;
}

// offset of slice z+1 minus offset of slice z in a macro-cell array (tri(n+1-z) points in slice z)
__device__ __forceinline__ int64_t slice_step( int n, int z ) { return int64_t( n + 1 - z ) * ( n + 2 - z ) / 2; }

// epilogue of a stencil operation at slot i: s = (A src)_i; invd the inverse diagonal at the point
template < typename T, typename A, int OP >
__device__ __forceinline__ void stencil_epilogue( int64_t i, A s, A invd, const T* src, const T* v1, T* v2, T* dst, A a0, A a1 )
{
   if constexpr ( OP == OP_APPLY ) stv( dst + i, s );
   else if constexpr ( OP == OP_APPLY_ADD ) stv( dst + i, A( ldc( dst + i ) ) + s );
   else if constexpr ( OP == OP_RESID ) stv( dst + i, A( ldv( v1 + i ) ) - s );
   else if constexpr ( OP == OP_JAC ) stv( dst + i, A( ldv( src + i ) ) + a0 * ( invd * ( A( ldv( v1 + i ) ) - s ) ) );
   else if constexpr ( OP == OP_CHEB0 ) stv( dst + i, invd * ( A( ldv( v1 + i ) ) - s ) );
   else if constexpr ( OP == OP_CHEBI )
   {
      stv( dst + i, invd * s );
      stv( v2 + i, A( ldc( v2 + i ) ) + a0 * A( ldv( src + i ) ) );
   }
   else if constexpr ( OP == OP_CHEBL ) stv( v2 + i, ( A( ldc( v2 + i ) ) + a0 * A( ldv( src + i ) ) ) + a1 * ( invd * s ) );
   else if constexpr ( OP == OP_DINV_APPLY ) stv( dst + i, invd * s );
}

}  // namespace hyb
