// CUDA kernels of the P1 vertex-DoF multigrid path (sm_100a).
//
// Two kernel families cover every operation:
//  * cell kernels: one warp per interior row (y, z) of a macro-cell, lanes over x.  The 15-point
//    stencil reads only the cell's own array, whose boundary slabs hold up-to-date copies of the
//    face/edge/vertex owners (write-through invariant).
//  * boundary kernels: one thread per owned DoF of a macro-face/edge/vertex.  The stencil is the
//    sum over the neighbouring macro-cells of the cell-restricted stencil of the point's position
//    class, read from each cell's array (the same decomposition as
//    P1ConstantOperator::apply_face3D_generated, P1ConstantOperator.cpp:239-357, which sums the
//    one-sided stencil of every neighbour cell).  The result is written to the owner and to every
//    copy in the neighbouring cell arrays.
// The path is bandwidth bound: no tensor cores, fp64 accumulation for fp64 storage and fp32
// accumulation for fp32/fp16 storage.
#include "../../include/hyteg_b200.h"
#include "hyb_internal.hpp"
#include "hyb_device.cuh"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <stdexcept>
#include <string>
#include <type_traits>

namespace hyb {

__constant__ int      c_dirs[kNumDirs][3];
__constant__ uint16_t c_cls_mask[kNumClasses];
__constant__ int8_t   c_mask_to_cls[16];

static void    sweep_attributes_all();
static double* noalloc_scratch( int device );
static PerDeviceOnce g_const_once;
// constant tables and kernel attributes of this file, once per device; called before any stream
// capture (prepare_device).  It also resolves the device address of the allocation-free dot's fixed
// scratch, so that entry point itself never has to load anything.
static void ensure_constants()
{
   g_const_once.run( [] {
      int dev = 0;
      check_cuda( cudaGetDevice( &dev ), "cudaGetDevice" );
      noalloc_scratch( dev );
      sweep_attributes_all();
      check_cuda( cudaMemcpyToSymbol( c_dirs, kDirs, sizeof( kDirs ) ), "constants(dirs)" );
      check_cuda( cudaMemcpyToSymbol( c_cls_mask, kClassDirMask, sizeof( kClassDirMask ) ), "constants(mask)" );
      int8_t m2c[16];
      for ( int m = 0; m < 16; ++m ) m2c[m] = -1;
      // z==0 -> bit0, y==0 -> bit1, x==0 -> bit2, x+y+z==n -> bit3
      const int faces[kNumClasses] = { 0, 1, 2, 4, 8, 3, 5, 9, 6, 10, 12, 7, 11, 13, 14 };
      for ( int c = 0; c < kNumClasses; ++c ) m2c[faces[c]] = int8_t( c );
      check_cuda( cudaMemcpyToSymbol( c_mask_to_cls, m2c, sizeof( m2c ) ), "constants(classes)" );
   } );
}


__device__ __forceinline__ int point_class( int n, int x, int y, int z )
{
   const int m = ( z == 0 ) | ( ( y == 0 ) << 1 ) | ( ( x == 0 ) << 2 ) | ( ( x + y + z == n ) << 3 );
   return c_mask_to_cls[m];
}


// ---------------------------------------------------------------------------------------------
// stencil sweeps
// ---------------------------------------------------------------------------------------------

// y-marching cell sweep: a warp owns x0..x0+31 of slice z and walks the rows y_first..y_last.  The
// rows (y-1, y, y+1) of slice z, (y-1, y) of slice z+1 and (y, y+1) of slice z-1 roll through
// registers, so each step loads three new rows (x-1, x, x+1 per lane; neighbours hit L1) instead
// of fifteen values per point.
template < typename T, typename A >
struct Row3
{
   A m, o, p;
};

template < typename T, typename A >
__device__ __forceinline__ Row3< T, A > load_row( const T* s, int n, int yy, int zz, int x )
{
   const int64_t rb  = cidx( n, 0, yy, zz );
   const int     len = n - yy - zz;  // last valid x of the row
   Row3< T, A >  r;
   r.m = ( x - 1 <= len ) ? A( ldv( s + rb + x - 1 ) ) : A( 0 );
   r.o = ( x <= len ) ? A( ldv( s + rb + x ) ) : A( 0 );
   r.p = ( x + 1 <= len ) ? A( ldv( s + rb + x + 1 ) ) : A( 0 );
   return r;
}

__device__ __forceinline__ void prefetch_l2( const void* p ) { asm volatile( "prefetch.global.L2 [%0];" ::"l"( p ) ); }

template < typename T, typename A, int OP >
__global__ void __launch_bounds__( 256 ) k_cell_march( LevelView v, OpView< A > o, uint32_t flag, const T* __restrict__ src,
                                                        const T* __restrict__ v1, T* v2, T* dst, A a0, A a1 )
{
   const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
   const int item = blockIdx.x * 8 + warp;
   const int c    = blockIdx.y;
   if ( item >= v.nmarch ) return;
   if ( !( v.cell_bc[c] & flag ) ) return;
   const int4    it   = v.march[item];
   const int     z = it.x, x = it.y + lane, ya = it.z, yb = it.w, n = v.n;
   const int64_t base = v.cell_off[c];
   const T*      s    = src + base;
   const A*      W    = o.W + size_t( c ) * kNumClasses * kNumDirs;
   const A w0 = W[0], wW = W[1], wE = W[2], wS = W[3], wN = W[4], wB = W[5], wT = W[6], wNW = W[7], wSE = W[8], wTW = W[9],
           wBE = W[10], wTS = W[11], wBN = W[12], wTSE = W[13], wBNW = W[14];
   const A invd = o.invd_c[c];
   Row3< T, A > cm = load_row< T, A >( s, n, ya - 1, z, x );
   Row3< T, A > c0 = load_row< T, A >( s, n, ya, z, x );
   Row3< T, A > tm = load_row< T, A >( s, n, ya - 1, z + 1, x );
   Row3< T, A > b0 = load_row< T, A >( s, n, ya, z - 1, x );
   constexpr int pd = 8;  // rows pulled into L2 ahead of the march
#pragma unroll 2
   for ( int y = ya; y <= yb; ++y )
   {
      if ( pd > 0 )
      {
         // pull the rows needed pd steps ahead into L2 (addresses stay inside the cell array)
         const int yp = y + pd;
         if ( yp + 1 + z <= n && x <= n - yp - 1 - z ) prefetch_l2( s + cidx( n, x, yp + 1, z ) );
         if ( yp + z + 1 <= n && x <= n - yp - z - 1 ) prefetch_l2( s + cidx( n, x, yp, z + 1 ) );
         if ( yp + 1 + z - 1 <= n && x <= n - yp - z ) prefetch_l2( s + cidx( n, x, yp + 1, z - 1 ) );
      }
      const Row3< T, A > cp = load_row< T, A >( s, n, y + 1, z, x );
      const Row3< T, A > t0 = load_row< T, A >( s, n, y, z + 1, x );
      const Row3< T, A > bp = load_row< T, A >( s, n, y + 1, z - 1, x );
      if ( x + y + z <= n - 1 )
      {
         A acc = w0 * c0.o;
         acc += wW * c0.m;
         acc += wE * c0.p;
         acc += wS * cm.o;
         acc += wN * cp.o;
         acc += wB * b0.o;
         acc += wT * t0.o;
         acc += wNW * cp.m;
         acc += wSE * cm.p;
         acc += wTW * t0.m;
         acc += wBE * b0.p;
         acc += wTS * tm.o;
         acc += wBN * bp.o;
         acc += wTSE * tm.p;
         acc += wBNW * bp.m;
         stencil_epilogue< T, A, OP >( base + cidx( n, x, y, z ), acc, invd, src, v1, v2, dst, a0, a1 );
      }
      cm = c0;
      c0 = cp;
      tm = t0;
      b0 = bp;
   }
}



// epilogue of the z-streamed sweep: the centre of src and the second vector come from the stage
template < typename T, typename A, int OP >
__device__ __forceinline__ void sweep_epilogue( int64_t i, A s, A invd, A centre, A aux, T* v2, T* dst, A a0, A a1 )
{
   if constexpr ( OP == OP_APPLY ) stv( dst + i, s );
   else if constexpr ( OP == OP_APPLY_ADD ) stv( dst + i, aux + s );
   else if constexpr ( OP == OP_RESID ) stv( dst + i, aux - s );
   else if constexpr ( OP == OP_JAC ) stv( dst + i, centre + a0 * ( invd * ( aux - s ) ) );
   else if constexpr ( OP == OP_CHEB0 ) stv( dst + i, invd * ( aux - s ) );
   else if constexpr ( OP == OP_CHEBI )
   {
      stv( dst + i, invd * s );
      stv( v2 + i, aux + a0 * centre );
   }
   else if constexpr ( OP == OP_CHEBL ) stv( v2 + i, ( aux + a0 * centre ) + a1 * ( invd * s ) );
   else if constexpr ( OP == OP_DINV_APPLY ) stv( dst + i, invd * s );
}

// ---------------------------------------------------------------------------------------------
// Cell-interior sweep for levels with n >= 32 (every stencil operation, every value type).
//
// Work unit: the rows y0..y0+kSwR-1 and the x-points x0..x0+63 (x0..x0+31 for a half-width unit)
// of the slices z_first..z_last of one macro-cell, interior points only (x, y, z >= 1,
// x + y + z <= n - 1).  Every warp of a launch owns a fixed list of units (balanced on the host)
// and runs them on its own: it streams the rows y0-1..y0+kSwR of the slices z_first-1..z_last+1,
// with one point of halo in x, into a private ring of kSwD shared-memory stages with
// cp.async.bulk (one copy per row, issued by one lane each, completing on the stage's mbarrier),
// keeping kSwD-1 slice loads in flight while it computes one.  Loads run ahead across unit
// boundaries.  The second vector of an epilogue (b of residual / Jacobi / Chebyshev, the running
// update of later Chebyshev steps, dst for apply-add) is staged in the same stage, rows y0..y0+kSwR-1
// without halo.
//
// Partial sums in y and z: lane l owns the points x = x0 + l + 32k (k < 2) of the unit's rows.  The
// values (x-1, x, x+1) of row y of slice s are read from the stage once and give every stencil term
// that involves them: the bottom terms (B, BE, BN, BNW) of slice s+1 in rows y and y-1, the middle
// terms (W, C, E, S, SE, N, NW) of slice s in rows y-1, y and y+1, and the top terms (T, TW, TS,
// TSE) of slice s-1 in rows y and y+1.  A point of slice s-1 is complete once rows y-1 and y of
// slice s are folded in and is written right away.  A slice step therefore reads three values per
// point plus four per column for the two halo rows, and issues exactly 15 multiply-adds per point.
// The running sums of slices s-1, s and s+1 occupy three register slots that rotate; the slice loop
// is unrolled by three so the rotation costs no moves.  The centre value and the second-vector value
// of a point are read in the step of its own slice and carried to the next step.
//
// Each point sums its 15 terms in one fixed order (bottom terms, middle terms, top terms, each in
// row order), whatever unit computes it, so results are deterministic.  Waits on the stages are
// bounded by the global timer; a warp whose wait runs out records an error in *err, waits (bounded)
// for its copies in flight and returns.
// ---------------------------------------------------------------------------------------------
template < typename T, int OP >
struct SwCfg
{
   static constexpr bool   AUX   = sweep_aux< OP >();
   static constexpr bool   CEN   = OP == OP_JAC || OP == OP_CHEBI || OP == OP_CHEBL;  // epilogue reads the centre value
   // blocks per SM, by the register budget of the running sums (and of the centre and second-vector
   // values the smoother epilogues carry)
   static constexpr int    BPS   = sizeof( T ) == 8 ? ( ( CEN || AUX ) ? 2 : 3 ) : ( AUX ? 3 : 4 );
   static constexpr int    al    = 16 / int( sizeof( T ) );                             // elements per 16 bytes
   static constexpr int    RW    = ( kSwTX + 2 + 2 * al + al - 1 ) / al * al;          // source row (elements)
   static constexpr int    RWA   = ( kSwTX + 2 * al + al - 1 ) / al * al;              // second-vector row
   static constexpr int    rows  = kSwR + 2;                                           // tile rows + halo
   static constexpr int    aux0  = rows * RW;                                          // second-vector rows start here
   static constexpr int    stage = aux0 + ( AUX ? kSwR * RWA : 0 );                    // elements per stage
   static constexpr int    Draw  = int( ( 216 * 1024 ) / ( BPS * kSwWarps ) / ( stage * int( sizeof( T ) ) ) );
   static constexpr int    D     = Draw < 3 ? 3 : ( Draw > 8 ? 8 : Draw );             // ring depth
   static constexpr size_t warp_elems = size_t( D ) * stage;
   static constexpr size_t smem_bytes = kSwWarps * warp_elems * sizeof( T );
   static_assert( ( stage * sizeof( T ) ) % 16 == 0 && ( RW * sizeof( T ) ) % 16 == 0 && ( RWA * sizeof( T ) ) % 16 == 0,
                  "bulk copies need 16-byte aligned stage rows" );
   static_assert( kSwR + 2 + ( AUX ? kSwR : 0 ) <= 32, "one row copy per lane" );
   static_assert( kSwR == 4, "the row prefetch of k_cell_sweep is written out for six stage rows" );
};

template < typename T, typename A, int OP >
__global__ void __launch_bounds__( kSwWarps * 32, SwCfg< T, OP >::BPS )
    k_cell_sweep( LevelView v, OpView< A > o, uint32_t flag, const T* __restrict__ src, const T* __restrict__ v1, T* v2, T* dst, A a0,
                  A a1, int nC, int* err )
{
   using Cfg                = SwCfg< T, OP >;
   constexpr bool AUX       = Cfg::AUX;
   constexpr bool CEN       = Cfg::CEN;
   constexpr int  D = Cfg::D, RW = Cfg::RW, RWA = Cfg::RWA, AL = Cfg::al, R = kSwR;
   extern __shared__ __align__( 128 ) unsigned char sw_raw[];
   __shared__ uint64_t bars[kSwWarps][D];
   const int           warp = threadIdx.x >> 5, lane = threadIdx.x & 31, n = v.n;
   T* const            ring = reinterpret_cast< T* >( sw_raw ) + size_t( warp ) * Cfg::warp_elems;
   uint64_t* const     full = bars[warp];
   if ( lane == 0 )
   {
      for ( int s = 0; s < D; ++s ) mbar_init( &full[s], 1 );
      asm volatile( "fence.mbarrier_init.release.cluster;" ::: "memory" );
   }
   __syncwarp();
   constexpr int bi  = Cfg::BPS - 2;
   const int     gw  = blockIdx.x * kSwWarps + warp;
   const int*    ucl = v.swcell[bi];
   const int4*   uu  = v.swunits[bi];
   const int     u1  = v.swbegin[bi][gw + 1];
   const T*      aux = ( OP == OP_CHEBI || OP == OP_CHEBL ) ? v2 : ( OP == OP_APPLY_ADD ? dst : v1 );
   auto active = [&]( int u ) {
      const int c = ucl[u];
      return c < nC && ( v.cell_bc[c] & flag ) != 0;
   };

   // ---- loads: one cursor walks the same unit sequence as the computation, up to D loads ahead.
   // Lane r < R+2 copies source row y0-1+r, lane R+2+r (AUX) second-vector row y0+r; each lane keeps
   // its row's offset in the slice being loaded and advances it by additions.
   const bool is_src = lane < R + 2, is_aux = AUX && lane >= R + 2 && lane < 2 * R + 2;
   int        pu = v.swbegin[bi][gw];
   int        ps = 0, pyy = 0;  // next slice of unit pu to load; this lane's row
   int64_t    prb = 0;          // offset of that row in slice ps (cell-relative)
   int4       PU  = make_int4( 0, 0, 0, 0 );
   int64_t    pcb = 0;
   auto       open = [&]() {
      while ( pu < u1 && !active( pu ) ) ++pu;
      if ( pu < u1 )
      {
         PU  = uu[pu];
         pcb = v.cell_off[ucl[pu]];
         ps  = PU.z - 1;
         pyy = is_src ? PU.y - 1 + lane : PU.y + ( lane - R - 2 );
         prb = cidx( n, 0, pyy, ps );
      }
   };
   open();
   int  issued = 0, ist = 0;  // loads issued; stage of the next one
   auto issue  = [&]() {
      if ( pu >= u1 ) return;
      const int  st   = ist;
      const int  x0   = PU.x & kSwUnitXMask, tw = ( PU.x & kSwUnitHalf ) ? 32 : kSwTX;
      const int  xa   = is_src ? x0 - 1 : x0;
      const int  xe   = is_src ? min( x0 + tw, n - pyy - ps ) : min( x0 + tw - 1, n - 1 - pyy - ps );
      const bool live = ( is_src && pyy + ps <= n && xe >= xa ) || ( is_aux && ps >= PU.z && ps <= PU.w && xe >= xa );
      uint32_t   bytes = 0;
      int64_t    a0s   = 0;
      if ( live )
      {
         const int64_t s0 = prb + xa, e1 = prb + xe + 1;
         const int     sh = int( s0 & ( AL - 1 ) );  // the cell array starts on a 32-element boundary
         a0s              = s0 - sh;
         bytes            = uint32_t( ( ( e1 + AL - 1 ) / AL * AL - a0s ) * int64_t( sizeof( T ) ) );
      }
      const uint32_t total = __reduce_add_sync( 0xffffffffu, bytes );
      if ( lane == 0 ) mbar_expect_tx( &full[st], total );
      __syncwarp();
      if ( bytes )
         bulk_copy_g2s( ring + st * Cfg::stage + ( is_src ? lane * RW : Cfg::aux0 + ( lane - R - 2 ) * RWA ), ( is_src ? src : aux ) + pcb + a0s,
                        bytes, &full[st] );
      ++issued;
      ist = ist + 1 == D ? 0 : ist + 1;
      // cidx(0, y, z+1) = cidx(0, y, z) + tri(n+1-z) - y
      prb += slice_step( n, ps ) - pyy;
      if ( ++ps > PU.w + 1 )
      {
         ++pu;
         open();
      }
   };
   for ( int i = 0; i < D; ++i ) issue();


   int  ld = 0, cst = 0;  // loads consumed; stage of the next one
   uint32_t cph  = 0;     // its phase parity
   auto fail = [&]() {
      if ( lane == 0 )
      {
         atomicExch( err, 1 );
         // the copies still in flight must land before the block's shared memory is released
         for ( int i = ld; i < issued; ++i )
            if ( !mbar_wait_bounded( &full[i % D], uint32_t( ( i / D ) & 1 ), nullptr ) ) break;
      }
      __syncwarp();
   };

   A   w[kNumDirs], invd = A( 0 );
   int cw = -1;
   for ( int u = v.swbegin[bi][gw]; u < u1; ++u )
   {
      if ( !active( u ) ) continue;
      const int c = ucl[u];
      if ( c != cw )
      {
#pragma unroll
         for ( int d = 0; d < kNumDirs; ++d ) w[d] = o.W[size_t( c ) * kNumClasses * kNumDirs + d];  // interior class 0
         invd = o.invd_c[c];
         cw   = c;
      }
      const int4    U  = uu[u];
      const int     x0 = U.x & kSwUnitXMask, y0 = U.y, za = U.z, zb = U.w;
      const int64_t cb = v.cell_off[c];
      const int64_t cbx = cb + x0 + lane;  // index of point (x0 + lane, 0, 0) of the cell
      auto          unit = [&]( auto kp_c ) -> bool {
         constexpr int KP = decltype( kp_c )::value;
         A             acc[3][R][KP];
         A             cen[3][R][KP];
         A             axv[3][R][KP];
         // cell-relative start of row y0-1+jj in the slice read last; the slice loop advances it before
         // every step, so it starts one slice below z_first-1 (the offset formula and its recurrence
         // cidx(0, y, z+1) = cidx(0, y, z) + tri(n+1-z) - y are one polynomial identity, so the
         // start value for slice z_first-2 >= -1 is exact)
         int rb[R + 2];
#pragma unroll
         for ( int jj = 0; jj < R + 2; ++jj ) rb[jj] = int( cidx( n, 0, y0 - 1 + jj, za - 2 ) );
         // one slice step: slice s (the next load) folded into the sums of slot PH (points of slice s),
         // slot (PH+2)%3 (slice s-1, completed and written when s-1 >= z_first) and slot (PH+1)%3
         // (slice s+1).  The steps of slices z_first-1 and z_last+1 run the same code: what they add to
         // slices outside the unit is never written.
         auto step = [&]( int s, auto ph_c ) -> bool {
            constexpr int PH = decltype( ph_c )::value, CS = PH, NS = ( PH + 1 ) % 3, PS = ( PH + 2 ) % 3;
            // every lane waits; a wait that ran out on any lane fails the whole warp
            if ( !__all_sync( 0xffffffffu, mbar_wait_bounded( &full[cst], cph, nullptr ) ) ) return false;
            const T*   Rg   = ring + cst * Cfg::stage;
            const int  sst  = int( slice_step( n, s - 1 ) );
            const int  lim  = s > za ? n - x0 - y0 - s : -64;  // point (x0 + l, y0 + j, s - 1) is written iff l + j <= lim
            // the values (x-1, x, x+1) of stage row jj; the rows are read one ahead of the arithmetic
            // and stores of the current row, so the shared loads never wait behind global stores
            A    va[R + 2][KP], vb[R + 2][KP], vc[R + 2][KP];
            auto fetch = [&]( auto jj_c ) {
               constexpr int jj   = decltype( jj_c )::value;
               const int     rnew = rb[jj] + sst - ( y0 - 1 + jj );
               const T*      rp   = Rg + jj * RW + ( ( rnew + x0 - 1 ) & ( AL - 1 ) ) + lane;  // rp[0] = x - 1 for k = 0
#pragma unroll
               for ( int k = 0; k < KP; ++k )
               {
                  vb[jj][k] = A( rp[32 * k + 1] );
                  va[jj][k] = jj > 0 ? A( rp[32 * k] ) : A( 0 );
                  vc[jj][k] = jj < R + 1 ? A( rp[32 * k + 2] ) : A( 0 );
               }
            };
            fetch( std::integral_constant< int, 0 >{} );
#pragma unroll
            for ( int jj = 0; jj < R + 2; ++jj )
            {
               if ( jj + 1 < R + 2 )
               {
                  // static dispatch of the next row's fetch (jj is a compile-time value after unrolling)
                  if ( jj == 0 ) fetch( std::integral_constant< int, 1 >{} );
                  if ( jj == 1 ) fetch( std::integral_constant< int, 2 >{} );
                  if ( jj == 2 ) fetch( std::integral_constant< int, 3 >{} );
                  if ( jj == 3 ) fetch( std::integral_constant< int, 4 >{} );
                  if ( jj == 4 ) fetch( std::integral_constant< int, 5 >{} );
               }
               const int j    = jj - 1;  // tile row of this stage row (-1 and R are halo rows)
               const int rold = rb[jj];
               const int rnew = rold + sst - ( y0 - 1 + jj );
               rb[jj]         = rnew;
               const int64_t io = cbx + rold;  // output index of (x0 + lane, y, s-1)
#pragma unroll
               for ( int k = 0; k < KP; ++k )
               {
                  const int q = 32 * k;
                  const A   b = vb[jj][k], a = va[jj][k], cc = vc[jj][k];
                  // bottom terms of slice s+1
                  if ( j >= 0 && j < R )
                  {
                     acc[NS][j][k] = w[5] * b;
                     acc[NS][j][k] += w[10] * cc;
                  }
                  if ( j >= 1 )
                  {
                     acc[NS][j - 1][k] += w[12] * b;
                     acc[NS][j - 1][k] += w[14] * a;
                  }
                  // middle terms of slice s
                  if ( j + 1 < R )
                  {
                     acc[CS][j + 1][k] += w[3] * b;
                     acc[CS][j + 1][k] += w[8] * cc;
                  }
                  if ( j >= 0 && j < R )
                  {
                     acc[CS][j][k] += w[1] * a;
                     acc[CS][j][k] += w[0] * b;
                     acc[CS][j][k] += w[2] * cc;
                     if constexpr ( CEN ) cen[CS][j][k] = b;
                     if constexpr ( AUX ) axv[CS][j][k] = A( Rg[Cfg::aux0 + j * RWA + ( ( rnew + x0 ) & ( AL - 1 ) ) + lane + q] );
                  }
                  if ( j >= 1 )
                  {
                     acc[CS][j - 1][k] += w[4] * b;
                     acc[CS][j - 1][k] += w[7] * a;
                  }
                  // top terms of slice s-1; a point is complete after its own row
                  if ( j + 1 < R )
                  {
                     acc[PS][j + 1][k] += w[11] * b;
                     acc[PS][j + 1][k] += w[13] * cc;
                  }
                  if ( j >= 0 && j < R )
                  {
                     acc[PS][j][k] += w[6] * b;
                     acc[PS][j][k] += w[9] * a;
                     if ( lane + q + j <= lim )
                        sweep_epilogue< T, A, OP >( io + q, acc[PS][j][k], invd, cen[PS][j][k], axv[PS][j][k], v2, dst, a0, a1 );
                  }
               }
            }
            // every lane has read the stage: hand it back to the async proxy and refill it
            asm volatile( "fence.proxy.async.shared::cta;" ::: "memory" );
            __syncwarp();
            ++ld;
            if ( ++cst == D ) cst = 0, cph ^= 1u;
            issue();
            return true;
         };
         // the slot of the points of slice p is (p - z_first + 1) mod 3; the steps run z_first-1 .. z_last+1
         using I0 = std::integral_constant< int, 0 >;
         using I1 = std::integral_constant< int, 1 >;
         using I2 = std::integral_constant< int, 2 >;
         for ( int s = za - 1;; )
         {
            if ( !step( s, I0{} ) ) return false;
            if ( ++s > zb + 1 ) return true;
            if ( !step( s, I1{} ) ) return false;
            if ( ++s > zb + 1 ) return true;
            if ( !step( s, I2{} ) ) return false;
            if ( ++s > zb + 1 ) return true;
         }
      };
      const bool ok = ( U.x & kSwUnitHalf ) ? unit( std::integral_constant< int, 1 >{} ) : unit( std::integral_constant< int, kSwTX / 32 >{} );
      if ( !ok ) return fail();
   }
}

// ---------------------------------------------------------------------------------------------
// Rolled-register z-streamed cell sweep, for the operations with a second vector (residual, Jacobi,
// Chebyshev steps, apply-add) on levels with n >= 32.
//
// A unit is the tile x0..x0+63, y0..y0+7 of slices z_first..z_last of one macro-cell.  Two producer
// warps stream the tile's rows of every slice (one-point halo in x and y, plus the tile rows of the
// second vector) into a ring of shared-memory stages with cp.async.bulk: lane r issues one copy per
// row, each stage's full barrier completes when all bytes have landed.  Eight consumer warps (one
// per tile row, two x per lane) march up the slices; of the 15 stencil values, four in slice z-1 and
// four in slice z were read in the previous step and roll through registers, so a step reads three
// values of slice z and four of slice z+1 from shared memory, and slice z is released (empty
// barrier, one arrival per consumer warp) as soon as step z ends.  Keeping the producer work in two
// warps and the consumers' state small (about 96 registers) gives 20 warps per SM, which these
// register-heavy epilogues need more than the fewer shared reads of the partial-sum sweep above.
// Global rows start at arbitrary element offsets: each row copy is widened to 16-byte boundaries
// and its shift is published with the stage as 3-bit fields of one word.  Every wait is bounded by
// the global timer; when one runs out the block records an error in *err, raises a block-wide abort
// flag, stops issuing copies, waits (bounded) for the copies it has in flight and returns.
// ---------------------------------------------------------------------------------------------
constexpr int kZTileXR = 64;  // x-points per tile row (two per consumer lane)
template < typename T, bool AUX >
struct ZCfg
{
      static constexpr int kZTileX = kZTileXR;                                      // x-points per tile row
   static constexpr int pts     = kZTileX / 32;                                 // x-points per consumer lane
   static constexpr int al    = 16 / int( sizeof( T ) );                         // elements per 16 bytes
   static constexpr int RW    = ( kZTileX + 2 + 2 * al + al - 1 ) / al * al;    // source row width (elements)
   static constexpr int RWA   = ( kZTileX + 2 * al + al - 1 ) / al * al;        // second-vector row width
   static constexpr int rows  = kZTileY + 2;                                   // tile rows + halo
   static constexpr int aux0  = rows * RW;                                     // second-vector rows start here
   static constexpr int stage = aux0 + ( AUX ? kZTileY * RWA : 0 );            // elements per stage
   static constexpr int S     = AUX ? 8 : 10;                                   // ring depth
   static constexpr size_t smem_bytes = size_t( S ) * stage * sizeof( T );
};
constexpr int kZWarps     = kZTileY;
// Two producer warps (load l is issued by producer l % 2): one warp's issue and hand-off chain per
// slice load is what limits a single-producer ring (measured on B200: 0.163 -> 0.136 ms for the
// level-8 cube apply in FP64, 0.154 -> 0.108 ms in FP32).
constexpr int kZProducers = 2;
constexpr int kZThreads   = ( kZWarps + kZProducers ) * 32;  // consumer warps + producer warps


// producer warp: streams the rows of every slice of the block's units into the ring.  Lane r < 10
// copies source row y0-1+r; with AUX, lane 10+r copies row y0+r of the second vector (slices
// z_first..z_last only, rows with interior points only).  Row offsets advance by additions from
// slice to slice: cidx(0, y, z+1) = cidx(0, y, z) + tri(n+1-z) - y.
template < typename T, bool AUX >
__device__ __forceinline__ void zstream_produce( const LevelView& v, uint32_t flag, const T* __restrict__ src,
                                                 const T* __restrict__ aux, int nC, T* ring, uint64_t* full, uint64_t* empty,
                                                 uint32_t* shw, volatile int* abort_flag, int* err )
{
   using Cfg = ZCfg< T, AUX >;
   constexpr int S = Cfg::S, AL = Cfg::al, kZTileX = Cfg::kZTileX;
   static_assert( S % kZProducers == 0, "every stage must belong to one producer warp" );
   const int     lane = threadIdx.x & 31, n = v.n, me = ( threadIdx.x >> 5 ) - kZWarps;
   const int*    zb = v.zbegin;
   const int4*   zu = v.zunits;
   const int*    zcl = v.zcell;
   const int     u0 = zb[blockIdx.x], u1 = zb[blockIdx.x + 1];
   const bool    is_src = lane < Cfg::rows, is_aux = AUX && lane >= Cfg::rows && lane < Cfg::rows + kZTileY;
   const int     dsto   = is_src ? lane * Cfg::RW : Cfg::aux0 + ( lane - Cfg::rows ) * Cfg::RWA;
   const T*      gbase  = is_src ? src : aux;
   const int     shbit  = is_src ? 3 * lane : ( is_aux ? 3 * ( lane - Cfg::rows ) : 0 );
   int           ld = 0;  // sequence number of the next slice load
   bool          ok = true;
   {
      for ( int u = u0; u < u1 && ok; ++u )
      {
         const int c = zcl[u];
         if ( c >= nC || !( v.cell_bc[c] & flag ) ) continue;
         const int64_t cb = v.cell_off[c];
         const int4 U  = zu[u];  // x0 (| half-width flag), y0, z_first, z_last
         const int  ux = U.x & kSwUnitXMask, tw = ( U.x & kSwUnitHalf ) ? kZTileX / 2 : kZTileX;
         const int  yy = is_src ? U.y - 1 + lane : U.y + ( lane - Cfg::rows );
         const int  xa = is_src ? ux - 1 : ux;  // first x of the row segment
         int64_t    rb = cidx( n, 0, yy, U.z - 1 );
         for ( int zz = U.z - 1; zz <= U.w + 1; rb += slice_step( n, zz ) - yy, ++zz, ++ld )
         {
            if ( ld % kZProducers != me ) continue;
            const int st = ld % S;
            if ( ld >= S && !mbar_wait_bounded( &empty[st], uint32_t( ( ld / S - 1 ) & 1 ), abort_flag ) )
            {
               ok = false;
               break;
            }
            uint32_t bytes = 0, sh = 0;
            int64_t  a0    = 0;
            // last x of the segment: the halo point (source) or the last interior point (second vector)
            const int  xe   = is_src ? min( ux + tw, n - yy - zz ) : min( ux + tw - 1, n - 1 - yy - zz );
            const bool live = ( is_src && yy + zz <= n && xe >= xa ) || ( is_aux && zz >= U.z && zz <= U.w && xe >= xa );
            if ( live )
            {
               const int64_t s0 = rb + xa;
               const int64_t e1 = rb + xe + 1;  // one past the segment
               sh               = uint32_t( s0 & ( AL - 1 ) );
               a0               = s0 - sh;
               bytes            = uint32_t( ( ( e1 + AL - 1 ) / AL * AL - a0 ) * int64_t( sizeof( T ) ) );
            }
            const uint32_t total = __reduce_add_sync( 0xffffffffu, bytes );
            const uint32_t w0    = __reduce_or_sync( 0xffffffffu, is_src ? sh << shbit : 0u );
            const uint32_t w1    = AUX ? __reduce_or_sync( 0xffffffffu, is_aux ? sh << shbit : 0u ) : 0u;
            if ( lane == 0 )
            {
               shw[2 * st]     = w0;
               shw[2 * st + 1] = w1;
               mbar_expect_tx( &full[st], total );
            }
            __syncwarp();
            if ( bytes ) bulk_copy_g2s( ring + st * Cfg::stage + dsto, gbase + cb + a0, bytes, &full[st] );
         }
      }
   }
   if ( !ok && lane == 0 )
   {
      atomicExch( err, 1 );
      *abort_flag = 1;
   }
   // drain: the latest load issued on every stage has landed before the block may exit
   if ( lane == 0 )
      for ( int s = me; s < S && s < ld; s += kZProducers )
      {
         const int j = s + ( ( ld - 1 - s ) / S ) * S;
         if ( !mbar_wait_bounded( &full[s], uint32_t( ( j / S ) & 1 ), nullptr ) ) atomicExch( err, 1 );
      }
}

// the eight values of one point that roll over from one slice step to the next
template < typename A >
struct ZPoint
{
   A B, BE, BN, BNW;  // slice z-1: (x,y), (x+1,y), (x,y+1), (x-1,y+1)
   A C, W, S, SE;     // slice z:   (x,y), (x-1,y), (x,y-1), (x+1,y-1)
};

template < typename T, typename A, int OP >
__global__ void __launch_bounds__( kZThreads, 2 ) k_cell_zstream( LevelView v, OpView< A > o, uint32_t flag, const T* __restrict__ src,
                                                                  const T* __restrict__ v1, T* v2, T* dst, A a0, A a1, int nC,
                                                                  int* err )
{
   constexpr bool AUX = sweep_aux< OP >();
   using Cfg          = ZCfg< T, AUX >;
   constexpr int S = Cfg::S, RW = Cfg::RW;
   extern __shared__ __align__( 128 ) unsigned char zs_raw[];
   T*                  ring = reinterpret_cast< T* >( zs_raw );
   __shared__ uint64_t full[S], empty[S];
   __shared__ uint32_t shw[2 * S];
   __shared__ A        wsm[kZWarps][16];  // per consumer warp: the cell's 15 weights and 1/diagonal
   __shared__ int      abort_flag;
   const int           warp = threadIdx.x >> 5, lane = threadIdx.x & 31, n = v.n;
   if ( threadIdx.x == 0 )
   {
      for ( int s = 0; s < S; ++s )
      {
         mbar_init( &full[s], 1 );
         mbar_init( &empty[s], kZWarps );
      }
      abort_flag = 0;
      asm volatile( "fence.mbarrier_init.release.cluster;" ::: "memory" );
   }
   __syncthreads();
   volatile int* abrt = &abort_flag;
   if ( warp >= kZWarps )
   {
      const T* aux = ( OP == OP_CHEBI || OP == OP_CHEBL ) ? v2 : ( OP == OP_APPLY_ADD ? dst : v1 );
      zstream_produce< T, AUX >( v, flag, src, aux, nC, ring, full, empty, shw, abrt, err );
      return;
   }

   // consumer warp `warp` owns tile row y0 + warp; stage row r holds global row y0 - 1 + r; lane
   // owns x = x0 + lane + 32 k, k < kZPts
   constexpr int kZPts = Cfg::pts;
   const int*    zb    = v.zbegin;
   const int4*   zu    = v.zunits;
   const int*    zcl   = v.zcell;
   const int     u0 = zb[blockIdx.x], u1 = zb[blockIdx.x + 1];
   const int rS = warp, rC = warp + 1, rN = warp + 2;  // rows y-1, y, y+1 of the stage
   auto at = [&]( const T* st, uint32_t word, int r, int k, int dx ) -> A {
      return A( st[r * RW + int( ( word >> ( 3 * r ) ) & 7u ) + lane + 32 * k + 1 + dx] );
   };
   auto fail = [&]() {
      if ( lane == 0 )
      {
         atomicExch( err, 1 );
         *abrt = 1;
      }
   };
   int ld = 0;
   // the weights are read from shared memory at every use (broadcast, shared by the lane's points)
   // rather than held in 30 registers
   A* w = wsm[warp];
   int cw = -1;  // cell whose weights are in w
   {
      for ( int u = u0; u < u1; ++u )
      {
         const int c = zcl[u];
         if ( c >= nC || !( v.cell_bc[c] & flag ) ) continue;
         const int64_t base = v.cell_off[c];
         if ( c != cw )
         {
            __syncwarp();
            if ( lane < kNumDirs ) w[lane] = o.W[size_t( c ) * kNumClasses * kNumDirs + lane];  // interior class 0
            if ( lane == kNumDirs ) w[kNumDirs] = o.invd_c[c];
            __syncwarp();
            cw = c;
         }
         const int4 U    = zu[u];
         const int  x0   = U.x & kSwUnitXMask;
         const bool half = ( U.x & kSwUnitHalf ) != 0;  // the tile's rows end within 32 points
         const int  x = x0 + lane, y = U.y + warp;
         // one unit with KP points per lane (kZPts, or 1 for half-width units)
         auto unit = [&]( auto kp_c ) -> bool {
            constexpr int KP = decltype( kp_c )::value;
            // prologue: slice z_first-1 (load ld) and slice z_first (load ld+1)
            const int sm = ld % S, s0 = ( ld + 1 ) % S;
            if ( !mbar_wait_bounded( &full[sm], uint32_t( ( ld / S ) & 1 ), abrt ) ||
                 !mbar_wait_bounded( &full[s0], uint32_t( ( ( ld + 1 ) / S ) & 1 ), abrt ) )
               return false;
            ZPoint< A > P[KP];
            {
               const T*       Rm = ring + sm * Cfg::stage;
               const T*       R0 = ring + s0 * Cfg::stage;
               const uint32_t wm = shw[2 * sm], wc = shw[2 * s0];
   #pragma unroll
               for ( int k = 0; k < KP; ++k )
               {
                  P[k].B   = at( Rm, wm, rC, k, 0 );
                  P[k].BE  = at( Rm, wm, rC, k, 1 );
                  P[k].BN  = at( Rm, wm, rN, k, 0 );
                  P[k].BNW = at( Rm, wm, rN, k, -1 );
                  P[k].C   = at( R0, wc, rC, k, 0 );
                  P[k].W   = at( R0, wc, rC, k, -1 );
                  P[k].S   = at( R0, wc, rS, k, 0 );
                  P[k].SE  = at( R0, wc, rS, k, 1 );
               }
            }
            __syncwarp();
            if ( lane == 0 ) mbar_arrive( &empty[sm] );
            int64_t out = base + cidx( n, x, y, U.z );  // output offset of point k = 0, advanced per slice
            // unrolled by two so that the rolled values alternate registers instead of being copied
   #pragma unroll 2
            for ( int z = U.z; z <= U.w; out += slice_step( n, z ) - y, ++z )
            {
               const int lz = ld + 1 + ( z - U.z ), lp = lz + 1;
               const int sz = lz % S, sp = lp % S;
               if ( !mbar_wait_bounded( &full[sp], uint32_t( ( lp / S ) & 1 ), abrt ) ) return false;
               const T*       Rz = ring + sz * Cfg::stage;
               const T*       Rp = ring + sp * Cfg::stage;
               const uint32_t wz = shw[2 * sz], wp = shw[2 * sp];
               const uint32_t wa = AUX ? shw[2 * sz + 1] : 0u;
   #pragma unroll
               for ( int k = 0; k < KP; ++k )
               {
                  const A E = at( Rz, wz, rC, k, 1 ), N = at( Rz, wz, rN, k, 0 ), NW = at( Rz, wz, rN, k, -1 );
                  const A Tt = at( Rp, wp, rC, k, 0 ), TW = at( Rp, wp, rC, k, -1 ), TS = at( Rp, wp, rS, k, 0 ),
                          TSE = at( Rp, wp, rS, k, 1 );
                  ZPoint< A >& p = P[k];
                  if ( x + 32 * k + y + z <= n - 1 )
                  {
                     A auxv = A( 0 );
                     if constexpr ( AUX )
                        auxv = A( Rz[Cfg::aux0 + warp * Cfg::RWA + int( ( wa >> ( 3 * warp ) ) & 7u ) + lane + 32 * k] );
                     // three independent partial sums: the dependent FMA chain is 7 deep instead of 15
                     A s0 = w[0] * p.C, s1 = w[5] * p.B, s2 = w[10] * p.BE;
                     s0 += w[1] * p.W;
                     s1 += w[6] * Tt;
                     s2 += w[11] * TS;
                     s0 += w[2] * E;
                     s1 += w[7] * NW;
                     s2 += w[12] * p.BN;
                     s0 += w[3] * p.S;
                     s1 += w[8] * p.SE;
                     s2 += w[13] * TSE;
                     s0 += w[4] * N;
                     s1 += w[9] * TW;
                     s2 += w[14] * p.BNW;
                     const A acc = s0 + ( s1 + s2 );
                     sweep_epilogue< T, A, OP >( out + 32 * k, acc, w[kNumDirs], p.C, auxv, v2, dst, a0, a1 );
                  }
                  p.B   = p.C;
                  p.BE  = E;
                  p.BN  = N;
                  p.BNW = NW;
                  p.C   = Tt;
                  p.W   = TW;
                  p.S   = TS;
                  p.SE  = TSE;
               }
               __syncwarp();
               if ( lane == 0 ) mbar_arrive( &empty[sz] );
            }
            // slice z_last+1 is no longer needed either
            __syncwarp();
            if ( lane == 0 ) mbar_arrive( &empty[( ld + 2 + ( U.w - U.z ) ) % S] );
            return true;
         };
         const bool good = half ? unit( std::integral_constant< int, 1 >{} ) : unit( std::integral_constant< int, kZPts >{} );
         if ( !good ) return fail();
         ld += U.w - U.z + 3;
      }
   }
}

template < typename T, typename A, int OP >
static void sweep_attribute( int sms )
{
   if constexpr ( sweep_aux< OP >() )
   {
      check_cuda( cudaFuncSetAttribute( k_cell_zstream< T, A, OP >, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        int( ZCfg< T, true >::smem_bytes ) ),
                  "cudaFuncSetAttribute(rolled sweep shared memory)" );
   }
   else
   {
      using Cfg = SwCfg< T, OP >;
      check_cuda( cudaFuncSetAttribute( k_cell_sweep< T, A, OP >, cudaFuncAttributeMaxDynamicSharedMemorySize, int( Cfg::smem_bytes ) ),
                  "cudaFuncSetAttribute(cell sweep shared memory)" );
      int nb = 0;
      check_cuda( cudaOccupancyMaxActiveBlocksPerMultiprocessor( &nb, k_cell_sweep< T, A, OP >, kSwWarps * 32, Cfg::smem_bytes ),
                  "cell sweep occupancy" );
      // the unit lists assume every block of the launch is resident at once
      if ( nb < Cfg::BPS )
         throw std::runtime_error( "cell sweep: " + std::to_string( nb ) + " resident blocks per SM, the unit lists need " +
                                   std::to_string( Cfg::BPS ) );
   }
   (void) sms;
}

template < typename T, typename A >
static void sweep_attributes( int sms )
{
   sweep_attribute< T, A, OP_APPLY >( sms );
   sweep_attribute< T, A, OP_APPLY_ADD >( sms );
   sweep_attribute< T, A, OP_RESID >( sms );
   sweep_attribute< T, A, OP_JAC >( sms );
   sweep_attribute< T, A, OP_CHEB0 >( sms );
   sweep_attribute< T, A, OP_CHEBI >( sms );
   sweep_attribute< T, A, OP_CHEBL >( sms );
   sweep_attribute< T, A, OP_DINV_APPLY >( sms );
}

static void sweep_attributes_all()
{
   int dev = 0, sms = 0;
   check_cuda( cudaGetDevice( &dev ), "cudaGetDevice" );
   check_cuda( cudaDeviceGetAttribute( &sms, cudaDevAttrMultiProcessorCount, dev ), "device attribute" );
   sweep_attributes< double, double >( sms );
   sweep_attributes< float, float >( sms );
   sweep_attributes< __half, float >( sms );
}


// Stencil of one position class at cell-local (x, y, z): the 15 directions are unrolled with the
// seven row bases derived from the point's own row by additions (row y of slice z holds n+1-z-y
// points, slice z holds tri(n+1-z) points), so all loads of a point are independent and in flight
// together.  Bases of directions outside the cell are never used: the class mask skips them.
// class_stencil returns the sum; class_stencil_at also returns the cell-array offset of the point.
template < typename A >
struct StencilAt
{
   A       sum;
   int64_t centre;
};

template < typename T, typename A >
__device__ __forceinline__ StencilAt< A > class_stencil_at( const T* s, const A* W, uint16_t mask, int n, int x, int y, int z )
{
   const int64_t r00 = cidx( n, 0, y, z );
   const int64_t ly  = n + 1 - z - y;                      // points in row y of slice z
   const int64_t tz  = int64_t( n + 1 - z ) * ( n + 2 - z ) / 2;  // points in slice z
   const int64_t rm0 = r00 - ( ly + 1 );                  // row y-1 of slice z
   const int64_t rp0 = r00 + ly;                          // row y+1 of slice z
   const int64_t r0p = r00 + tz - y;                      // row y of slice z+1
   const int64_t r0m = r00 - ( tz + ( n + 2 - z ) - y );  // row y of slice z-1 (slice z-1 holds tz + n+2-z points)
   const int64_t rmp = r0p - ly;                          // row y-1 of slice z+1
   const int64_t rpm = r0m + ly + 1;                      // row y+1 of slice z-1
   const int64_t idx[kNumDirs] = { r00 + x,     r00 + x - 1, r00 + x + 1, rm0 + x,     rp0 + x,
                                   r0m + x,     r0p + x,     rp0 + x - 1, rm0 + x + 1, r0p + x - 1,
                                   r0m + x + 1, rmp + x,     rpm + x,     rmp + x + 1, rpm + x - 1 };
   A acc = A( 0 );
#pragma unroll
   for ( int d = 0; d < kNumDirs; ++d )
      if ( mask & ( 1u << d ) ) acc += W[d] * A( ldv( s + idx[d] ) );
   return { acc, r00 + x };
}

// the same sum for a point given by its slot c in the level buffer (cell offset included) and its row
// y and slice z in the cell: the neighbours are c plus offsets that depend on y and z only
template < typename T, typename A >
__device__ __forceinline__ A class_stencil_slot( const T* src, const A* W, uint16_t mask, int n, int64_t c, int y, int z )
{
   const int64_t ly  = n + 1 - z - y;
   const int64_t tz  = int64_t( n + 1 - z ) * ( n + 2 - z ) / 2;
   const int64_t dm0 = -( ly + 1 ), dp0 = ly, d0p = tz - y, d0m = -( tz + ( n + 2 - z ) - y );
   const int64_t dmp = d0p - ly, dpm = d0m + ly + 1;
   const int64_t idx[kNumDirs] = { c,           c - 1,       c + 1,       c + dm0,     c + dp0,
                                   c + d0m,     c + d0p,     c + dp0 - 1, c + dm0 + 1, c + d0p - 1,
                                   c + d0m + 1, c + dmp,     c + dpm,     c + dmp + 1, c + dpm - 1 };
   A acc = A( 0 );
#pragma unroll
   for ( int d = 0; d < kNumDirs; ++d )
      if ( mask & ( 1u << d ) ) acc += W[d] * A( ldv( src + idx[d] ) );
   return acc;
}

template < typename T, typename A >
__device__ __forceinline__ A class_stencil( const T* s, const A* W, uint16_t mask, int n, int x, int y, int z )
{
   return class_stencil_at< T, A >( s, W, mask, n, x, y, z ).sum;
}

// One owned face / edge / vertex DoF (boundary task t): the sum over its neighbour cells of the
// stencil of its position class in each cell, the operation's epilogue, and the write to the owner
// and every copy in the neighbouring cell arrays.
template < typename T, typename A, int OP >
__device__ __forceinline__ void bnd_task( const LevelView& v, const OpView< A >& o, uint32_t flag, int copy_unflagged,
                                          const T* __restrict__ src, const T* __restrict__ v1, T* v2, T* dst, A a0, A a1, int4 tk )
{
   const int     b     = tk.x, i = tk.y, j = tk.z, n = v.n;
   const int64_t owner = owner_slot( v, b, i, j );
   if ( !( v.bc[b] & flag ) )
   {
      if ( !copy_unflagged ) return;
      if constexpr ( OP == OP_JAC || OP == OP_CHEB0 ) write_through( v, dst, b, i, j, owner, A( ldv( src + owner ) ) );
      else if constexpr ( OP == OP_CHEBI ) write_through( v, dst, b, i, j, owner, A( ldc( v2 + owner ) ) );
      return;
   }
   A         acc = A( 0 );
   const int q0 = v.inc_begin[b], q1 = v.inc_begin[b + 1];
   if ( q1 - q0 == 2 )
   {
      // a face between two cells: both class stencils written out, so the loads of the two cells
      // are in flight together (same sum, same order as the loop); the copies of the owner in the
      // two cell arrays are the stencils' centres
      const Incidence I0 = v.inc[q0], I1 = v.inc[q0 + 1];
      int             x0, y0, z0, x1, y1, z1;
      inc_point( I0, n, i, j, x0, y0, z0 );
      inc_point( I1, n, i, j, x1, y1, z1 );
      const int64_t         cb0 = v.cell_off[I0.cell], cb1 = v.cell_off[I1.cell];
      const StencilAt< A >  s0  = class_stencil_at< T, A >( src + cb0, o.W + ( size_t( I0.cell ) * kNumClasses + I0.cls ) * kNumDirs,
                                                           c_cls_mask[I0.cls], n, x0, y0, z0 );
      const StencilAt< A >  s1  = class_stencil_at< T, A >( src + cb1, o.W + ( size_t( I1.cell ) * kNumClasses + I1.cls ) * kNumDirs,
                                                           c_cls_mask[I1.cls], n, x1, y1, z1 );
      const int64_t         c0 = s0.centre, c1 = s1.centre;
      acc                       = ( acc + s0.sum ) + s1.sum;
      const A invd = o.invd_b[b];
      auto    put  = [&]( T* vec, A val ) {
         stv( vec + owner, val );
         stv( vec + cb0 + c0, val );
         stv( vec + cb1 + c1, val );
      };
      if constexpr ( OP == OP_APPLY ) put( dst, acc );
      else if constexpr ( OP == OP_APPLY_ADD ) put( dst, A( ldc( dst + owner ) ) + acc );
      else if constexpr ( OP == OP_RESID ) put( dst, A( ldv( v1 + owner ) ) - acc );
      else if constexpr ( OP == OP_JAC ) put( dst, A( ldv( src + owner ) ) + a0 * ( invd * ( A( ldv( v1 + owner ) ) - acc ) ) );
      else if constexpr ( OP == OP_CHEB0 ) put( dst, invd * ( A( ldv( v1 + owner ) ) - acc ) );
      else if constexpr ( OP == OP_CHEBI )
      {
         put( dst, invd * acc );
         put( v2, A( ldc( v2 + owner ) ) + a0 * A( ldv( src + owner ) ) );
      }
      else if constexpr ( OP == OP_CHEBL ) put( v2, ( A( ldc( v2 + owner ) ) + a0 * A( ldv( src + owner ) ) ) + a1 * ( invd * acc ) );
      else if constexpr ( OP == OP_DINV_APPLY ) put( dst, invd * acc );
      return;
   }
   else
      // edges and vertices: two incidences' stencils in flight, summed in incidence order
      for ( int q = q0; q < q1; q += 2 )
      {
         A sq[2];
#pragma unroll
         for ( int u = 0; u < 2; ++u )
         {
            sq[u] = A( 0 );
            if ( q + u < q1 )
            {
               const Incidence I = v.inc[q + u];
               int             x, y, z;
               inc_point( I, n, i, j, x, y, z );
               sq[u] = class_stencil< T, A >( src + v.cell_off[I.cell], o.W + ( size_t( I.cell ) * kNumClasses + I.cls ) * kNumDirs,
                                              c_cls_mask[I.cls], n, x, y, z );
            }
         }
         acc += sq[0];
         if ( q + 1 < q1 ) acc += sq[1];
      }
   const A invd = o.invd_b[b];
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

// threads per block of the boundary kernel
constexpr int kBndThreads = 256;

template < typename T, typename A, int OP >
__global__ void __launch_bounds__( kBndThreads ) k_bnd_stencil( LevelView v, OpView< A > o, TaskSegments seg, uint32_t flag, int copy_unflagged,
                                                         const T* __restrict__ src, const T* __restrict__ v1, T* v2, T* dst,
                                                         A a0, A a1 )
{
   // tasks of the primitives whose boundary type is flagged (or all, when unflagged owners are
   // copied): up to four contiguous groups of the type-sorted task list
   int t = blockIdx.x * blockDim.x + threadIdx.x, at = -1;
#pragma unroll
   for ( int g = 0; g < 4; ++g )  // unrolled: the segment arrays are read with constant indices
   {
      if ( at < 0 && t < seg.count[g] ) at = seg.start[g] + t;
      if ( at < 0 ) t -= seg.count[g];
   }
   if ( at < 0 ) return;
   // a flagged face point between two cells: everything the stencil needs comes from one record,
   // so the value loads follow a single dependent load (the same sums, in the same order, as bnd_task)
   const FaceRec r = v.frec[at];
   if ( r.cell0 >= 0 && ( r.bc & flag ) )
   {
      const A s0 = class_stencil_slot< T, A >( src, o.W + ( size_t( r.cell0 ) * kNumClasses + r.cls0 ) * kNumDirs, c_cls_mask[r.cls0], v.n,
                                              r.c0, r.y0, r.z0 );
      const A s1 = class_stencil_slot< T, A >( src, o.W + ( size_t( r.cell1 ) * kNumClasses + r.cls1 ) * kNumDirs, c_cls_mask[r.cls1], v.n,
                                              r.c1, r.y1, r.z1 );
      const A acc  = ( A( 0 ) + s0 ) + s1;
      const A invd = o.invd_b[r.b];
      auto    put  = [&]( T* vec, A val ) {
         stv( vec + r.owner, val );
         stv( vec + r.c0, val );
         stv( vec + r.c1, val );
      };
      if constexpr ( OP == OP_APPLY ) put( dst, acc );
      else if constexpr ( OP == OP_APPLY_ADD ) put( dst, A( ldc( dst + r.owner ) ) + acc );
      else if constexpr ( OP == OP_RESID ) put( dst, A( ldv( v1 + r.owner ) ) - acc );
      else if constexpr ( OP == OP_JAC ) put( dst, A( ldv( src + r.owner ) ) + a0 * ( invd * ( A( ldv( v1 + r.owner ) ) - acc ) ) );
      else if constexpr ( OP == OP_CHEB0 ) put( dst, invd * ( A( ldv( v1 + r.owner ) ) - acc ) );
      else if constexpr ( OP == OP_CHEBI )
      {
         put( dst, invd * acc );
         put( v2, A( ldc( v2 + r.owner ) ) + a0 * A( ldv( src + r.owner ) ) );
      }
      else if constexpr ( OP == OP_CHEBL ) put( v2, ( A( ldc( v2 + r.owner ) ) + a0 * A( ldv( src + r.owner ) ) ) + a1 * ( invd * acc ) );
      else if constexpr ( OP == OP_DINV_APPLY ) put( dst, invd * acc );
      return;
   }
   bnd_task< T, A, OP >( v, o, flag, copy_unflagged, src, v1, v2, dst, a0, a1, v.btasks[at] );
}

template < typename T, typename A, int OP >
static void run_stencil( Context* ctx, const LevelView& v, const OpView< A >& o, int nC, const StencilArgs& a )
{
   const T* src = (const T*) a.src;
   const T* v1  = (const T*) a.v1;
   T*       v2  = (T*) a.v2;
   T*       dst = (T*) a.dst;
   // the bulk-copy sweep from n = 32 on (two 64-point tiles per row and up), the y-marching sweep on
   // the small levels, where a slice holds too few rows to fill a ring
   using Cfg = SwCfg< T, OP >;
   // cell interiors and boundary owners write disjoint slots and read only src (and their own
   // slots of the second vector), so the two kernels may run in either order
   const TaskSegments seg = task_segments( v, a.flag, a.copy_unflagged );
   const int          nt  = seg.count[0] + seg.count[1] + seg.count[2] + seg.count[3];
   // the partial-sum sweep for the operations without a second vector, the rolled-register sweep
   // for the others (their epilogues' registers would leave the partial-sum sweep 8 warps per SM)
   constexpr bool ROLLED = sweep_aux< OP >();
   const bool     big    = v.n >= 32 && nC > 0 && ( ROLLED ? v.nzblocks > 0 : v.nswarps[Cfg::BPS - 2] > 0 );
   auto           cell   = [&]() {
      if constexpr ( ROLLED )
      {
         constexpr size_t smem = ZCfg< T, true >::smem_bytes;  // attribute set by ensure_constants
         k_cell_zstream< T, A, OP ><<< v.nzblocks, kZThreads, smem, ctx->stream >>>( v, o, a.flag, src, v1, v2, dst, A( a.a0 ),
                                                                                    A( a.a1 ), nC, ctx->d_error );
      }
      else
         k_cell_sweep< T, A, OP ><<< v.nswarps[Cfg::BPS - 2] / kSwWarps, kSwWarps * 32, Cfg::smem_bytes, ctx->stream >>>(
             v, o, a.flag, src, v1, v2, dst, A( a.a0 ), A( a.a1 ), nC, ctx->d_error );
      ++ctx->launches;
   };
   cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
   check_cuda( cudaStreamIsCapturing( ctx->stream, &cap ), "cudaStreamIsCapturing" );
   if ( big && cap == cudaStreamCaptureStatusNone )
   {
      // Launched one by one, the boundary kernel goes first on the same stream: the sweep occupies
      // every SM's registers, so a forked boundary kernel would only wait for it and add the latency of
      // two cross-stream dependencies.  In a captured graph the fork below becomes two parallel
      // branches, and the boundary kernel fills the SMs the sweep's last blocks leave idle.
      if ( nt > 0 )
      {
         k_bnd_stencil< T, A, OP ><<< ( nt + kBndThreads - 1 ) / kBndThreads, kBndThreads, 0, ctx->stream >>>( v, o, seg, a.flag, a.copy_unflagged, src, v1, v2, dst,
                                                                                   A( a.a0 ), A( a.a1 ) );
         ++ctx->launches;
      }
      cell();
      check_cuda( cudaGetLastError(), "stencil launch" );
      return;
   }
   // the cell kernel and the boundary kernel side by side on two streams
   Fork fk( ctx );
   if ( big ) cell();
   else if ( v.nmarch > 0 && nC > 0 )
   {
      dim3 grid( ( v.nmarch + 7 ) / 8, nC );
      k_cell_march< T, A, OP ><<< grid, 256, 0, ctx->stream >>>( v, o, a.flag, src, v1, v2, dst, A( a.a0 ), A( a.a1 ) );
      ++ctx->launches;
   }
   if ( nt > 0 )
   {
      k_bnd_stencil< T, A, OP ><<< ( nt + kBndThreads - 1 ) / kBndThreads, kBndThreads, 0, fk.aux() >>>( v, o, seg, a.flag, a.copy_unflagged, src, v1, v2, dst,
                                                                             A( a.a0 ), A( a.a1 ) );
      ++ctx->launches;
   }
   check_cuda( cudaGetLastError(), "stencil launch" );
}

template < typename T, typename A >
static void dispatch_stencil( Context* ctx, const LevelView& v, const OpView< A >& o, int nC, const StencilArgs& a )
{
   switch ( a.op )
   {
   case OP_APPLY: run_stencil< T, A, OP_APPLY >( ctx, v, o, nC, a ); break;
   case OP_APPLY_ADD: run_stencil< T, A, OP_APPLY_ADD >( ctx, v, o, nC, a ); break;
   case OP_RESID: run_stencil< T, A, OP_RESID >( ctx, v, o, nC, a ); break;
   case OP_JAC: run_stencil< T, A, OP_JAC >( ctx, v, o, nC, a ); break;
   case OP_CHEB0: run_stencil< T, A, OP_CHEB0 >( ctx, v, o, nC, a ); break;
   case OP_CHEBI: run_stencil< T, A, OP_CHEBI >( ctx, v, o, nC, a ); break;
   case OP_CHEBL: run_stencil< T, A, OP_CHEBL >( ctx, v, o, nC, a ); break;
   case OP_DINV_APPLY: run_stencil< T, A, OP_DINV_APPLY >( ctx, v, o, nC, a ); break;
   default: throw std::invalid_argument( "unknown stencil op" );
   }
}

void launch_stencil( Context* ctx, Mesh* m, Operator* Op, int L, int dtype, const StencilArgs& a )
{
   ensure_constants();
   if ( Op->elementwise )
   {
      launch_elementwise( ctx, m, Op, L, dtype, a );
      return;
   }
   if ( Op->kind == HYB_P2_CONST_LAPLACE )
   {
      launch_p2_constant( ctx, m, Op, L, dtype, a );
      return;
   }
   LevelView v  = make_view( m, L );
   OpLevel&  ol = Op->lv.at( L );
   ensure_device_op( ol );
   const int nC = m->topo.nC;
   if ( dtype == F64 )
      dispatch_stencil< double, double >( ctx, v, OpView< double >{ ol.d_W, ol.d_invd_b, ol.d_invd_c }, nC, a );
   else if ( dtype == F32 )
      dispatch_stencil< float, float >( ctx, v, OpView< float >{ ol.d_Wf, ol.d_invd_bf, ol.d_invd_cf }, nC, a );
   else
      dispatch_stencil< __half, float >( ctx, v, OpView< float >{ ol.d_Wf, ol.d_invd_bf, ol.d_invd_cf }, nC, a );
}

// ---------------------------------------------------------------------------------------------
// pointwise operations on owned DoFs
// ---------------------------------------------------------------------------------------------
template < typename T, typename A, int OP >
__device__ __forceinline__ A point_value( int64_t i, int nsrc, const T* s0, const T* s1, const T* s2, const T* dst, A a0, A a1, A a2 )
{
   if constexpr ( OP == PT_LINCOMB || OP == PT_ADD )
   {
      A r = a0 * A( ldc( s0 + i ) );
      if ( nsrc > 1 ) r += a1 * A( ldc( s1 + i ) );
      if ( nsrc > 2 ) r += a2 * A( ldc( s2 + i ) );
      if constexpr ( OP == PT_ADD ) r = A( ldc( dst + i ) ) + r;
      return r;
   }
   else if constexpr ( OP == PT_MULT ) return A( ldc( s0 + i ) ) * A( ldc( s1 + i ) );
   else if constexpr ( OP == PT_INVERT ) return A( 1 ) / A( ldc( s0 + i ) );
   else if constexpr ( OP == PT_SET ) return a0;
   else if constexpr ( OP == PT_SYNC ) return A( ldc( dst + i ) );
   return A( 0 );
}

template < typename T, typename A, int OP >
__global__ void __launch_bounds__( 256 ) k_cell_point( LevelView v, uint32_t flag, int nsrc, const T* s0, const T* s1, const T* s2,
                                                        T* dst, A a0, A a1, A a2, const double* sc )
{
   const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
   const int r    = blockIdx.x * 8 + warp;
   const int c    = blockIdx.y;
   if ( r >= v.nrows ) return;
   if ( !( v.cell_bc[c] & flag ) ) return;
   if constexpr ( OP == PT_CG_XR || OP == PT_CG_P )
      if ( sc[6] != 0.0 ) return;
   const int2    yz   = v.rows[r];
   const int64_t base = v.cell_off[c] + cidx( v.n, 0, yz.x, yz.y );
   const int     xmax = v.n - 1 - yz.x - yz.y;
   for ( int x = 1 + lane; x <= xmax; x += 32 )
   {
      const int64_t i = base + x;
      if constexpr ( OP == PT_CG_XR )
      {
         const double alpha = sc[4];
         stv( (T*) s0 + i, A( ldc( s0 + i ) ) + A( alpha ) * A( ldc( s1 + i ) ) );
         stv( dst + i, A( ldc( dst + i ) ) - A( alpha ) * A( ldc( s2 + i ) ) );
      }
      else if constexpr ( OP == PT_CG_P )
      {
         const double beta = sc[5];
         stv( dst + i, A( ldc( s0 + i ) ) + A( beta ) * A( ldc( dst + i ) ) );
      }
      else
         stv( dst + i, point_value< T, A, OP >( i, nsrc, s0, s1, s2, dst, a0, a1, a2 ) );
   }
}

template < typename T, typename A, int OP >
__global__ void __launch_bounds__( 256 ) k_bnd_point( LevelView v, uint32_t flag, int nsrc, const T* s0, const T* s1, const T* s2,
                                                       T* dst, A a0, A a1, A a2, const double* sc )
{
   const int t = blockIdx.x * blockDim.x + threadIdx.x;
   if ( t >= v.ntasks ) return;
   const int4 tk = v.tasks[t];
   const int  b = tk.x, i = tk.y, j = tk.z;
   if ( !( v.bc[b] & flag ) ) return;
   if constexpr ( OP == PT_CG_XR || OP == PT_CG_P )
      if ( sc[6] != 0.0 ) return;
   const int64_t owner = owner_slot( v, b, i, j );
   if constexpr ( OP == PT_CG_XR )
   {
      const double alpha = sc[4];
      write_through( v, (T*) s0, b, i, j, owner, A( ldc( s0 + owner ) ) + A( alpha ) * A( ldc( s1 + owner ) ) );
      write_through( v, dst, b, i, j, owner, A( ldc( dst + owner ) ) - A( alpha ) * A( ldc( s2 + owner ) ) );
   }
   else if constexpr ( OP == PT_CG_P )
   {
      const double beta = sc[5];
      write_through( v, dst, b, i, j, owner, A( ldc( s0 + owner ) ) + A( beta ) * A( ldc( dst + owner ) ) );
   }
   else
      write_through( v, dst, b, i, j, owner, point_value< T, A, OP >( owner, nsrc, s0, s1, s2, dst, a0, a1, a2 ) );
}

template < typename T, typename A, int OP >
static void run_point( Context* ctx, const LevelView& v, int nC, const PointArgs& a )
{
   Fork fk( ctx );
   if ( v.nrows > 0 && nC > 0 && OP != PT_SYNC )
   {
      dim3 grid( ( v.nrows + 7 ) / 8, nC );
      k_cell_point< T, A, OP ><<< grid, 256, 0, ctx->stream >>>( v, a.flag, a.nsrc, (const T*) a.s0, (const T*) a.s1,
                                                                 (const T*) a.s2, (T*) a.dst, A( a.a0 ), A( a.a1 ), A( a.a2 ),
                                                                 a.dev_scalars );
      ++ctx->launches;
   }
   if ( v.ntasks > 0 )
   {
      k_bnd_point< T, A, OP ><<< ( v.ntasks + 255 ) / 256, 256, 0, fk.aux() >>>(
          v, a.flag, a.nsrc, (const T*) a.s0, (const T*) a.s1, (const T*) a.s2, (T*) a.dst, A( a.a0 ), A( a.a1 ), A( a.a2 ),
          a.dev_scalars );
      ++ctx->launches;
   }
   check_cuda( cudaGetLastError(), "pointwise launch" );
}

template < typename T, typename A >
static void dispatch_point( Context* ctx, const LevelView& v, int nC, const PointArgs& a )
{
   switch ( a.op )
   {
   case PT_LINCOMB: run_point< T, A, PT_LINCOMB >( ctx, v, nC, a ); break;
   case PT_ADD: run_point< T, A, PT_ADD >( ctx, v, nC, a ); break;
   case PT_MULT: run_point< T, A, PT_MULT >( ctx, v, nC, a ); break;
   case PT_INVERT: run_point< T, A, PT_INVERT >( ctx, v, nC, a ); break;
   case PT_SET: run_point< T, A, PT_SET >( ctx, v, nC, a ); break;
   case PT_CG_XR: run_point< T, A, PT_CG_XR >( ctx, v, nC, a ); break;
   case PT_CG_P: run_point< T, A, PT_CG_P >( ctx, v, nC, a ); break;
   case PT_SYNC: run_point< T, A, PT_SYNC >( ctx, v, nC, a ); break;
   default: throw std::invalid_argument( "unknown pointwise op" );
   }
}

void launch_point( Context* ctx, Mesh* m, int L, int dtype, const PointArgs& a )
{
   ensure_constants();
   LevelView v  = make_view( m, L );
   const int nC = m->topo.nC;
   if ( dtype == F64 ) dispatch_point< double, double >( ctx, v, nC, a );
   else if ( dtype == F32 ) dispatch_point< float, float >( ctx, v, nC, a );
   else dispatch_point< __half, float >( ctx, v, nC, a );
}

// whole-buffer linear combination (flag All): every slot, copies included, stays consistent
template < typename T, typename A >
__global__ void k_flat_lincomb( int64_t count, T* dst, int nsrc, const T* s0, const T* s1, const T* s2, A a0, A a1, A a2 )
{
   for ( int64_t i = blockIdx.x * int64_t( blockDim.x ) + threadIdx.x; i < count; i += int64_t( gridDim.x ) * blockDim.x )
   {
      A r = nsrc > 0 ? a0 * A( ldc( s0 + i ) ) : a0;
      if ( nsrc > 1 ) r += a1 * A( ldc( s1 + i ) );
      if ( nsrc > 2 ) r += a2 * A( ldc( s2 + i ) );
      stv( dst + i, r );
   }
}

void launch_flat_lincomb( Context* ctx, int64_t count, int dtype, void* dst, int nsrc, const void* const* srcs, const double* scal )
{
   if ( count <= 0 ) return;
   const int blocks = int( std::min< int64_t >( ( count + 255 ) / 256, 148 * 16 ) );
   const void* s0 = nsrc > 0 ? srcs[0] : nullptr;
   const void* s1 = nsrc > 1 ? srcs[1] : nullptr;
   const void* s2 = nsrc > 2 ? srcs[2] : nullptr;
   if ( dtype == F64 )
      k_flat_lincomb< double, double ><<< blocks, 256, 0, ctx->stream >>>( count, (double*) dst, nsrc, (const double*) s0,
                                                                          (const double*) s1, (const double*) s2, scal[0],
                                                                          scal[1], scal[2] );
   else if ( dtype == F32 )
      k_flat_lincomb< float, float ><<< blocks, 256, 0, ctx->stream >>>( count, (float*) dst, nsrc, (const float*) s0,
                                                                        (const float*) s1, (const float*) s2, float( scal[0] ),
                                                                        float( scal[1] ), float( scal[2] ) );
   else
      k_flat_lincomb< __half, float ><<< blocks, 256, 0, ctx->stream >>>( count, (__half*) dst, nsrc, (const __half*) s0,
                                                                         (const __half*) s1, (const __half*) s2, float( scal[0] ),
                                                                         float( scal[1] ), float( scal[2] ) );
   ++ctx->launches;
   check_cuda( cudaGetLastError(), "flat lincomb launch" );
}

template < typename TD, typename TS >
__global__ void k_convert( int64_t count, TD* dst, const TS* src, double scale )
{
   for ( int64_t i = blockIdx.x * int64_t( blockDim.x ) + threadIdx.x; i < count; i += int64_t( gridDim.x ) * blockDim.x )
   {
      if constexpr ( std::is_same< TD, __half >::value ) dst[i] = __float2half_rn( float( double( ldc( src + i ) ) * scale ) );
      else if constexpr ( std::is_same< TD, float >::value ) dst[i] = float( double( ldc( src + i ) ) * scale );
      else dst[i] = TD( double( ldc( src + i ) ) * scale );
   }
}

// packed index i -> primitive p (largest p with poff[p] <= i) -> padded slot off[p] + (i - poff[p])
template < typename T >
__global__ void k_repack( int64_t count, int np, const int64_t* __restrict__ poff, const int64_t* __restrict__ off, int to_padded,
                          double* packed, T* vec )
{
   for ( int64_t i = blockIdx.x * int64_t( blockDim.x ) + threadIdx.x; i < count; i += int64_t( gridDim.x ) * blockDim.x )
   {
      int lo = 0, hi = np - 1;
      while ( lo < hi )
      {
         const int mid = ( lo + hi + 1 ) >> 1;
         if ( poff[mid] <= i ) lo = mid;
         else hi = mid - 1;
      }
      const int64_t slot = off[lo] + ( i - poff[lo] );
      if ( to_padded )
      {
         if constexpr ( std::is_same< T, __half >::value ) vec[slot] = __float2half_rn( float( packed[i] ) );
         else vec[slot] = T( packed[i] );
      }
      else packed[i] = double( ldc( vec + slot ) );
   }
}

void launch_repack( Context* ctx, Mesh* m, int L, int dtype, int to_padded, double* packed, void* vec )
{
   P1Level& P = m->level( L );
   ensure_device( m, P );
   const int64_t count = P.packed_size;
   if ( count <= 0 ) return;
   const int np     = int( P.off.size() );
   const int blocks = int( std::min< int64_t >( ( count + 255 ) / 256, 148 * 16 ) );
   if ( dtype == F64 ) k_repack< double ><<< blocks, 256, 0, ctx->stream >>>( count, np, P.d_poff, P.d_off, to_padded, packed, (double*) vec );
   else if ( dtype == F32 ) k_repack< float ><<< blocks, 256, 0, ctx->stream >>>( count, np, P.d_poff, P.d_off, to_padded, packed, (float*) vec );
   else k_repack< __half ><<< blocks, 256, 0, ctx->stream >>>( count, np, P.d_poff, P.d_off, to_padded, packed, (__half*) vec );
   ++ctx->launches;
   check_cuda( cudaGetLastError(), "repack launch" );
}

void launch_convert( Context* ctx, int64_t count, int dd, void* dst, int sd, const void* src, double scale )
{
   if ( count <= 0 ) return;
   const int blocks = int( std::min< int64_t >( ( count + 255 ) / 256, 148 * 16 ) );
#define HYB_CONV( TD, TS ) k_convert< TD, TS ><<< blocks, 256, 0, ctx->stream >>>( count, (TD*) dst, (const TS*) src, scale )
   if ( dd == F64 && sd == F64 ) HYB_CONV( double, double );
   else if ( dd == F64 && sd == F32 ) HYB_CONV( double, float );
   else if ( dd == F64 && sd == F16 ) HYB_CONV( double, __half );
   else if ( dd == F32 && sd == F64 ) HYB_CONV( float, double );
   else if ( dd == F32 && sd == F32 ) HYB_CONV( float, float );
   else if ( dd == F32 && sd == F16 ) HYB_CONV( float, __half );
   else if ( dd == F16 && sd == F64 ) HYB_CONV( __half, double );
   else if ( dd == F16 && sd == F32 ) HYB_CONV( __half, float );
   else HYB_CONV( __half, __half );
#undef HYB_CONV
   ++ctx->launches;
   check_cuda( cudaGetLastError(), "convert launch" );
}


// x (fp64) += a * convert(c) over every slot
template < typename TS >
__global__ void k_axpy_to_f64( int64_t count, double* x, const TS* c, double a )
{
   for ( int64_t i = blockIdx.x * int64_t( blockDim.x ) + threadIdx.x; i < count; i += int64_t( gridDim.x ) * blockDim.x )
      x[i] += a * double( ldc( c + i ) );
}

void launch_axpy_to_f64( Context* ctx, int64_t count, double* x, int src_dtype, const void* c, double a )
{
   if ( count <= 0 ) return;
   const int blocks = int( std::min< int64_t >( ( count + 255 ) / 256, 148 * 16 ) );
   if ( src_dtype == F64 ) k_axpy_to_f64< double ><<< blocks, 256, 0, ctx->stream >>>( count, x, (const double*) c, a );
   else if ( src_dtype == F32 ) k_axpy_to_f64< float ><<< blocks, 256, 0, ctx->stream >>>( count, x, (const float*) c, a );
   else k_axpy_to_f64< __half ><<< blocks, 256, 0, ctx->stream >>>( count, x, (const __half*) c, a );
   ++ctx->launches;
   check_cuda( cudaGetLastError(), "axpy launch" );
}

// seeded uniform values in [-1, 1] (splitmix64 of seed and slot index), every slot of a level
template < typename T >
__global__ void k_fill_uniform( int64_t count, T* dst, uint64_t seed )
{
   for ( int64_t i = blockIdx.x * int64_t( blockDim.x ) + threadIdx.x; i < count; i += int64_t( gridDim.x ) * blockDim.x )
   {
      uint64_t z = seed + 0x9E3779B97F4A7C15ull * uint64_t( i + 1 );
      z          = ( z ^ ( z >> 30 ) ) * 0xBF58476D1CE4E5B9ull;
      z          = ( z ^ ( z >> 27 ) ) * 0x94D049BB133111EBull;
      z ^= z >> 31;
      const double u = double( z >> 11 ) * ( 1.0 / 9007199254740992.0 );
      using Acc = typename AccT< T >::type;
      stv( dst + i, Acc( 2.0 * u - 1.0 ) );
   }
}

void launch_fill_uniform( Context* ctx, int64_t count, int dtype, void* dst, uint64_t seed )
{
   if ( count <= 0 ) return;
   const int blocks = int( std::min< int64_t >( ( count + 255 ) / 256, 148 * 16 ) );
   if ( dtype == F64 ) k_fill_uniform< double ><<< blocks, 256, 0, ctx->stream >>>( count, (double*) dst, seed );
   else if ( dtype == F32 ) k_fill_uniform< float ><<< blocks, 256, 0, ctx->stream >>>( count, (float*) dst, seed );
   else k_fill_uniform< __half ><<< blocks, 256, 0, ctx->stream >>>( count, (__half*) dst, seed );
   ++ctx->launches;
   check_cuda( cudaGetLastError(), "fill launch" );
}

// ---------------------------------------------------------------------------------------------
// deterministic dot product over owned flagged DoFs
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ double block_sum( double v )
{
   __shared__ double sh[32];
   for ( int o = 16; o > 0; o >>= 1 ) v += __shfl_down_sync( 0xffffffffu, v, o );
   const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
   if ( lane == 0 ) sh[warp] = v;
   __syncthreads();
   const int nw = ( blockDim.x + 31 ) >> 5;
   v            = ( threadIdx.x < nw ) ? sh[threadIdx.x] : 0.0;
   if ( warp == 0 )
      for ( int o = 16; o > 0; o >>= 1 ) v += __shfl_down_sync( 0xffffffffu, v, o );
   return v;
}

template < typename T >
__global__ void __launch_bounds__( 256 ) k_dot_cells( LevelView v, uint32_t flag, const T* a, const T* b, double* partials )
{
   const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
   const int r    = blockIdx.x * 8 + warp;
   const int c    = blockIdx.y;
   double    acc  = 0.0;
   if ( r < v.nrows && ( v.cell_bc[c] & flag ) )
   {
      const int2    yz   = v.rows[r];
      const int64_t base = v.cell_off[c] + cidx( v.n, 0, yz.x, yz.y );
      const int     xmax = v.n - 1 - yz.x - yz.y;
      for ( int x = 1 + lane; x <= xmax; x += 32 ) acc += double( ldv( a + base + x ) ) * double( ldv( b + base + x ) );
   }
   acc = block_sum( acc );
   if ( threadIdx.x == 0 ) partials[size_t( blockIdx.y ) * gridDim.x + blockIdx.x] = acc;
}

template < typename T >
__global__ void __launch_bounds__( 256 ) k_dot_bnd( LevelView v, uint32_t flag, const T* a, const T* b, double* partials )
{
   const int t   = blockIdx.x * blockDim.x + threadIdx.x;
   double    acc = 0.0;
   if ( t < v.ntasks )
   {
      const int4 tk = v.tasks[t];
      if ( tk.x >= 0 && ( v.bc[tk.x] & flag ) )  // x < 0: padding of a per-copy task list
      {
         const int64_t o = owner_slot( v, tk.x, tk.y, tk.z );
         acc             = double( ldv( a + o ) ) * double( ldv( b + o ) );
      }
   }
   acc = block_sum( acc );
   if ( threadIdx.x == 0 ) partials[blockIdx.x] = acc;
}

__global__ void __launch_bounds__( 1024 ) k_sum_partials( const double* partials, int count, double* out )
{
   double acc = 0.0;
   for ( int i = threadIdx.x; i < count; i += blockDim.x ) acc += partials[i];
   acc = block_sum( acc );
   if ( threadIdx.x == 0 ) *out = acc;
}

static double* partials( Context* ctx, int count )
{
   if ( count > ctx->partial_cap )
   {
      // a captured graph may still read the old buffer: keep it until the context goes away
      if ( ctx->d_partials ) ctx->retired.push_back( ctx->d_partials ), ctx->retired_bytes += int64_t( ctx->partial_cap ) * 8;
      ctx->d_partials  = nullptr;
      ctx->partial_cap = std::max( { count, 1 << 16, 2 * ctx->partial_cap } );
      check_cuda( cudaMalloc( &ctx->d_partials, sizeof( double ) * ctx->partial_cap ), "cudaMalloc(partials)" );
   }
   return ctx->d_partials;
}

template < typename T >
static void run_dot( Context* ctx, const LevelView& v, int nC, uint32_t flag, const void* a, const void* b, double* out )
{
   const int nb_cells = ( v.nrows > 0 && nC > 0 ) ? ( ( v.nrows + 7 ) / 8 ) * nC : 0;
   const int nb_bnd   = v.ntasks > 0 ? ( v.ntasks + 255 ) / 256 : 0;
   double*   p        = partials( ctx, nb_cells + nb_bnd + 1 );
   {
      Fork fk( ctx );
      if ( nb_cells )
      {
      dim3 grid( ( v.nrows + 7 ) / 8, nC );
      k_dot_cells< T ><<< grid, 256, 0, ctx->stream >>>( v, flag, (const T*) a, (const T*) b, p );
      ++ctx->launches;
      }
      if ( nb_bnd )
      {
         k_dot_bnd< T ><<< nb_bnd, 256, 0, fk.aux() >>>( v, flag, (const T*) a, (const T*) b, p + nb_cells );
         ++ctx->launches;
      }
   }
   k_sum_partials<<< 1, 1024, 0, ctx->stream >>>( p, nb_cells + nb_bnd, out );
   ++ctx->launches;
   check_cuda( cudaGetLastError(), "dot launch" );
}

// sums of the partials of copy r of a replicated mesh: its cells' row blocks (contiguous, cells are
// ordered copy by copy) and its boundary blocks (contiguous in the per-copy task list), in that order
__global__ void __launch_bounds__( 256 ) k_sum_replicas( const double* partials, int cell_blocks, int bnd_blocks, int nb_cells_total,
                                                          double* out )
{
   const int r   = blockIdx.x;
   double    acc = 0.0;
   for ( int i = threadIdx.x; i < cell_blocks; i += blockDim.x ) acc += partials[size_t( r ) * cell_blocks + i];
   for ( int i = threadIdx.x; i < bnd_blocks; i += blockDim.x ) acc += partials[nb_cells_total + size_t( r ) * bnd_blocks + i];
   acc = block_sum( acc );
   if ( threadIdx.x == 0 ) out[r] = acc;
}

template < typename T >
static void run_dot_replicas( Context* ctx, LevelView v, int nC, uint32_t flag, const void* a, const void* b, int R, const int4* tasks,
                              int tpad, double* out )
{
   const int rb       = ( v.nrows + 7 ) / 8;  // row blocks per cell
   const int nb_cells = v.nrows > 0 ? rb * nC : 0;
   const int bnd_per  = tpad / 256;
   const int nb_bnd   = bnd_per * R;
   double*   p        = partials( ctx, nb_cells + nb_bnd + 1 );
   if ( nb_cells )
   {
      dim3 grid( rb, nC );
      k_dot_cells< T ><<< grid, 256, 0, ctx->stream >>>( v, flag, (const T*) a, (const T*) b, p );
      ++ctx->launches;
   }
   if ( nb_bnd )
   {
      v.tasks  = tasks;
      v.ntasks = tpad * R;
      k_dot_bnd< T ><<< nb_bnd, 256, 0, ctx->stream >>>( v, flag, (const T*) a, (const T*) b, p + nb_cells );
      ++ctx->launches;
   }
   k_sum_replicas<<< R, 256, 0, ctx->stream >>>( p, nb_cells ? rb * ( nC / R ) : 0, bnd_per, nb_cells, out );
   ++ctx->launches;
   check_cuda( cudaGetLastError(), "replica dot launch" );
}

// per-copy dot products on a mesh made of R disjoint copies of one mesh (cells ordered copy by copy):
// out[r] = sum over copy r's owned flagged DoFs of a b; tasks: the boundary tasks regrouped copy by
// copy, each copy padded to tpad (a multiple of 256) with tasks whose x is -1.  The sums per copy
// follow a fixed order, so they do not depend on the other copies' values.
void launch_dot_replicas( Context* ctx, Mesh* m, int L, int dtype, uint32_t flag, const void* a, const void* b, int R, const int4* tasks,
                          int tpad, double* out )
{
   ensure_constants();
   LevelView v  = make_view( m, L );
   const int nC = m->topo.nC;
   if ( R < 1 || nC % R != 0 || tpad % 256 != 0 ) throw std::invalid_argument( "replica dot: bad copy count or task padding" );
   if ( dtype == F64 ) run_dot_replicas< double >( ctx, v, nC, flag, a, b, R, tasks, tpad, out );
   else if ( dtype == F32 ) run_dot_replicas< float >( ctx, v, nC, flag, a, b, R, tasks, tpad, out );
   else run_dot_replicas< __half >( ctx, v, nC, flag, a, b, R, tasks, tpad, out );
}

// packed <-> padded with explicit primitive offsets (a copy of a replicated mesh)
void launch_repack_map( Context* ctx, int64_t count, int np, const int64_t* poff, const int64_t* off, int dtype, int to_padded,
                        double* packed, void* vec )
{
   if ( count <= 0 ) return;
   const int blocks = int( std::min< int64_t >( ( count + 255 ) / 256, 148 * 16 ) );
   if ( dtype == F64 ) k_repack< double ><<< blocks, 256, 0, ctx->stream >>>( count, np, poff, off, to_padded, packed, (double*) vec );
   else if ( dtype == F32 ) k_repack< float ><<< blocks, 256, 0, ctx->stream >>>( count, np, poff, off, to_padded, packed, (float*) vec );
   else k_repack< __half ><<< blocks, 256, 0, ctx->stream >>>( count, np, poff, off, to_padded, packed, (__half*) vec );
   ++ctx->launches;
   check_cuda( cudaGetLastError(), "repack launch" );
}

void launch_dot( Context* ctx, Mesh* m, int L, int dtype, uint32_t flag, const void* a, const void* b, double* out )
{
   ensure_constants();
   LevelView v  = make_view( m, L );
   const int nC = m->topo.nC;
   if ( dtype == F64 ) run_dot< double >( ctx, v, nC, flag, a, b, out );
   else if ( dtype == F32 ) run_dot< float >( ctx, v, nC, flag, a, b, out );
   else run_dot< __half >( ctx, v, nC, flag, a, b, out );
}

// ---------------------------------------------------------------------------------------------
// Allocation-free dot product.
//
// Some callers cannot let a call allocate device memory: a host runtime that reserves the device
// memory up front and hands it out through its own allocator (a cudaMalloc behind its back can
// fail or fragment the reserve), or a latency-critical loop that must not pay the implicit
// device synchronisation of cudaMalloc/cudaFree.  launch_dot grows the context's partials buffer
// on demand; this variant runs the same dot kernels but keeps the per-block partial sums and the
// result in one file-scope device array of fixed size.
//  * set-up: the library's per-device set-up (run by the first operation on a device, with that
//    device current) resolves the array's address once with cudaGetSymbolAddress, together with the
//    constant tables; this entry point refuses to run before it, so it never loads or allocates.
//  * limit: at most kNoAllocPartials block partials (cell-row blocks plus boundary blocks of the
//    level); larger levels are rejected with an error.
//  * nothing has to start at zero: every block of the sweep writes its own partial and the final
//    kernel overwrites the result slot.
//  * the array is shared by all callers on the device, so calls that overlap in time (other
//    streams, other host threads) race on it and must be serialised by the caller.
// ---------------------------------------------------------------------------------------------
constexpr int kNoAllocPartials = 1 << 16;
static __device__ __align__( 256 ) double g_noalloc_dot[kNoAllocPartials + 1];  // partials, result

static double* noalloc_scratch( int device )
{
   static std::mutex mu;
   static double*    ptrs[256] = {};
   if ( device < 0 || device >= 256 ) throw std::invalid_argument( "device ordinal out of range" );
   std::lock_guard< std::mutex > lock( mu );
   if ( !ptrs[device] )
   {
      void* p = nullptr;
      check_cuda( cudaGetSymbolAddress( &p, g_noalloc_dot ), "cudaGetSymbolAddress(allocation-free dot scratch)" );
      ptrs[device] = static_cast< double* >( p );
   }
   return ptrs[device];
}

template < typename T >
static void run_dot_fixed( Context* ctx, const LevelView& v, int nC, uint32_t flag, const void* a, const void* b, double* p,
                           double* out )
{
   const int nb_cells = ( v.nrows > 0 && nC > 0 ) ? ( ( v.nrows + 7 ) / 8 ) * nC : 0;
   const int nb_bnd   = v.ntasks > 0 ? ( v.ntasks + 255 ) / 256 : 0;
   {
      Fork fk( ctx );
      if ( nb_cells )
      {
         dim3 grid( ( v.nrows + 7 ) / 8, nC );
         k_dot_cells< T ><<< grid, 256, 0, ctx->stream >>>( v, flag, (const T*) a, (const T*) b, p );
         ++ctx->launches;
      }
      if ( nb_bnd )
      {
         k_dot_bnd< T ><<< nb_bnd, 256, 0, fk.aux() >>>( v, flag, (const T*) a, (const T*) b, p + nb_cells );
         ++ctx->launches;
      }
   }
   k_sum_partials<<< 1, 1024, 0, ctx->stream >>>( p, nb_cells + nb_bnd, out );
   ++ctx->launches;
   check_cuda( cudaGetLastError(), "dot launch" );
}

void launch_dot_noalloc( Context* ctx, Mesh* m, int L, int dtype, uint32_t flag, const void* a, const void* b, double* host_out )
{
   auto it = m->levels.find( L );
   if ( it == m->levels.end() || !it->second->d_off )
      throw std::invalid_argument( "allocation-free dot: the level's index tables are not on the device yet "
                                   "(run any operation on this level first)" );
   // no set-up here: constant tables, kernel attributes and the scratch address were prepared by an
   // earlier operation on this device (loading them now could allocate device memory)
   if ( !g_const_once.done_on_current_device() )
      throw std::invalid_argument( "allocation-free dot: no operation of this library has run on this device yet "
                                   "(run one first, for example an apply on this level)" );
   double*         scratch  = noalloc_scratch( ctx->device );
   const LevelView v        = make_view( m, L );
   const int       nC       = m->topo.nC;
   const int64_t   nb_cells = ( v.nrows > 0 && nC > 0 ) ? int64_t( ( v.nrows + 7 ) / 8 ) * nC : 0;
   const int64_t   nb_bnd   = v.ntasks > 0 ? ( v.ntasks + 255 ) / 256 : 0;
   if ( nb_cells + nb_bnd > kNoAllocPartials )
      throw std::invalid_argument( "allocation-free dot: this level needs " + std::to_string( nb_cells + nb_bnd ) +
                                   " block partials, the fixed scratch holds " + std::to_string( kNoAllocPartials ) );
   double* out = scratch + kNoAllocPartials;
   if ( dtype == F64 ) run_dot_fixed< double >( ctx, v, nC, flag, a, b, scratch, out );
   else if ( dtype == F32 ) run_dot_fixed< float >( ctx, v, nC, flag, a, b, scratch, out );
   else run_dot_fixed< __half >( ctx, v, nC, flag, a, b, scratch, out );
   check_cuda( cudaMemcpyAsync( host_out, out, sizeof( double ), cudaMemcpyDeviceToHost, ctx->stream ), "dot readback" );
   check_cuda( cudaStreamSynchronize( ctx->stream ), "dot sync" );
}

// ---------------------------------------------------------------------------------------------
// restriction (generated pull kernel semantics, R = P^T) and prolongation
// ---------------------------------------------------------------------------------------------
template < typename T, typename A >
__global__ void __launch_bounds__( 256 ) k_restrict_cells( LevelView cv, LevelView fv, uint32_t flag, const T* __restrict__ fine,
                                                            T* coarse )
{
   const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
   const int r    = blockIdx.x * 8 + warp;
   const int c    = blockIdx.y;
   if ( r >= cv.nrows ) return;
   if ( !( cv.cell_bc[c] & flag ) ) return;
   const int2    yz   = cv.rows[r];
   const int     y = yz.x, z = yz.y, nf = fv.n;
   const T*      f    = fine + fv.cell_off[c];
   const int64_t cb   = cv.cell_off[c] + cidx( cv.n, 0, y, z );
   const int     xmax = cv.n - 1 - y - z;
   for ( int x = 1 + lane; x <= xmax; x += 32 )
   {
      const int X = 2 * x, Y = 2 * y, Z = 2 * z;
      A         leaves = A( 0 );
#pragma unroll
      for ( int d = 1; d < kNumDirs; ++d )
         leaves += A( ldv( f + cidx( nf, X + c_dirs[d][0], Y + c_dirs[d][1], Z + c_dirs[d][2] ) ) );
      stv( coarse + cb + x, A( ldv( f + cidx( nf, X, Y, Z ) ) ) + A( 0.5 ) * leaves );
   }
}

template < typename T, typename A >
__global__ void __launch_bounds__( 256 ) k_restrict_bnd( LevelView cv, LevelView fv, uint32_t flag, const T* __restrict__ fine,
                                                          T* coarse )
{
   const int t = blockIdx.x * blockDim.x + threadIdx.x;
   if ( t >= cv.ntasks ) return;
   const int4 tk = cv.tasks[t];
   const int  b = tk.x, i = tk.y, j = tk.z;
   if ( !( cv.bc[b] & flag ) ) return;
   const int nf  = fv.n;
   A         acc = A( 0 );
   for ( int q = cv.inc_begin[b]; q < cv.inc_begin[b + 1]; ++q )
   {
      const Incidence I = cv.inc[q];
      int             x, y, z;
      inc_point( I, cv.n, i, j, x, y, z );
      const int      X = 2 * x, Y = 2 * y, Z = 2 * z;
      const T*       f    = fine + fv.cell_off[I.cell];
      const float*   ncc  = fv.ncell_cls + size_t( I.cell ) * kNumClasses;
      const uint16_t mask = c_cls_mask[I.cls];
      A              part = A( ldv( f + cidx( nf, X, Y, Z ) ) ) / A( ncc[I.cls] );
      for ( int d = 1; d < kNumDirs; ++d )
         if ( mask & ( 1u << d ) )
         {
            const int px = X + c_dirs[d][0], py = Y + c_dirs[d][1], pz = Z + c_dirs[d][2];
            part += A( 0.5 ) / A( ncc[point_class( nf, px, py, pz )] ) * A( ldv( f + cidx( nf, px, py, pz ) ) );
         }
      acc += part;
   }
   write_through( cv, coarse, b, i, j, owner_slot( cv, b, i, j ), acc );
}

// coarse micro-edge through an odd fine point: direction per odd-coordinate pattern
__device__ __forceinline__ void parity_dir( int x, int y, int z, int& dx, int& dy, int& dz )
{
   const int p = ( x & 1 ) | ( ( y & 1 ) << 1 ) | ( ( z & 1 ) << 2 );
   dx = dy = dz = 0;
   switch ( p )
   {
   case 1: dx = 1; break;
   case 2: dy = 1; break;
   case 4: dz = 1; break;
   case 3: dx = 1, dy = -1; break;
   case 5: dx = 1, dz = -1; break;
   case 6: dy = 1, dz = -1; break;
   case 7: dx = 1, dy = -1, dz = 1; break;
   default: break;
   }
}

template < typename T, typename A >
__device__ __forceinline__ A interp( const T* c, int nc, int x, int y, int z )
{
   int dx, dy, dz;
   parity_dir( x, y, z, dx, dy, dz );
   if ( ( dx | dy | dz ) == 0 ) return A( ldv( c + cidx( nc, x >> 1, y >> 1, z >> 1 ) ) );
   const A a = A( ldv( c + cidx( nc, ( x - dx ) >> 1, ( y - dy ) >> 1, ( z - dz ) >> 1 ) ) );
   const A b = A( ldv( c + cidx( nc, ( x + dx ) >> 1, ( y + dy ) >> 1, ( z + dz ) >> 1 ) ) );
   return A( 0.5 ) * a + A( 0.5 ) * b;
}

template < typename T, typename A >
__global__ void __launch_bounds__( 256 ) k_prolong_cells( LevelView cv, LevelView fv, uint32_t flag, const T* __restrict__ coarse,
                                                           T* fine, int add )
{
   const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
   const int r    = blockIdx.x * 8 + warp;
   const int c    = blockIdx.y;
   if ( r >= fv.nrows ) return;
   if ( !( fv.cell_bc[c] & flag ) ) return;
   const int2    yz   = fv.rows[r];
   const int     y = yz.x, z = yz.y;
   const T*      cc   = coarse + cv.cell_off[c];
   const int64_t fb   = fv.cell_off[c] + cidx( fv.n, 0, y, z );
   const int     xmax = fv.n - 1 - y - z;
   for ( int x = 1 + lane; x <= xmax; x += 32 )
   {
      const A val = interp< T, A >( cc, cv.n, x, y, z );
      stv( fine + fb + x, add ? A( ldc( fine + fb + x ) ) + val : val );
   }
}

template < typename T, typename A >
__global__ void __launch_bounds__( 256 ) k_prolong_bnd( LevelView cv, LevelView fv, uint32_t flag, const T* __restrict__ coarse,
                                                         T* fine, int add )
{
   const int t = blockIdx.x * blockDim.x + threadIdx.x;
   if ( t >= fv.ntasks ) return;
   const int4 tk = fv.tasks[t];
   const int  b = tk.x, i = tk.y, j = tk.z;
   if ( !( fv.bc[b] & flag ) ) return;
   const Incidence I = fv.inc[fv.inc_begin[b]];
   int             x, y, z;
   inc_point( I, fv.n, i, j, x, y, z );
   const A       val   = interp< T, A >( coarse + cv.cell_off[I.cell], cv.n, x, y, z );
   const int64_t owner = owner_slot( fv, b, i, j );
   write_through( fv, fine, b, i, j, owner, add ? A( ldc( fine + owner ) ) + val : val );
}

template < typename T, typename A >
static void run_restrict( Context* ctx, const LevelView& cv, const LevelView& fv, int nC, uint32_t flag, const void* fine,
                          void* coarse )
{
   Fork fk( ctx );
   if ( cv.nrows > 0 && nC > 0 )
   {
      dim3 grid( ( cv.nrows + 7 ) / 8, nC );
      k_restrict_cells< T, A ><<< grid, 256, 0, ctx->stream >>>( cv, fv, flag, (const T*) fine, (T*) coarse );
      ++ctx->launches;
   }
   if ( cv.ntasks > 0 )
   {
      k_restrict_bnd< T, A ><<< ( cv.ntasks + 255 ) / 256, 256, 0, fk.aux() >>>( cv, fv, flag, (const T*) fine, (T*) coarse );
      ++ctx->launches;
   }
   check_cuda( cudaGetLastError(), "restrict launch" );
}

void launch_restrict( Context* ctx, Mesh* m, int Lf, int dtype, uint32_t flag, const void* fine, void* coarse )
{
   ensure_constants();
   LevelView fv = make_view( m, Lf );
   LevelView cv = make_view( m, Lf - 1 );
   const int nC = m->topo.nC;
   if ( dtype == F64 ) run_restrict< double, double >( ctx, cv, fv, nC, flag, fine, coarse );
   else if ( dtype == F32 ) run_restrict< float, float >( ctx, cv, fv, nC, flag, fine, coarse );
   else run_restrict< __half, float >( ctx, cv, fv, nC, flag, fine, coarse );
}

template < typename T, typename A >
static void run_prolong( Context* ctx, const LevelView& cv, const LevelView& fv, int nC, uint32_t flag, const void* coarse,
                         void* fine, int add )
{
   Fork fk( ctx );
   if ( fv.nrows > 0 && nC > 0 )
   {
      dim3 grid( ( fv.nrows + 7 ) / 8, nC );
      k_prolong_cells< T, A ><<< grid, 256, 0, ctx->stream >>>( cv, fv, flag, (const T*) coarse, (T*) fine, add );
      ++ctx->launches;
   }
   if ( fv.ntasks > 0 )
   {
      k_prolong_bnd< T, A ><<< ( fv.ntasks + 255 ) / 256, 256, 0, fk.aux() >>>( cv, fv, flag, (const T*) coarse, (T*) fine,
                                                                                     add );
      ++ctx->launches;
   }
   check_cuda( cudaGetLastError(), "prolongate launch" );
}

void launch_prolongate( Context* ctx, Mesh* m, int Lc, int dtype, uint32_t flag, const void* coarse, void* fine, int add )
{
   ensure_constants();
   LevelView cv = make_view( m, Lc );
   LevelView fv = make_view( m, Lc + 1 );
   const int nC = m->topo.nC;
   if ( dtype == F64 ) run_prolong< double, double >( ctx, cv, fv, nC, flag, coarse, fine, add );
   else if ( dtype == F32 ) run_prolong< float, float >( ctx, cv, fv, nC, flag, coarse, fine, add );
   else run_prolong< __half, float >( ctx, cv, fv, nC, flag, coarse, fine, add );
}

// ---------------------------------------------------------------------------------------------
// P2 quadratic transfers (P2toP2QuadraticProlongation::prolongateAdditively3D,
// P2toP2QuadraticProlongation.cpp:217-424; P2toP2QuadraticRestriction::restrictAdditively3D,
// P2toP2QuadraticRestriction.cpp:131-286), on the P2 storage: P2 level l lives on storage level l+1.
// A fine node F (storage level Lc+1) lies in the coarse micro-cell of anchor A = F / 4 (and offset
// pattern F mod 4) and takes the coarse quadratic there: sum_k w_k u(2A + o_k) over the nodes with
// non-zero basis value (at most ten; on a macro-cell face only the nodes of that face, so every
// referenced coarse node lies in the same macro-cell).  Restriction is the transpose: the coarse
// node J pulls w r(2J + d) over its stencil (per parity class of J), each fine value divided by the
// number of macro-cells sharing its primitive, and owners of face/edge/vertex nodes sum over their
// macro-cells (the reference's scaling plus additive communication).
// ---------------------------------------------------------------------------------------------
constexpr int kP2RMax = 320;
__constant__ int         c_p2p_n[64];
__constant__ signed char c_p2p_o[64][10][3];
__constant__ double      c_p2p_w[64][10];
__constant__ int         c_p2r_begin[9];
__constant__ signed char c_p2r_d[kP2RMax][3];
__constant__ double      c_p2r_w[kP2RMax];

static void ensure_p2_transfer_tables()
{
   static PerDeviceOnce once;
   once.run( [] {
      // micro-cell types (vertex offsets), the same table as the refinement itself
      static const int mc[6][4][3] = { { { 0, 0, 0 }, { 1, 0, 0 }, { 0, 1, 0 }, { 0, 0, 1 } }, { { 1, 0, 0 }, { 1, 1, 0 }, { 0, 1, 0 }, { 1, 0, 1 } },
                                       { { 1, 0, 0 }, { 0, 1, 0 }, { 1, 0, 1 }, { 0, 0, 1 } }, { { 1, 1, 0 }, { 1, 1, 1 }, { 0, 1, 1 }, { 1, 0, 1 } },
                                       { { 1, 0, 1 }, { 0, 1, 1 }, { 0, 0, 1 }, { 0, 1, 0 } }, { { 0, 1, 0 }, { 1, 1, 0 }, { 1, 0, 1 }, { 0, 1, 1 } } };
      static const int ed[6][2] = { { 2, 3 }, { 1, 3 }, { 1, 2 }, { 0, 3 }, { 0, 2 }, { 0, 1 } };
      int              pn[64];
      signed char      po[64][10][3] = {};
      double           pw[64][10]    = {};
      for ( int pat = 0; pat < 64; ++pat )
      {
         const int r[3] = { pat & 3, ( pat >> 2 ) & 3, pat >> 4 };
         const int F[3] = { 4 + r[0], 4 + r[1], 4 + r[2] }, A[3] = { 1, 1, 1 };
         bool      found = false;
         for ( int e = 0; e < 8 && !found; ++e )
         {
            const int a[3] = { A[0] - ( e & 1 ), A[1] - ( ( e >> 1 ) & 1 ), A[2] - ( e >> 2 ) };
            for ( int ty = 0; ty < 6 && !found; ++ty )
            {
               // barycentric coordinates x4 from the unimodular offset matrix (integer inverse)
               int E[3][3];
               for ( int i = 0; i < 3; ++i )
                  for ( int k = 0; k < 3; ++k ) E[i][k] = mc[ty][k + 1][i] - mc[ty][0][i];
               const int det = E[0][0] * ( E[1][1] * E[2][2] - E[1][2] * E[2][1] ) - E[0][1] * ( E[1][0] * E[2][2] - E[1][2] * E[2][0] ) +
                               E[0][2] * ( E[1][0] * E[2][1] - E[1][1] * E[2][0] );
               const int inv[3][3] = { { ( E[1][1] * E[2][2] - E[1][2] * E[2][1] ) * det, ( E[0][2] * E[2][1] - E[0][1] * E[2][2] ) * det,
                                         ( E[0][1] * E[1][2] - E[0][2] * E[1][1] ) * det },
                                       { ( E[1][2] * E[2][0] - E[1][0] * E[2][2] ) * det, ( E[0][0] * E[2][2] - E[0][2] * E[2][0] ) * det,
                                         ( E[0][2] * E[1][0] - E[0][0] * E[1][2] ) * det },
                                       { ( E[1][0] * E[2][1] - E[1][1] * E[2][0] ) * det, ( E[0][1] * E[2][0] - E[0][0] * E[2][1] ) * det,
                                         ( E[0][0] * E[1][1] - E[0][1] * E[1][0] ) * det } };  // det = +-1
               int rel[3];
               for ( int i = 0; i < 3; ++i ) rel[i] = F[i] - 4 * ( a[i] + mc[ty][0][i] );
               int mu4[4] = { 4, 0, 0, 0 };
               for ( int k = 0; k < 3; ++k )
               {
                  mu4[k + 1] = inv[k][0] * rel[0] + inv[k][1] * rel[1] + inv[k][2] * rel[2];
                  mu4[0] -= mu4[k + 1];
               }
               bool inside = true;
               for ( int k = 0; k < 4; ++k ) inside &= mu4[k] >= 0 && mu4[k] <= 4;
               if ( !inside ) continue;
               found = true;
               double mu[4], N[10];
               int    node[10][3];
               for ( int k = 0; k < 4; ++k ) mu[k] = mu4[k] / 4.0;
               for ( int k = 0; k < 4; ++k )
               {
                  N[k] = mu[k] * ( 2.0 * mu[k] - 1.0 );
                  for ( int i = 0; i < 3; ++i ) node[k][i] = 2 * ( a[i] + mc[ty][k][i] );
               }
               for ( int k = 0; k < 6; ++k )
               {
                  N[4 + k] = 4.0 * mu[ed[k][0]] * mu[ed[k][1]];
                  for ( int i = 0; i < 3; ++i ) node[4 + k][i] = ( node[ed[k][0]][i] + node[ed[k][1]][i] ) / 2;
               }
               pn[pat] = 0;
               for ( int k = 0; k < 10; ++k )
                  if ( N[k] != 0.0 )
                  {
                     for ( int i = 0; i < 3; ++i ) po[pat][pn[pat]][i] = static_cast< signed char >( node[k][i] - 2 * A[i] );
                     pw[pat][pn[pat]++] = N[k];
                  }
            }
         }
         if ( !found ) throw std::logic_error( "P2 transfer table: no micro-cell contains a fine node" );
      }
      // restriction stencils: class p = J mod 2, entries (d = r - 2 o, w)
      int         begin[9] = {};
      signed char rd[kP2RMax][3];
      double      rw[kP2RMax];
      int         cnt = 0;
      for ( int p = 0; p < 8; ++p )
      {
         begin[p] = cnt;
         for ( int pat = 0; pat < 64; ++pat )
            for ( int k = 0; k < pn[pat]; ++k )
            {
               const int o[3] = { po[pat][k][0], po[pat][k][1], po[pat][k][2] };
               if ( ( ( o[0] & 1 ) | ( ( o[1] & 1 ) << 1 ) | ( ( o[2] & 1 ) << 2 ) ) != p ) continue;
               if ( cnt >= kP2RMax ) throw std::logic_error( "P2 restriction stencil table overflow" );
               const int r[3] = { pat & 3, ( pat >> 2 ) & 3, pat >> 4 };
               for ( int i = 0; i < 3; ++i ) rd[cnt][i] = static_cast< signed char >( r[i] - 2 * o[i] );
               rw[cnt++] = pw[pat][k];
            }
      }
      begin[8] = cnt;
      check_cuda( cudaMemcpyToSymbol( c_p2p_n, pn, sizeof( pn ) ), "P2 transfer tables" );
      check_cuda( cudaMemcpyToSymbol( c_p2p_o, po, sizeof( po ) ), "P2 transfer tables" );
      check_cuda( cudaMemcpyToSymbol( c_p2p_w, pw, sizeof( pw ) ), "P2 transfer tables" );
      check_cuda( cudaMemcpyToSymbol( c_p2r_begin, begin, sizeof( begin ) ), "P2 transfer tables" );
      check_cuda( cudaMemcpyToSymbol( c_p2r_d, rd, sizeof( rd ) ), "P2 transfer tables" );
      check_cuda( cudaMemcpyToSymbol( c_p2r_w, rw, sizeof( rw ) ), "P2 transfer tables" );
   } );
}

// coarse quadratic at fine cell-local node (x, y, z); nc = coarse storage micro-edges per edge
template < typename T, typename A >
__device__ __forceinline__ A p2_interp( const T* c, int nc, int x, int y, int z )
{
   const int ax = x >> 2, ay = y >> 2, az = z >> 2;
   const int pat = ( x & 3 ) | ( ( y & 3 ) << 2 ) | ( ( z & 3 ) << 4 );
   A         v   = A( 0 );
   for ( int k = 0; k < c_p2p_n[pat]; ++k )
      v += A( c_p2p_w[pat][k] ) *
           A( ldv( c + cidx( nc, 2 * ax + c_p2p_o[pat][k][0], 2 * ay + c_p2p_o[pat][k][1], 2 * az + c_p2p_o[pat][k][2] ) ) );
   return v;
}

template < typename T, typename A >
__global__ void __launch_bounds__( 256 ) k_p2_prolong_cells( LevelView cv, LevelView fv, uint32_t flag, const T* __restrict__ coarse,
                                                              T* fine, int add )
{
   const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
   const int r    = blockIdx.x * 8 + warp;
   const int c    = blockIdx.y;
   if ( r >= fv.nrows ) return;
   if ( !( fv.cell_bc[c] & flag ) ) return;
   const int2    yz   = fv.rows[r];
   const int     y = yz.x, z = yz.y;
   const T*      cc   = coarse + cv.cell_off[c];
   const int64_t fb   = fv.cell_off[c] + cidx( fv.n, 0, y, z );
   const int     xmax = fv.n - 1 - y - z;
   for ( int x = 1 + lane; x <= xmax; x += 32 )
   {
      const A val = p2_interp< T, A >( cc, cv.n, x, y, z );
      stv( fine + fb + x, add ? A( ldc( fine + fb + x ) ) + val : val );
   }
}

template < typename T, typename A >
__global__ void __launch_bounds__( 256 ) k_p2_prolong_bnd( LevelView cv, LevelView fv, uint32_t flag, const T* __restrict__ coarse,
                                                            T* fine, int add )
{
   const int t = blockIdx.x * blockDim.x + threadIdx.x;
   if ( t >= fv.ntasks ) return;
   const int4 tk = fv.tasks[t];
   const int  b = tk.x, i = tk.y, j = tk.z;
   if ( !( fv.bc[b] & flag ) ) return;
   const Incidence I = fv.inc[fv.inc_begin[b]];
   int             x, y, z;
   inc_point( I, fv.n, i, j, x, y, z );
   const A       val   = p2_interp< T, A >( coarse + cv.cell_off[I.cell], cv.n, x, y, z );
   const int64_t owner = owner_slot( fv, b, i, j );
   write_through( fv, fine, b, i, j, owner, add ? A( ldc( fine + owner ) ) + val : val );
}

// one macro-cell's share of the restriction at coarse cell-local node (x, y, z)
template < typename T, typename A >
__device__ __forceinline__ A p2_restrict_share( const T* f, const float* ncc, int nf, int x, int y, int z )
{
   const int p = ( x & 1 ) | ( ( y & 1 ) << 1 ) | ( ( z & 1 ) << 2 );
   A         s = A( 0 );
   for ( int k = c_p2r_begin[p]; k < c_p2r_begin[p + 1]; ++k )
   {
      const int X = 2 * x + c_p2r_d[k][0], Y = 2 * y + c_p2r_d[k][1], Z = 2 * z + c_p2r_d[k][2];
      if ( X < 0 || Y < 0 || Z < 0 || X + Y + Z > nf ) continue;
      s += A( c_p2r_w[k] ) / A( ncc[point_class( nf, X, Y, Z )] ) * A( ldv( f + cidx( nf, X, Y, Z ) ) );
   }
   return s;
}

template < typename T, typename A >
__global__ void __launch_bounds__( 256 ) k_p2_restrict_cells( LevelView cv, LevelView fv, uint32_t flag, const T* __restrict__ fine,
                                                               T* coarse )
{
   const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
   const int r    = blockIdx.x * 8 + warp;
   const int c    = blockIdx.y;
   if ( r >= cv.nrows ) return;
   if ( !( cv.cell_bc[c] & flag ) ) return;
   const int2    yz   = cv.rows[r];
   const int     y = yz.x, z = yz.y;
   const T*      f    = fine + fv.cell_off[c];
   const float*  ncc  = fv.ncell_cls + size_t( c ) * kNumClasses;
   const int64_t cb   = cv.cell_off[c] + cidx( cv.n, 0, y, z );
   const int     xmax = cv.n - 1 - y - z;
   for ( int x = 1 + lane; x <= xmax; x += 32 ) stv( coarse + cb + x, p2_restrict_share< T, A >( f, ncc, fv.n, x, y, z ) );
}

template < typename T, typename A >
__global__ void __launch_bounds__( 256 ) k_p2_restrict_bnd( LevelView cv, LevelView fv, uint32_t flag, const T* __restrict__ fine,
                                                             T* coarse )
{
   const int t = blockIdx.x * blockDim.x + threadIdx.x;
   if ( t >= cv.ntasks ) return;
   const int4 tk = cv.tasks[t];
   const int  b = tk.x, i = tk.y, j = tk.z;
   if ( !( cv.bc[b] & flag ) ) return;
   A acc = A( 0 );
   for ( int q = cv.inc_begin[b]; q < cv.inc_begin[b + 1]; ++q )
   {
      const Incidence I = cv.inc[q];
      int             x, y, z;
      inc_point( I, cv.n, i, j, x, y, z );
      acc += p2_restrict_share< T, A >( fine + fv.cell_off[I.cell], fv.ncell_cls + size_t( I.cell ) * kNumClasses, fv.n, x, y, z );
   }
   write_through( cv, coarse, b, i, j, owner_slot( cv, b, i, j ), acc );
}

template < typename T, typename A >
static void run_p2_restrict( Context* ctx, const LevelView& cv, const LevelView& fv, int nC, uint32_t flag, const void* fine,
                             void* coarse )
{
   Fork fk( ctx );
   if ( cv.nrows > 0 && nC > 0 )
   {
      dim3 grid( ( cv.nrows + 7 ) / 8, nC );
      k_p2_restrict_cells< T, A ><<< grid, 256, 0, ctx->stream >>>( cv, fv, flag, (const T*) fine, (T*) coarse );
      ++ctx->launches;
   }
   if ( cv.ntasks > 0 )
   {
      k_p2_restrict_bnd< T, A ><<< ( cv.ntasks + 255 ) / 256, 256, 0, fk.aux() >>>( cv, fv, flag, (const T*) fine, (T*) coarse );
      ++ctx->launches;
   }
   check_cuda( cudaGetLastError(), "P2 restrict launch" );
}

// Lf: fine STORAGE level (P2 level Lf-1 restricted to P2 level Lf-2)
void launch_p2_restrict( Context* ctx, Mesh* m, int Lf, int dtype, uint32_t flag, const void* fine, void* coarse )
{
   ensure_constants();
   ensure_p2_transfer_tables();
   LevelView fv = make_view( m, Lf );
   LevelView cv = make_view( m, Lf - 1 );
   const int nC = m->topo.nC;
   if ( dtype == F64 ) run_p2_restrict< double, double >( ctx, cv, fv, nC, flag, fine, coarse );
   else if ( dtype == F32 ) run_p2_restrict< float, float >( ctx, cv, fv, nC, flag, fine, coarse );
   else run_p2_restrict< __half, float >( ctx, cv, fv, nC, flag, fine, coarse );
}

template < typename T, typename A >
static void run_p2_prolong( Context* ctx, const LevelView& cv, const LevelView& fv, int nC, uint32_t flag, const void* coarse,
                            void* fine, int add )
{
   Fork fk( ctx );
   if ( fv.nrows > 0 && nC > 0 )
   {
      dim3 grid( ( fv.nrows + 7 ) / 8, nC );
      k_p2_prolong_cells< T, A ><<< grid, 256, 0, ctx->stream >>>( cv, fv, flag, (const T*) coarse, (T*) fine, add );
      ++ctx->launches;
   }
   if ( fv.ntasks > 0 )
   {
      k_p2_prolong_bnd< T, A ><<< ( fv.ntasks + 255 ) / 256, 256, 0, fk.aux() >>>( cv, fv, flag, (const T*) coarse, (T*) fine,
                                                                                        add );
      ++ctx->launches;
   }
   check_cuda( cudaGetLastError(), "P2 prolongate launch" );
}

// Lc: coarse STORAGE level
void launch_p2_prolongate( Context* ctx, Mesh* m, int Lc, int dtype, uint32_t flag, const void* coarse, void* fine, int add )
{
   ensure_constants();
   ensure_p2_transfer_tables();
   LevelView cv = make_view( m, Lc );
   LevelView fv = make_view( m, Lc + 1 );
   const int nC = m->topo.nC;
   if ( dtype == F64 ) run_p2_prolong< double, double >( ctx, cv, fv, nC, flag, coarse, fine, add );
   else if ( dtype == F32 ) run_p2_prolong< float, float >( ctx, cv, fv, nC, flag, coarse, fine, add );
   else run_p2_prolong< __half, float >( ctx, cv, fv, nC, flag, coarse, fine, add );
}

// allocate every lazily created device table for levels minL..maxL (needed before graph capture)
// ---------------------------------------------------------------------------------------------
// Gauss-Seidel / SOR (P1Operator::smooth_sor, P1Operator.hpp:339-420, with the generated
// sor_3D_macrocell_P1 / sor_3D_macroface_P1 kernels): x <- x + relax D^-1 (b - A x) point by point.
// The reference sweeps the macro-vertices, -edges, -faces and -cells in turn, each
// lexicographically.  Here the same primitive order with colour sets inside each class: vertex DoFs
// (no two are neighbours), edge DoFs by the parity of their edge index, face DoFs by (i + 2j) mod 3,
// cell interiors by (x + 2y + 3z) mod 4.  The last is a proper colouring of the 15-point stencil
// (the offsets give 1, 2, 3, 1, 2, 1 and 2 mod 4), so a cell colour is updated in place.  Points of
// different faces or edges can be neighbours, so a boundary colour set is computed from the values
// before the set (into a scratch array) and then written through: every set is deterministic.
// Backward sweeps run the sets in reverse order.
// ---------------------------------------------------------------------------------------------
template < typename T, typename A >
__global__ void __launch_bounds__( 256 ) k_sor_cell( LevelView v, OpView< A > o, uint32_t flag, int color, const T* __restrict__ rhs,
                                                      T* x, A relax )
{
   const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
   const int r    = blockIdx.x * 8 + warp;
   const int c    = blockIdx.y;
   if ( r >= v.nrows || !( v.cell_bc[c] & flag ) ) return;
   const int2    yz   = v.rows[r];
   const int     y = yz.x, z = yz.y, n = v.n;
   const int64_t base = v.cell_off[c];
   T*            s    = x + base;
   const int64_t r00 = cidx( n, 0, y, z ), rm0 = cidx( n, 0, y - 1, z ), rp0 = cidx( n, 0, y + 1, z );
   const int64_t r0m = cidx( n, 0, y, z - 1 ), r0p = cidx( n, 0, y, z + 1 );
   const int64_t rmp = cidx( n, 0, y - 1, z + 1 ), rpm = cidx( n, 0, y + 1, z - 1 );
   const A*      W    = o.W + size_t( c ) * kNumClasses * kNumDirs;  // interior class 0
   const A       invd = o.invd_c[c];
   const int     xmax = n - 1 - y - z;
   const int     x0   = 1 + ( ( ( color - 1 - 2 * y - 3 * z ) % 4 ) + 4 ) % 4;  // first x >= 1 of the colour
   for ( int xx = x0 + 4 * lane; xx <= xmax; xx += 128 )
   {
      A acc = W[0] * A( ldc( s + r00 + xx ) );
      acc += W[1] * A( ldc( s + r00 + xx - 1 ) );
      acc += W[2] * A( ldc( s + r00 + xx + 1 ) );
      acc += W[3] * A( ldc( s + rm0 + xx ) );
      acc += W[4] * A( ldc( s + rp0 + xx ) );
      acc += W[5] * A( ldc( s + r0m + xx ) );
      acc += W[6] * A( ldc( s + r0p + xx ) );
      acc += W[7] * A( ldc( s + rp0 + xx - 1 ) );
      acc += W[8] * A( ldc( s + rm0 + xx + 1 ) );
      acc += W[9] * A( ldc( s + r0p + xx - 1 ) );
      acc += W[10] * A( ldc( s + r0m + xx + 1 ) );
      acc += W[11] * A( ldc( s + rmp + xx ) );
      acc += W[12] * A( ldc( s + rpm + xx ) );
      acc += W[13] * A( ldc( s + rmp + xx + 1 ) );
      acc += W[14] * A( ldc( s + rpm + xx - 1 ) );
      const int64_t i = base + r00 + xx;
      stv( x + i, A( ldc( x + i ) ) + relax * ( invd * ( A( ldc( rhs + i ) ) - acc ) ) );
   }
}

// colour of boundary task tk in its primitive class (kind 0 vertex, 1 edge, 2 face)
__device__ __forceinline__ int sor_task_color( int kind, const int4& tk ) { return kind == 1 ? ( tk.y & 1 ) : kind == 2 ? ( tk.y + 2 * tk.z ) % 3 : 0; }

template < typename T, typename A >
__global__ void __launch_bounds__( 256 ) k_sor_bnd_new( LevelView v, OpView< A > o, uint32_t flag, int kind, int color,
                                                         const T* __restrict__ rhs, const T* x, A relax, A* nv )
{
   const int t = blockIdx.x * blockDim.x + threadIdx.x;
   if ( t >= v.ntasks ) return;
   const int4 tk = v.tasks[t];
   const int  b  = tk.x;
   if ( v.bkind[b] != kind || !( v.bc[b] & flag ) || sor_task_color( kind, tk ) != color ) return;
   const int     n     = v.n;
   const int64_t owner = owner_slot( v, b, tk.y, tk.z );
   A             acc   = A( 0 );
   for ( int q = v.inc_begin[b]; q < v.inc_begin[b + 1]; ++q )
   {
      const Incidence I = v.inc[q];
      int             px, py, pz;
      inc_point( I, n, tk.y, tk.z, px, py, pz );
      acc += class_stencil< T, A >( x + v.cell_off[I.cell], o.W + ( size_t( I.cell ) * kNumClasses + I.cls ) * kNumDirs, c_cls_mask[I.cls],
                                    n, px, py, pz );
   }
   nv[t] = A( ldc( x + owner ) ) + relax * ( o.invd_b[b] * ( A( ldc( rhs + owner ) ) - acc ) );
}

template < typename T, typename A >
__global__ void __launch_bounds__( 256 ) k_sor_bnd_write( LevelView v, uint32_t flag, int kind, int color, const A* __restrict__ nv, T* x )
{
   const int t = blockIdx.x * blockDim.x + threadIdx.x;
   if ( t >= v.ntasks ) return;
   const int4 tk = v.tasks[t];
   const int  b  = tk.x;
   if ( v.bkind[b] != kind || !( v.bc[b] & flag ) || sor_task_color( kind, tk ) != color ) return;
   write_through( v, x, b, tk.y, tk.z, owner_slot( v, b, tk.y, tk.z ), nv[t] );
}

static double* sor_scratch( Context* ctx, int64_t ntasks )
{
   if ( ctx->sor_cap < ntasks )
   {
      // a captured graph may still read the old buffer: keep it until the context goes away
      if ( ctx->d_sor ) ctx->retired.push_back( ctx->d_sor ), ctx->retired_bytes += ctx->sor_cap * 8;
      ctx->d_sor   = nullptr;
      ctx->sor_cap = std::max( ntasks, 2 * ctx->sor_cap );
      check_cuda( cudaMalloc( &ctx->d_sor, size_t( ctx->sor_cap ) * sizeof( double ) ), "cudaMalloc(SOR scratch)" );
   }
   return ctx->d_sor;
}

template < typename T, typename A >
static void run_sor( Context* ctx, const LevelView& v, const OpView< A >& o, int nC, uint32_t flag, T* x, const T* rhs, A relax, int backwards )
{
   A* nv = reinterpret_cast< A* >( sor_scratch( ctx, std::max( v.ntasks, 1 ) ) );
   // sets: (kind, colour) with kind 3 the cell interiors
   static const int kSets[10][2] = { { 0, 0 }, { 1, 0 }, { 1, 1 }, { 2, 0 }, { 2, 1 }, { 2, 2 }, { 3, 0 }, { 3, 1 }, { 3, 2 }, { 3, 3 } };
   for ( int k = 0; k < 10; ++k )
   {
      const int kind = kSets[backwards ? 9 - k : k][0], color = kSets[backwards ? 9 - k : k][1];
      if ( kind == 3 )
      {
         if ( v.nrows <= 0 || nC <= 0 ) continue;
         dim3 grid( ( v.nrows + 7 ) / 8, nC );
         k_sor_cell< T, A ><<< grid, 256, 0, ctx->stream >>>( v, o, flag, color, rhs, x, relax );
         ++ctx->launches;
         continue;
      }
      if ( v.ntasks <= 0 ) continue;
      const int nb = ( v.ntasks + 255 ) / 256;
      k_sor_bnd_new< T, A ><<< nb, 256, 0, ctx->stream >>>( v, o, flag, kind, color, rhs, x, relax, nv );
      k_sor_bnd_write< T, A ><<< nb, 256, 0, ctx->stream >>>( v, flag, kind, color, nv, x );
      ctx->launches += 2;
   }
   check_cuda( cudaGetLastError(), "SOR launch" );
}

void launch_sor( Context* ctx, Mesh* m, Operator* op, int L, int dtype, uint32_t flag, void* x, const void* rhs, double relax,
                 int backwards )
{
   ensure_constants();
   if ( op->elementwise ) throw std::invalid_argument( "Gauss-Seidel / SOR is provided for constant-stencil operators" );
   LevelView v  = make_view( m, L );
   OpLevel&  ol = op->lv.at( L );
   ensure_device_op( ol );
   const int nC = m->topo.nC;
   if ( dtype == F64 )
      run_sor< double, double >( ctx, v, OpView< double >{ ol.d_W, ol.d_invd_b, ol.d_invd_c }, nC, flag, (double*) x, (const double*) rhs,
                                 relax, backwards );
   else if ( dtype == F32 )
      run_sor< float, float >( ctx, v, OpView< float >{ ol.d_Wf, ol.d_invd_bf, ol.d_invd_cf }, nC, flag, (float*) x, (const float*) rhs,
                               float( relax ), backwards );
   else
      run_sor< __half, float >( ctx, v, OpView< float >{ ol.d_Wf, ol.d_invd_bf, ol.d_invd_cf }, nC, flag, (__half*) x, (const __half*) rhs,
                                float( relax ), backwards );
}

void prepare_device( Context* ctx, Mesh* m, Operator* op, int minL, int maxL, int dtype )
{
   ensure_constants();
   if ( op && op->order == 2 ) ensure_p2_transfer_tables();
   int most = 1;
   for ( int L = minL; L <= maxL; ++L )
   {
      LevelView v = make_view( m, L );
      if ( op && op->kind == HYB_P2_CONST_LAPLACE )
      {
         ensure_p2_constant_device();
         ensure_p2_constant_tables( op->p2c.at( L ) );
      }
      else if ( op && !op->elementwise ) ensure_device_op( op->lv.at( L ) );
      if ( op && op->elementwise )
      {
         ensure_elementwise_level( ctx, op, L, dtype );
         if ( L == minL && dtype != F64 ) ensure_elementwise_level( ctx, op, L, F64 );
      }
      const int nb = ( ( v.nrows + 7 ) / 8 ) * m->topo.nC + ( v.ntasks + 255 ) / 256 + 1;
      most         = std::max( most, nb );
      if ( op && !op->elementwise && op->order == 1 ) sor_scratch( ctx, std::max( v.ntasks, 1 ) );
   }
   partials( ctx, most );
}

// ---------------------------------------------------------------------------------------------
// CG scalars on the device (CGSolver.hpp:94-206 control flow without host round trips)
// state: [0] prsold [1] res_start [2] pAp [3] rsnew [4] alpha [5] beta [6] done [7] iterations
// ---------------------------------------------------------------------------------------------
__global__ void k_cg_scalar( double* s, int stage, double rtol, double atol )
{
   if ( stage == 0 )
   {
      s[0] = s[3];
      s[1] = sqrt( s[3] );
      s[6] = ( s[1] < atol ) ? 1.0 : 0.0;
      s[7] = 0.0;
      s[4] = s[5] = 0.0;
      return;
   }
   if ( s[6] != 0.0 ) return;
   if ( stage == 1 ) { s[4] = s[0] / s[2]; }
   else
   {
      const double sq = sqrt( s[3] );
      s[7] += 1.0;
      if ( sq / s[1] < rtol || sq < atol ) { s[6] = 1.0; }
      else
      {
         s[5] = s[3] / s[0];
         s[0] = s[3];
      }
   }
}

void launch_cg_scalar( Context* ctx, double* state, int stage, double rtol, double atol )
{
   k_cg_scalar<<< 1, 1, 0, ctx->stream >>>( state, stage, rtol, atol );
   ++ctx->launches;
   check_cuda( cudaGetLastError(), "cg scalar launch" );
}

}  // namespace hyb
