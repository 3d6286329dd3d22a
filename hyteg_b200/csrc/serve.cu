// Serving loop: continuous admission of multigrid solve requests on one GPU.
//
// A request names a resident mesh, an operator (P1 Laplace or elementwise -div(k grad u) with
// optional shell blending), a level, a right-hand side, a tolerance and the precision mode
// (plain FP64 cycles, or FP64 defect correction around FP32 cycles).  Requests wait in a queue and
// are admitted in arrival order into "slots" as slots and the HBM budget allow (a request whose key
// has only busy slots waits for one of them and lets later requests pass).  A slot is a resident
// multigrid hierarchy (operator tables, functions on every level, the solver with its CUDA graph)
// keyed by (mesh, operator, coefficient, blending, level, precision); a finished request leaves its
// slot idle so the next request with the same key reuses it without any setup (the captured graph
// is replayed), and a further slot of a key copies the solver setup of the first.  Every slot owns a context with its own stream, so the cycles of different solves
// overlap on the device.  Each scheduler step launches one cycle on every running slot whose last
// residual check has come back, followed by an asynchronous residual norm (device dot, copy to
// pinned host memory, event); finished slots are retired as their events complete.  Kernels and
// reduction orders inside a slot do not depend on what else runs, so a request's result is the same
// alone and in a mix.
//
// Batches (batch_width > 1): FP64 P1 requests of one key share a batch slot of batch_width solves
// (P2 and mixed-precision requests keep one-solve slots).  Its
// multigrid hierarchy lives on a mesh made of batch_width disjoint copies of the request mesh
// (hyb_internal_mesh_replicate), so every launch of a cycle (sweeps, transfers, the coarse solve)
// serves all solves of the batch; copy r of the mesh carries the solve in batch place r.  A request
// is placed into a free place of a batch of its key (its right-hand side is generated or uploaded on
// the original mesh and scattered into the place, its iterate zeroed), the batch runs one V-cycle
// for all places per scheduler pass, and per-place residual norms (dot products restricted to each
// copy, in a fixed order) decide which solves retire; freed places take the next queued requests of
// the key while the others keep iterating.  Places without a solve hold zero right-hand sides and
// iterates.  Every kernel treats the copies independently except the coarse CG solve, whose step
// lengths come from dot products over all copies: a solve's iterates in a batch therefore agree with
// its iterates alone up to the coarse solve's tolerance (bitwise where the coarsest level has no
// free DoF, as on the six-tetrahedra cube).
#include "hyb_internal.hpp"
#include "../../include/hyteg_b200.h"

#include <chrono>
#include <cmath>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <random>
#include <stdexcept>
#include <vector>

namespace hyb {
double gmg_slot_bytes_estimate( Mesh* m, int minL, int maxL, int dtype, int elementwise );
}

struct ServeKey
{
   hyb_mesh* mesh;
   int       kind;
   int       blending;
   int       level;
   int       mixed;
   double    k[6];
   bool      operator<( const ServeKey& o ) const
   {
      if ( mesh != o.mesh ) return mesh < o.mesh;
      if ( kind != o.kind ) return kind < o.kind;
      if ( blending != o.blending ) return blending < o.blending;
      if ( level != o.level ) return level < o.level;
      if ( mixed != o.mixed ) return mixed < o.mixed;
      return std::memcmp( k, o.k, sizeof( k ) ) < 0;
   }
   bool operator==( const ServeKey& o ) const { return !( *this < o ) && !( o < *this ); }
};

struct ServeRequest
{
   int64_t             id;
   ServeKey            key;
   hyb_coeff           coeff;
   std::vector< double > rhs;  // packed host rhs (empty: seeded uniform [-1,1] on owned non-Dirichlet DoFs)
   uint64_t            seed;
   double              rtol;
   int                 max_cycles;
   double*             x_out;
   double              t_arrival = 0, t_admit = -1, t_done = -1;
   int                 state     = 0;  // 0 queued, 1 running, 2 done, 3 failed
   int                 cycles    = 0;
   double              r0 = 0, rn = 0;
};

struct ServeSlot
{
   ServeKey  key;
   // batch slots (reps > 1): the replicated mesh, one level of the original mesh for right-hand
   // sides, the copy maps, packed staging and the solve per place
   int                    reps    = 1;
   hyb_mesh*              umesh   = nullptr;
   hyb_fn*                scratch = nullptr;
   void*                  d_poff = nullptr;
   void*                  d_off  = nullptr;
   void*                  d_tasks = nullptr;
   int                    np = 0, tpad = 0;
   int64_t                count  = 0;
   double*                d_packed = nullptr;
   double*                h_packed = nullptr;
   double*                d_norms  = nullptr;  // 2 reps: ||b||^2 of fresh places, then ||r||^2 after the cycle
   double*                h_norms  = nullptr;
   std::vector< int64_t > rreq;
   std::vector< char >    rfresh;
   hyb_ctx*  ctx  = nullptr;
   hyb_op*   op   = nullptr;
   hyb_gmg*  gmg  = nullptr;
   hyb_fn*   x    = nullptr;
   hyb_fn*   b    = nullptr;
   hyb_fn*   tmp  = nullptr;
   double*   d_norm = nullptr;
   double*   h_norm = nullptr;
   cudaEvent_t ev = nullptr;
   int64_t   req  = -1;
   bool      pending = false;
   double    bytes   = 0;
   double    last_used = 0;
   double    scale     = 1.0;  // mixed mode: residual scaling of the cycle in flight
   bool      solved    = false;  // the solver setup (Chebyshev radii, coarse cap) exists
};

struct hyb_serve
{
   hyb_ctx*                              ctx = nullptr;
   hyb_serve_params                      p{};
   std::deque< int64_t >                 queue;
   std::map< int64_t, ServeRequest >     reqs;
   std::vector< std::unique_ptr< ServeSlot > > slots;
   double                                used_bytes = 0;
   int64_t                               next_id    = 0;
   std::chrono::steady_clock::time_point t0         = std::chrono::steady_clock::now();
   double now() const { return std::chrono::duration< double >( std::chrono::steady_clock::now() - t0 ).count(); }
};

extern "C" int hyb_internal_residual_async( hyb_op* op, hyb_fn* x, hyb_fn* b, hyb_fn* tmp, int level, double* d_out );
extern "C" int hyb_internal_mixed_step_async( hyb_gmg* g, int inner_dtype, hyb_op* op, hyb_fn* x, hyb_fn* b, int level, double rn,
                                              double* d_out );
extern "C" int hyb_fn_fill_random( hyb_fn* fn, int level, uint64_t seed );
extern "C" int hyb_internal_gmg_copy_setup( hyb_gmg* dst, const hyb_gmg* src );
extern "C" int hyb_internal_mesh_replicate( hyb_mesh* m, int R, hyb_mesh** out );
extern "C" int hyb_internal_replica_maps( hyb_mesh* orig, hyb_mesh* uni, int R, int Ls, void** d_poff, void** d_off, void** d_tasks,
                                          int* np_out, int64_t* count, int* tpad_out );
extern "C" int hyb_internal_replica_copy( hyb_fn* ufn, int level, int to_union, const void* d_poff, const void* d_off_r, int np,
                                          int64_t count, double* d_packed );
extern "C" int hyb_internal_fn_packed_device( hyb_fn* fn, int level, int to_padded, double* d_packed );
extern "C" int hyb_internal_residual_replicas_async( hyb_op* op, hyb_fn* x, hyb_fn* b, hyb_fn* tmp, int level, int R, const void* d_tasks,
                                                     int tpad, double* d_out );

static thread_local std::string s_err;

namespace {

void ok( int rc )
{
   if ( rc != HYB_OK ) throw std::runtime_error( hyb_last_error() );
}

void free_slot( hyb_serve* s, ServeSlot* sl )
{
   if ( sl->ctx ) hyb_ctx_synchronize( sl->ctx );
   if ( sl->ev ) cudaEventDestroy( sl->ev );
   if ( sl->h_norm ) cudaFreeHost( sl->h_norm );
   if ( sl->d_norm ) cudaFree( sl->d_norm );
   hyb_gmg_destroy( sl->gmg );
   hyb_fn_destroy( sl->x );
   hyb_fn_destroy( sl->b );
   hyb_fn_destroy( sl->tmp );
   hyb_fn_destroy( sl->scratch );
   hyb_op_destroy( sl->op );
   if ( sl->d_poff ) cudaFree( sl->d_poff );
   if ( sl->d_off ) cudaFree( sl->d_off );
   if ( sl->d_tasks ) cudaFree( sl->d_tasks );
   if ( sl->d_packed ) cudaFree( sl->d_packed );
   if ( sl->d_norms ) cudaFree( sl->d_norms );
   if ( sl->h_packed ) cudaFreeHost( sl->h_packed );
   if ( sl->h_norms ) cudaFreeHost( sl->h_norms );
   hyb_mesh_destroy( sl->umesh );
   hyb_ctx_destroy( sl->ctx );
   s->used_bytes -= sl->bytes;
}

// P2 requests keep P2 level l on the node set of storage level l+1
int shift_of( int kind ) { return kind == HYB_P2_ELEM_DIVKGRAD || kind == HYB_P2_CONST_LAPLACE ? 1 : 0; }

// the request's operator on a mesh (the request mesh or its replicated form), element matrices stored
void make_op( hyb_ctx* ctx, hyb_mesh* mesh, const ServeKey& key, const hyb_coeff& coeff, hyb_op** op )
{
   const int L = key.level;
   if ( key.kind == HYB_P1_CONST_LAPLACE || key.kind == HYB_P2_CONST_LAPLACE ) ok( hyb_op_create( ctx, mesh, key.kind, 0, L, op ) );
   else
   {
      // resident hierarchies are solved many times: compute the element matrices once
      if ( key.kind == HYB_P2_ELEM_DIVKGRAD ) ok( hyb_op_create_p2_divkgrad( ctx, mesh, 0, L, &coeff, key.blending, op ) );
      else ok( hyb_op_create_divkgrad( ctx, mesh, 0, L, &coeff, key.blending, op ) );
      ok( hyb_op_store_element_matrices( *op ) );
   }
}

void make_fn( hyb_ctx* ctx, hyb_mesh* mesh, int kind, int lo, int hi, hyb_fn** f )
{
   if ( shift_of( kind ) ) ok( hyb_fn_create_p2( ctx, mesh, HYB_F64, lo, hi, f ) );
   else ok( hyb_fn_create( ctx, mesh, HYB_F64, lo, hi, f ) );
}

// bytes a slot holds: x, b (all levels), tmp and the solver's temporaries (about six more vectors
// per level), plus the elementwise scratch
// (plus, for div-k-grad, the stored matrices, kept as assembled stencils: 15 values per DoF slot and
// level, in FP64 and for mixed slots also in FP32)
double slot_bytes( ServeKey k )
{
   int64_t total = 0;
   double  mats  = 0;
   const int sh = shift_of( k.kind );
   for ( int L = 0; L <= k.level; ++L )
   {
      int64_t n = 0;
      hyb_layout_packed_size( k.mesh, L + sh, &n );
      total += n;
      if ( k.kind == HYB_P1_ELEM_DIVKGRAD ) mats += double( n ) * 15.0;
      // 55 values per micro-cell; P2 level l has 8^l micro-cells per macro-cell and about 8^(l+1)/6
      // nodes, 0.75 micro-cells per node (44 values per node with the padding of the anchor rows)
      if ( k.kind == HYB_P2_ELEM_DIVKGRAD ) mats += double( n ) * 44.0;
   }
   return double( total ) * 8.0 * ( k.mixed ? 12.0 : 10.0 ) + mats * ( k.mixed ? 12.0 : 8.0 );
}

ServeSlot* make_slot( hyb_serve* s, const ServeRequest& r )
{
   auto sl = std::make_unique< ServeSlot >();
   sl->key = r.key;
   int dev = 0;
   cudaGetDevice( &dev );
   ok( hyb_ctx_create( dev, nullptr, &sl->ctx ) );
   const int L = r.key.level;
   make_op( sl->ctx, r.key.mesh, r.key, r.coeff, &sl->op );
   hyb_gmg_params gp;
   hyb_gmg_params_default( &gp );
   gp.min_level             = 0;
   gp.max_level             = L;
   gp.pre_smooth            = s->p.pre_smooth;
   gp.post_smooth           = s->p.post_smooth;
   gp.smoother              = HYB_SMOOTHER_CHEBYSHEV;
   gp.cheb_order            = 3;
   gp.cheb_power_iterations = s->p.power_iterations;
   gp.use_graph             = 1;
   ok( hyb_gmg_create( sl->ctx, sl->op, &gp, &sl->gmg ) );
   // a second slot of a key takes the first one's solver setup instead of repeating it
   for ( auto& up : s->slots )
      if ( up->key == r.key && up->solved )
      {
         ok( hyb_internal_gmg_copy_setup( sl->gmg, up->gmg ) );
         sl->solved = true;
         break;
      }
   make_fn( sl->ctx, r.key.mesh, r.key.kind, 0, L, &sl->x );
   make_fn( sl->ctx, r.key.mesh, r.key.kind, 0, L, &sl->b );
   make_fn( sl->ctx, r.key.mesh, r.key.kind, L, L, &sl->tmp );
   if ( cudaMalloc( &sl->d_norm, sizeof( double ) ) != cudaSuccess ) throw std::runtime_error( "cudaMalloc(norm)" );
   if ( cudaMallocHost( &sl->h_norm, sizeof( double ) ) != cudaSuccess ) throw std::runtime_error( "cudaMallocHost(norm)" );
   if ( cudaEventCreateWithFlags( &sl->ev, cudaEventDisableTiming ) != cudaSuccess ) throw std::runtime_error( "cudaEventCreate" );
   sl->bytes = slot_bytes( r.key );
   s->used_bytes += sl->bytes;
   s->slots.push_back( std::move( sl ) );
   return s->slots.back().get();
}

ServeSlot* make_batch( hyb_serve* s, const ServeRequest& r )
{
   auto      sl = std::make_unique< ServeSlot >();
   const int R  = s->p.batch_width, L = r.key.level;
   sl->key      = r.key;
   sl->reps     = R;
   int dev      = 0;
   cudaGetDevice( &dev );
   ok( hyb_ctx_create( dev, nullptr, &sl->ctx ) );
   ok( hyb_internal_mesh_replicate( r.key.mesh, R, &sl->umesh ) );
   make_op( sl->ctx, sl->umesh, r.key, r.coeff, &sl->op );
   hyb_gmg_params gp;
   hyb_gmg_params_default( &gp );
   gp.min_level             = 0;
   gp.max_level             = L;
   gp.pre_smooth            = s->p.pre_smooth;
   gp.post_smooth           = s->p.post_smooth;
   gp.smoother              = HYB_SMOOTHER_CHEBYSHEV;
   gp.cheb_order            = 3;
   gp.cheb_power_iterations = s->p.power_iterations;
   gp.use_graph             = 1;
   ok( hyb_gmg_create( sl->ctx, sl->op, &gp, &sl->gmg ) );
   for ( auto& up : s->slots )
      if ( up->key == r.key && up->reps == R && up->solved )
      {
         ok( hyb_internal_gmg_copy_setup( sl->gmg, up->gmg ) );
         sl->solved = true;
         break;
      }
   make_fn( sl->ctx, sl->umesh, r.key.kind, 0, L, &sl->x );
   make_fn( sl->ctx, sl->umesh, r.key.kind, 0, L, &sl->b );
   make_fn( sl->ctx, sl->umesh, r.key.kind, L, L, &sl->tmp );
   make_fn( sl->ctx, r.key.mesh, r.key.kind, L, L, &sl->scratch );
   ok( hyb_internal_replica_maps( r.key.mesh, sl->umesh, R, L + shift_of( r.key.kind ), &sl->d_poff, &sl->d_off, &sl->d_tasks, &sl->np,
                                  &sl->count, &sl->tpad ) );
   if ( cudaMalloc( &sl->d_packed, size_t( std::max< int64_t >( sl->count, 1 ) ) * sizeof( double ) ) != cudaSuccess ||
        cudaMallocHost( &sl->h_packed, size_t( std::max< int64_t >( sl->count, 1 ) ) * sizeof( double ) ) != cudaSuccess ||
        cudaMalloc( &sl->d_norms, 2 * R * sizeof( double ) ) != cudaSuccess || cudaMallocHost( &sl->h_norms, 2 * R * sizeof( double ) ) != cudaSuccess )
      throw std::runtime_error( "batch slot allocation failed" );
   if ( cudaEventCreateWithFlags( &sl->ev, cudaEventDisableTiming ) != cudaSuccess ) throw std::runtime_error( "cudaEventCreate" );
   for ( int l = 0; l <= L; ++l )
   {
      ok( hyb_fn_interpolate_const( sl->x, 0.0, l, HYB_ALL ) );
      ok( hyb_fn_interpolate_const( sl->b, 0.0, l, HYB_ALL ) );
   }
   sl->rreq.assign( R, -1 );
   sl->rfresh.assign( R, 0 );
   sl->bytes = slot_bytes( r.key ) * R;
   s->used_bytes += sl->bytes;
   s->slots.push_back( std::move( sl ) );
   return s->slots.back().get();
}

// a slot with no solve in it (may be evicted or, for single slots, reused)
bool idle( const ServeSlot* sl )
{
   if ( sl->reps == 1 ) return sl->req < 0;
   for ( int64_t q : sl->rreq )
      if ( q >= 0 ) return false;
   return !sl->pending;
}

int free_place( const ServeSlot* sl )
{
   for ( int i = 0; i < sl->reps; ++i )
      if ( sl->rreq[i] < 0 ) return i;
   return -1;
}

void* place_off( const ServeSlot* sl, int i ) { return static_cast< char* >( sl->d_off ) + size_t( i ) * sl->np * sizeof( int64_t ); }

// a request into place i of a batch: right-hand side generated (or uploaded) on the original mesh and
// scattered into copy i, the copy's iterate zeroed
void admit_place( hyb_serve* s, ServeSlot* sl, int i, ServeRequest& r )
{
   const int L = r.key.level;
   if ( r.rhs.empty() ) ok( hyb_fn_fill_random( sl->scratch, L, r.seed ) );
   else ok( hyb_fn_upload( sl->scratch, L, r.rhs.data() ) );
   ok( hyb_internal_fn_packed_device( sl->scratch, L, 0, sl->d_packed ) );
   ok( hyb_internal_replica_copy( sl->b, L, 1, sl->d_poff, place_off( sl, i ), sl->np, sl->count, sl->d_packed ) );
   void* st = nullptr;
   hyb_ctx_stream( sl->ctx, &st );
   if ( cudaMemsetAsync( sl->d_packed, 0, size_t( sl->count ) * sizeof( double ), (cudaStream_t) st ) != cudaSuccess )
      throw std::runtime_error( "cudaMemsetAsync" );
   ok( hyb_internal_replica_copy( sl->x, L, 1, sl->d_poff, place_off( sl, i ), sl->np, sl->count, sl->d_packed ) );
   sl->rreq[i]   = r.id;
   sl->rfresh[i] = 1;
   r.state       = 1;
   r.t_admit     = s->now();
   r.cycles      = 0;
}

// one V-cycle of every place, preceded by the right-hand-side norms of fresh places (their initial
// residual: the guess is zero), followed by every place's residual norm
void launch_batch( hyb_serve* s, ServeSlot* sl )
{
   const int L = sl->key.level, R = sl->reps, Ls = L + shift_of( sl->key.kind );
   bool      fresh = false;
   for ( int i = 0; i < R; ++i ) fresh = fresh || ( sl->rreq[i] >= 0 && sl->rfresh[i] );
   if ( fresh ) ok( hyb_internal_residual_replicas_async( sl->op, nullptr, sl->b, sl->tmp, Ls, R, sl->d_tasks, sl->tpad, sl->d_norms ) );
   ok( hyb_gmg_solve( sl->gmg, sl->x, sl->b, L ) );
   ok( hyb_internal_residual_replicas_async( sl->op, sl->x, sl->b, sl->tmp, Ls, R, sl->d_tasks, sl->tpad, sl->d_norms + R ) );
   void* st = nullptr;
   hyb_ctx_stream( sl->ctx, &st );
   if ( cudaMemcpyAsync( sl->h_norms, sl->d_norms, 2 * R * sizeof( double ), cudaMemcpyDeviceToHost, (cudaStream_t) st ) != cudaSuccess ||
        cudaEventRecord( sl->ev, (cudaStream_t) st ) != cudaSuccess )
      throw std::runtime_error( "residual check enqueue failed" );
   sl->pending = true;
}

// the finished check of a batch: retire converged places (their iterate copied out)
void retire_places( hyb_serve* s, ServeSlot* sl )
{
   const int R = sl->reps, L = sl->key.level;
   void*     st = nullptr;
   hyb_ctx_stream( sl->ctx, &st );
   for ( int i = 0; i < R; ++i )
   {
      if ( sl->rreq[i] < 0 ) continue;
      ServeRequest& r = s->reqs.at( sl->rreq[i] );
      if ( sl->rfresh[i] )
      {
         r.r0          = std::sqrt( std::max( 0.0, sl->h_norms[i] ) );
         sl->rfresh[i] = 0;
      }
      const double rn = std::sqrt( std::max( 0.0, sl->h_norms[R + i] ) );
      r.cycles += 1;
      r.rn            = rn;
      const bool conv = r.r0 == 0.0 || rn / r.r0 < r.rtol;
      if ( !( conv || r.cycles >= r.max_cycles || !std::isfinite( rn ) ) ) continue;
      if ( r.x_out )
      {
         ok( hyb_internal_replica_copy( sl->x, L, 0, sl->d_poff, place_off( sl, i ), sl->np, sl->count, sl->d_packed ) );
         if ( cudaMemcpyAsync( sl->h_packed, sl->d_packed, size_t( sl->count ) * sizeof( double ), cudaMemcpyDeviceToHost, (cudaStream_t) st ) !=
                  cudaSuccess ||
              cudaStreamSynchronize( (cudaStream_t) st ) != cudaSuccess )
            throw std::runtime_error( "solution read-back failed" );
         std::memcpy( r.x_out, sl->h_packed, size_t( sl->count ) * sizeof( double ) );
      }
      // the place's data returns to zero, so that an idle place stays idle
      if ( cudaMemsetAsync( sl->d_packed, 0, size_t( sl->count ) * sizeof( double ), (cudaStream_t) st ) != cudaSuccess )
         throw std::runtime_error( "cudaMemsetAsync" );
      ok( hyb_internal_replica_copy( sl->x, L, 1, sl->d_poff, place_off( sl, i ), sl->np, sl->count, sl->d_packed ) );
      ok( hyb_internal_replica_copy( sl->b, L, 1, sl->d_poff, place_off( sl, i ), sl->np, sl->count, sl->d_packed ) );
      r.t_done      = s->now();
      r.state       = ( conv && std::isfinite( rn ) ) ? 2 : 3;
      sl->rreq[i]   = -1;
      sl->last_used = r.t_done;
      sl->solved    = true;
   }
}

// queue the work of the next cycle (or the initial residual when rn < 0) and its residual check
void launch_cycle( hyb_serve* s, ServeSlot* sl, ServeRequest& r, double rn )
{
   const int L = r.key.level;
   if ( r.key.mixed )
      ok( hyb_internal_mixed_step_async( sl->gmg, s->p.inner_dtype, sl->op, sl->x, sl->b, L, rn < 0 ? 0.0 : rn, sl->d_norm ) );
   else
   {
      if ( rn >= 0 ) ok( hyb_gmg_solve( sl->gmg, sl->x, sl->b, L ) );
      ok( hyb_internal_residual_async( sl->op, sl->x, sl->b, sl->tmp, L + shift_of( r.key.kind ), sl->d_norm ) );
   }
   void* st = nullptr;
   hyb_ctx_stream( sl->ctx, &st );
   if ( cudaMemcpyAsync( sl->h_norm, sl->d_norm, sizeof( double ), cudaMemcpyDeviceToHost, (cudaStream_t) st ) != cudaSuccess ||
        cudaEventRecord( sl->ev, (cudaStream_t) st ) != cudaSuccess )
      throw std::runtime_error( "residual check enqueue failed" );
   sl->pending = true;
}

void admit( hyb_serve* s, ServeSlot* sl, ServeRequest& r )
{
   const int L = r.key.level;
   sl->req     = r.id;
   for ( int l = 0; l <= L; ++l ) ok( hyb_fn_interpolate_const( sl->x, 0.0, l, HYB_ALL ) );
   if ( r.rhs.empty() ) ok( hyb_fn_fill_random( sl->b, L, r.seed ) );
   else ok( hyb_fn_upload( sl->b, L, r.rhs.data() ) );
   r.state   = 1;
   r.t_admit = s->now();
   r.cycles  = -1;  // the first check is the initial residual
   launch_cycle( s, sl, r, -1.0 );
}

}  // namespace

extern "C" {

int hyb_serve_params_default( hyb_serve_params* p )
{
   if ( !p ) return HYB_EINVAL;
   *p                  = hyb_serve_params{};
   p->max_slots        = 32;
   p->hbm_budget_bytes = 0;  // 0: 80 % of the free device memory at creation
   p->inner_dtype      = HYB_F32;
   p->pre_smooth       = 3;
   p->post_smooth      = 3;
   p->power_iterations = 20;
   p->batch_width      = 1;
   return HYB_OK;
}

int hyb_serve_create( hyb_ctx* ctx, const hyb_serve_params* params, hyb_serve** out )
{
   try
   {
      if ( !ctx || !params || !out ) throw std::invalid_argument( "NULL argument" );
      if ( params->max_slots < 1 ) throw std::invalid_argument( "max_slots must be >= 1" );
      if ( params->inner_dtype != HYB_F32 && params->inner_dtype != HYB_F16 ) throw std::invalid_argument( "inner dtype must be F32 or F16" );
      if ( params->batch_width < 1 || params->batch_width > 256 ) throw std::invalid_argument( "batch_width must be 1..256" );
      auto* s = new hyb_serve();
      s->ctx  = ctx;
      s->p    = *params;
      if ( s->p.hbm_budget_bytes <= 0 )
      {
         size_t fr = 0, tot = 0;
         cudaMemGetInfo( &fr, &tot );
         s->p.hbm_budget_bytes = 0.8 * double( fr );
      }
      *out = s;
      return HYB_OK;
   } catch ( const std::exception& e )
   {
      s_err = e.what();
      return HYB_EINVAL;
   }
}

int hyb_serve_destroy( hyb_serve* s )
{
   if ( !s ) return HYB_OK;
   for ( auto& sl : s->slots ) free_slot( s, sl.get() );
   delete s;
   return HYB_OK;
}

double hyb_serve_now( hyb_serve* s ) { return s ? s->now() : 0.0; }

int hyb_serve_submit( hyb_serve* s, const hyb_request* rq, int64_t* id )
{
   if ( !s || !rq || !rq->mesh ) return HYB_EINVAL;
   if ( rq->op_kind != HYB_P1_CONST_LAPLACE && rq->op_kind != HYB_P1_ELEM_DIVKGRAD && rq->op_kind != HYB_P2_ELEM_DIVKGRAD &&
        rq->op_kind != HYB_P2_CONST_LAPLACE )
      return HYB_EINVAL;
   // the defect-correction step of the serving loop is written for P1 hierarchies
   if ( shift_of( rq->op_kind ) && rq->mixed ) return HYB_EINVAL;
   const bool elem = rq->op_kind == HYB_P1_ELEM_DIVKGRAD || rq->op_kind == HYB_P2_ELEM_DIVKGRAD;
   if ( rq->level < 1 || rq->level > 12 || !( rq->rtol > 0 ) || rq->max_cycles < 1 ) return HYB_EINVAL;
   ServeRequest r;
   r.id            = s->next_id++;
   r.key.mesh      = rq->mesh;
   r.key.kind      = rq->op_kind;
   r.key.blending  = elem ? rq->blending : 0;
   r.key.level     = rq->level;
   r.key.mixed     = rq->mixed ? 1 : 0;
   const double kk[6] = { double( rq->coeff.kind ), rq->coeff.value, rq->coeff.amp, rq->coeff.phase[0], rq->coeff.phase[1],
                          rq->coeff.phase[2] };
   for ( int i = 0; i < 6; ++i ) r.key.k[i] = elem ? kk[i] : 0.0;
   r.coeff      = rq->coeff;
   r.seed       = rq->seed;
   r.rtol       = rq->rtol;
   r.max_cycles = rq->max_cycles;
   r.x_out      = rq->x_out;
   r.t_arrival  = rq->arrival_time >= 0 ? rq->arrival_time : s->now();
   if ( rq->rhs )
   {
      int64_t n = 0;
      if ( hyb_layout_packed_size( rq->mesh, rq->level + shift_of( rq->op_kind ), &n ) != HYB_OK ) return HYB_EINVAL;
      r.rhs.assign( rq->rhs, rq->rhs + n );
   }
   if ( slot_bytes( r.key ) > s->p.hbm_budget_bytes ) return HYB_ENOMEM;  // can never be admitted
   const int64_t rid = r.id;
   s->reqs.emplace( rid, std::move( r ) );
   s->queue.push_back( rid );
   if ( id ) *id = rid;
   return HYB_OK;
}

int hyb_serve_step( hyb_serve* s, int* running, int* queued )
{
   if ( !s ) return HYB_EINVAL;
   try
   {
      // 1. finished residual checks: retire or launch the next cycle
      for ( auto& up : s->slots )
      {
         ServeSlot* sl = up.get();
         if ( sl->reps > 1 )
         {
            if ( sl->pending && cudaEventQuery( sl->ev ) == cudaSuccess )
            {
               sl->pending = false;
               retire_places( s, sl );
            }
            continue;
         }
         if ( sl->req < 0 || !sl->pending ) continue;
         if ( cudaEventQuery( sl->ev ) != cudaSuccess ) continue;
         sl->pending      = false;
         ServeRequest& r  = s->reqs.at( sl->req );
         const double  rn = std::sqrt( std::max( 0.0, *sl->h_norm ) );
         if ( r.cycles < 0 ) r.r0 = rn;
         r.cycles += 1;
         r.rn            = rn;
         const bool conv = r.r0 == 0.0 || rn / r.r0 < r.rtol;
         if ( conv || r.cycles >= r.max_cycles || !std::isfinite( rn ) )
         {
            if ( r.x_out ) ok( hyb_fn_download( sl->x, r.key.level, r.x_out ) );
            r.t_done      = s->now();
            r.state       = ( conv && std::isfinite( rn ) ) ? 2 : 3;
            sl->req       = -1;
            sl->last_used = r.t_done;
            sl->solved    = true;
         }
         else
            launch_cycle( s, sl, r, rn );
      }
      // 2. admission in arrival order, as slots and the memory budget allow.  A request takes an idle
      //    slot of its key, else a new slot where the budget and the slot limit leave room.  Idle
      //    slots of other keys are evicted (least recently used first) only for a key that has no
      //    slot at all; a request whose key has busy slots waits for one of them, and requests
      //    behind it that can start do.
      for ( auto qi = s->queue.begin(); qi != s->queue.end(); )
      {
         ServeRequest& r    = s->reqs.at( *qi );
         if ( s->p.batch_width > 1 && !r.key.mixed && !shift_of( r.key.kind ) )
         {
            // a free place of a batch of the key (not waiting for its check), else a new batch
            ServeSlot* batch = nullptr;
            int        place = -1;
            bool       has_key = false;
            for ( auto& up : s->slots )
               if ( up->reps > 1 && up->key == r.key )
               {
                  has_key = true;
                  const int i = free_place( up.get() );
                  if ( i >= 0 && !up->pending )
                  {
                     batch = up.get();
                     place = i;
                     break;
                  }
               }
            if ( !batch && !has_key )
            {
               const double need = slot_bytes( r.key ) * s->p.batch_width;
               auto room = [&]() { return s->used_bytes + need <= s->p.hbm_budget_bytes && int( s->slots.size() ) < s->p.max_slots; };
               while ( !room() )
               {
                  int victim = -1;
                  for ( size_t i = 0; i < s->slots.size(); ++i )
                     if ( idle( s->slots[i].get() ) && ( victim < 0 || s->slots[i]->last_used < s->slots[victim]->last_used ) ) victim = int( i );
                  if ( victim < 0 ) break;
                  free_slot( s, s->slots[victim].get() );
                  s->slots.erase( s->slots.begin() + victim );
               }
               if ( room() )
               {
                  batch = make_batch( s, r );
                  place = 0;
               }
            }
            if ( !batch )
            {
               ++qi;
               continue;
            }
            admit_place( s, batch, place, r );
            qi = s->queue.erase( qi );
            continue;
         }
         ServeSlot*    slot = nullptr;
         bool          has_key = false;
         for ( auto& up : s->slots )
            if ( up->key == r.key )
            {
               has_key = true;
               if ( up->req < 0 )
               {
                  slot = up.get();
                  break;
               }
            }
         if ( !slot )
         {
            const double need = slot_bytes( r.key );
            auto         room = [&]() { return s->used_bytes + need <= s->p.hbm_budget_bytes && int( s->slots.size() ) < s->p.max_slots; };
            while ( !room() && !has_key )
            {
               int victim = -1;
               for ( size_t i = 0; i < s->slots.size(); ++i )
                  if ( idle( s->slots[i].get() ) && ( victim < 0 || s->slots[i]->last_used < s->slots[victim]->last_used ) ) victim = int( i );
               if ( victim < 0 ) break;
               free_slot( s, s->slots[victim].get() );
               s->slots.erase( s->slots.begin() + victim );
            }
            if ( !room() )
            {
               ++qi;
               continue;
            }
            slot = make_slot( s, r );
         }
         admit( s, slot, r );
         qi = s->queue.erase( qi );
      }
      // 3. the next cycle of every batch with solves in it
      for ( auto& up : s->slots )
         if ( up->reps > 1 && !up->pending )
         {
            bool any = false;
            for ( int64_t q : up->rreq ) any = any || q >= 0;
            if ( any ) launch_batch( s, up.get() );
         }
      int run = 0;
      for ( auto& up : s->slots )
      {
         if ( up->reps == 1 ) run += up->req >= 0;
         else
            for ( int64_t q : up->rreq ) run += q >= 0;
      }
      if ( running ) *running = run;
      if ( queued ) *queued = int( s->queue.size() );
      return HYB_OK;
   } catch ( const std::exception& e )
   {
      s_err = e.what();
      return HYB_EDEVICE;
   }
}

int hyb_serve_status( hyb_serve* s, int64_t id, int* state, double* t_arrival, double* t_admit, double* t_done, int* cycles,
                      double* rel_res )
{
   if ( !s ) return HYB_EINVAL;
   auto it = s->reqs.find( id );
   if ( it == s->reqs.end() ) return HYB_EINVAL;
   const ServeRequest& r = it->second;
   if ( state ) *state = r.state;
   if ( t_arrival ) *t_arrival = r.t_arrival;
   if ( t_admit ) *t_admit = r.t_admit;
   if ( t_done ) *t_done = r.t_done;
   if ( cycles ) *cycles = std::max( r.cycles, 0 );
   if ( rel_res ) *rel_res = r.r0 > 0 ? r.rn / r.r0 : 0.0;
   return HYB_OK;
}

const char* hyb_serve_last_error( void ) { return s_err.c_str(); }

}  // extern "C"
