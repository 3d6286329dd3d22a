// extern "C" entry points of hyteg_b200 and the host-side solver drivers.
#include "hyb_internal.hpp"
#include "../../include/hyteg_b200.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <fstream>
#include <functional>
#include <random>
#include <sstream>
#include <stdexcept>

// Handles are reference counted: functions, operators and solvers keep their context, mesh and
// operator alive, so the caller may destroy handles in any order.
struct hyb_ctx
{
   hyb::Context c;
   int          refs = 1;
   ~hyb_ctx()
   {
      cudaStreamSynchronize( c.stream );
      cudaFree( c.d_partials );
      cudaFree( c.d_scalars );
      cudaFree( c.d_error );
      cudaFree( c.d_stage );
      cudaFree( c.d_sor );
      for ( void* p : c.retired ) cudaFree( p );
      if ( c.aux ) cudaStreamSynchronize( c.aux ), cudaStreamDestroy( c.aux );
      if ( c.ev_fork ) cudaEventDestroy( c.ev_fork );
      if ( c.ev_join ) cudaEventDestroy( c.ev_join );
      if ( c.own_stream ) cudaStreamDestroy( c.stream );
   }
};
struct hyb_mesh
{
   hyb::Mesh m;
   int       refs = 1;
};
static void ctx_ref( hyb_ctx* c )
{
   if ( c ) ++c->refs;
}
static void ctx_unref( hyb_ctx* c )
{
   if ( c && --c->refs == 0 ) delete c;
}
static void mesh_ref( hyb::Mesh* m )
{
   if ( m ) ++static_cast< hyb_mesh* >( m->handle )->refs;
}
static void mesh_unref( hyb::Mesh* m )
{
   if ( !m ) return;
   auto* h = static_cast< hyb_mesh* >( m->handle );
   if ( --h->refs == 0 )
   {
      hyb_ctx* c = static_cast< hyb_ctx* >( m->owner_ctx );
      delete h;
      ctx_unref( c );
   }
}
struct hyb_fn
{
   hyb::Function f;
   hyb_ctx*      ctx = nullptr;
   double*       stage     = nullptr;  // staging of the asynchronous transfers (packed doubles)
   int64_t       stage_cap = 0;
   ~hyb_fn()
   {
      if ( ctx ) cudaStreamSynchronize( ctx->c.stream );
      cudaFree( stage );
      for ( void* p : f.data ) cudaFree( p );
      f.data.clear();
      mesh_unref( f.mesh );
      ctx_unref( ctx );
   }
};
struct hyb_op
{
   hyb::Operator o;
   hyb_ctx*      ctx = nullptr;
   int           refs = 1;
};
static void op_unref( hyb_op* o )
{
   if ( !o || --o->refs > 0 ) return;
   hyb_ctx*   c = o->ctx;
   hyb::Mesh* m = o->o.mesh;
   cudaStreamSynchronize( c->c.stream );
   delete o;
   mesh_unref( m );
   ctx_unref( c );
}

namespace hyb {
std::vector< std::array< double, 3 > > g_unused;
int  read_gmsh( const std::string& path, std::vector< std::array< double, 3 > >& coords, std::vector< std::array< int, 4 > >& tets );
void cuboid( const double* lo, const double* hi, int nx, int ny, int nz, std::vector< std::array< double, 3 > >& coords,
             std::vector< std::array< int, 4 > >& tets );
void spherical_shell( int ntan, const std::vector< double >& layers, std::vector< std::array< double, 3 > >& coords,
                      std::vector< std::array< int, 4 > >& tets );
std::vector< double > chebyshev_coefficients( int order, double lower, double upper );
}  // namespace hyb

using namespace hyb;

static thread_local std::string g_err;

#define HYB_TRY try {
#define HYB_CATCH                                                                                                              \
   }                                                                                                                           \
   catch ( const std::invalid_argument& e )                                                                                    \
   {                                                                                                                           \
      g_err = e.what();                                                                                                        \
      return HYB_EINVAL;                                                                                                       \
   }                                                                                                                           \
   catch ( const std::bad_alloc& e )                                                                                           \
   {                                                                                                                           \
      g_err = "out of host memory";                                                                                            \
      return HYB_ENOMEM;                                                                                                       \
   }                                                                                                                           \
   catch ( const std::runtime_error& e )                                                                                       \
   {                                                                                                                           \
      g_err = e.what();                                                                                                        \
      return ( g_err.find( "out of memory" ) != std::string::npos ) ? HYB_ENOMEM : HYB_EDEVICE;                                \
   }                                                                                                                           \
   catch ( const std::exception& e )                                                                                           \
   {                                                                                                                           \
      g_err = e.what();                                                                                                        \
      return HYB_EINTERNAL;                                                                                                    \
   }                                                                                                                           \
   return HYB_OK;

static void require( bool cond, const char* msg )
{
   if ( !cond ) throw std::invalid_argument( msg );
}

static void require_level( const Function& f, int L )
{
   if ( L < f.minL || L > f.maxL ) throw std::invalid_argument( "level outside the function's level range" );
}

static void set_device( Context& c ) { check_cuda( cudaSetDevice( c.device ), "cudaSetDevice" ); }

// P2 objects keep P2 level l on the node set of storage level l+1 (lshift 1); entry points take the
// caller's level and work on storage levels
static int  lv( const hyb_fn* f, int level ) { return level + f->f.lshift; }
static void same_space( const hyb_fn* a, const hyb_fn* b )
{
   require( a->f.lshift == b->f.lshift, "P1 and P2 functions mixed in one call" );
}

extern "C" {

const char* hyb_version( void ) { return "hyteg_b200 0.1 (sm_100a)"; }
const char* hyb_last_error( void ) { return g_err.c_str(); }

int hyb_ctx_create( int device, void* stream, hyb_ctx** out )
{
   HYB_TRY
   require( out != nullptr, "out is NULL" );
   int count = 0;
   check_cuda( cudaGetDeviceCount( &count ), "cudaGetDeviceCount" );
   require( device >= 0 && device < count, "device ordinal out of range" );
   auto* h     = new hyb_ctx();
   h->c.device = device;
   set_device( h->c );
   if ( stream ) h->c.stream = (cudaStream_t) stream;
   else
   {
      check_cuda( cudaStreamCreateWithFlags( &h->c.stream, cudaStreamNonBlocking ), "cudaStreamCreate" );
      h->c.own_stream = true;
   }
   check_cuda( cudaMalloc( &h->c.d_scalars, 64 * sizeof( double ) ), "cudaMalloc(scalars)" );
   check_cuda( cudaStreamCreateWithFlags( &h->c.aux, cudaStreamNonBlocking ), "cudaStreamCreate(aux)" );
   check_cuda( cudaMalloc( &h->c.d_error, sizeof( int ) ), "cudaMalloc(error word)" );
   check_cuda( cudaMemset( h->c.d_error, 0, sizeof( int ) ), "cudaMemset(error word)" );
   check_cuda( cudaEventCreateWithFlags( &h->c.ev_fork, cudaEventDisableTiming ), "cudaEventCreate" );
   check_cuda( cudaEventCreateWithFlags( &h->c.ev_join, cudaEventDisableTiming ), "cudaEventCreate" );
   *out = h;
   HYB_CATCH
}

int hyb_ctx_destroy( hyb_ctx* ctx )
{
   HYB_TRY
   ctx_unref( ctx );
   HYB_CATCH
}

int hyb_ctx_synchronize( hyb_ctx* ctx )
{
   HYB_TRY
   require( ctx, "ctx is NULL" );
   check_cuda( cudaStreamSynchronize( ctx->c.stream ), "cudaStreamSynchronize" );
   int e = 0;
   check_cuda( cudaMemcpy( &e, ctx->c.d_error, sizeof( int ), cudaMemcpyDeviceToHost ), "error word readback" );
   if ( e )
   {
      cudaMemset( ctx->c.d_error, 0, sizeof( int ) );
      if ( e == 2 )
      {
         g_err = "a kernel's index self-check failed (an access outside its buffers was skipped)";
         return HYB_EINTERNAL;
      }
      g_err = "a device-side bounded wait ran out (shared-memory staging did not complete)";
      return HYB_ETIMEOUT;
   }
   HYB_CATCH
}

int hyb_ctx_scratch_bytes( const hyb_ctx* ctx, int64_t* out )
{
   HYB_TRY
   require( ctx && out, "NULL argument" );
   const Context& c = ctx->c;
   *out = int64_t( c.partial_cap ) * 8 + c.sor_cap * 8 + c.stage_cap * 8 + c.retired_bytes + ( c.d_scalars ? 64 * 8 : 0 ) +
          ( c.d_error ? 4 : 0 );
   HYB_CATCH
}

int hyb_ctx_launch_count( const hyb_ctx* ctx, int64_t* out )
{
   HYB_TRY
   require( ctx && out, "NULL argument" );
   *out = ctx->c.launches;
   HYB_CATCH
}

int hyb_ctx_stream( const hyb_ctx* ctx, void** stream )
{
   HYB_TRY
   require( ctx && stream, "NULL argument" );
   *stream = (void*) ctx->c.stream;
   HYB_CATCH
}

// ------------------------------------------------------------------------------------------- mesh
static int make_mesh( hyb_ctx* ctx, const std::vector< std::array< double, 3 > >& coords,
                      const std::vector< std::array< int, 4 > >& tets, hyb_mesh** out )
{
   require( out != nullptr, "out is NULL" );
   require( !tets.empty(), "mesh without tetrahedra" );
   auto* h        = new hyb_mesh();
   h->m.ctx       = ctx ? &ctx->c : nullptr;
   h->m.handle    = h;
   h->m.owner_ctx = ctx;
   try
   {
      h->m.topo.build( coords, tets );
   } catch ( ... )
   {
      delete h;
      throw;
   }
   ctx_ref( ctx );
   *out = h;
   return HYB_OK;
}

int hyb_mesh_create( hyb_ctx* ctx, int nverts, const double* coords, int ntets, const int* tets, hyb_mesh** out )
{
   HYB_TRY
   require( nverts > 0 && ntets > 0 && coords && tets, "empty mesh" );
   std::vector< std::array< double, 3 > > c( nverts );
   std::vector< std::array< int, 4 > >    t( ntets );
   for ( int i = 0; i < nverts; ++i ) c[i] = { coords[3 * i], coords[3 * i + 1], coords[3 * i + 2] };
   for ( int i = 0; i < ntets; ++i ) t[i] = { tets[4 * i], tets[4 * i + 1], tets[4 * i + 2], tets[4 * i + 3] };
   return make_mesh( ctx, c, t, out );
   HYB_CATCH
}

int hyb_mesh_create_cuboid( hyb_ctx* ctx, const double* lo, const double* hi, int nx, int ny, int nz, hyb_mesh** out )
{
   HYB_TRY
   require( lo && hi && nx > 0 && ny > 0 && nz > 0, "invalid cuboid" );
   for ( int d = 0; d < 3; ++d ) require( lo[d] < hi[d], "cuboid lower corner must be below upper corner" );
   std::vector< std::array< double, 3 > > c;
   std::vector< std::array< int, 4 > >    t;
   cuboid( lo, hi, nx, ny, nz, c, t );
   return make_mesh( ctx, c, t, out );
   HYB_CATCH
}

int hyb_mesh_create_spherical_shell( hyb_ctx* ctx, int ntan, int nrad, double rmin, double rmax, hyb_mesh** out )
{
   HYB_TRY
   require( nrad >= 2, "nrad must be >= 2" );
   require( rmin > 0 && rmin < rmax, "need 0 < rmin < rmax" );
   std::vector< double > layers( nrad );
   for ( int k = 0; k < nrad; ++k ) layers[k] = rmin + ( ( rmax - rmin ) / double( nrad - 1 ) ) * double( k );
   std::vector< std::array< double, 3 > > c;
   std::vector< std::array< int, 4 > >    t;
   spherical_shell( ntan, layers, c, t );
   int rc = make_mesh( ctx, c, t, out );
   ( *out )->m.topo.shell_rmin = rmin;
   ( *out )->m.topo.shell_rmax = rmax;
   return rc;
   HYB_CATCH
}

int hyb_mesh_create_gmsh( hyb_ctx* ctx, const char* path, hyb_mesh** out )
{
   HYB_TRY
   require( path, "path is NULL" );
   std::vector< std::array< double, 3 > > c;
   std::vector< std::array< int, 4 > >    t;
   read_gmsh( path, c, t );
   return make_mesh( ctx, c, t, out );
   HYB_CATCH
}

int hyb_mesh_destroy( hyb_mesh* mesh )
{
   HYB_TRY
   if ( mesh ) mesh_unref( &mesh->m );
   HYB_CATCH
}

int hyb_mesh_set_boundary_flags_on_boundary( hyb_mesh* mesh, int on_boundary, int inner )
{
   HYB_TRY
   require( mesh, "mesh is NULL" );
   require( mesh->m.levels.empty(), "boundary flags must be set before functions or operators use the mesh" );
   mesh->m.topo.set_boundary_flags_on_boundary( on_boundary, inner );
   HYB_CATCH
}

int hyb_mesh_set_bc_type( hyb_mesh* mesh, int flag, uint32_t dof_type )
{
   HYB_TRY
   require( mesh, "mesh is NULL" );
   require( mesh->m.levels.empty(), "boundary types must be set before functions or operators use the mesh" );
   require( dof_type == kInner || dof_type == kDirichlet || dof_type == kNeumann || dof_type == kFreeslip,
            "dof_type must be a single DoFType bit" );
   mesh->m.topo.bc_of_flag[flag] = dof_type;
   HYB_CATCH
}

int hyb_mesh_counts( const hyb_mesh* mesh, int* counts )
{
   HYB_TRY
   require( mesh && counts, "NULL argument" );
   counts[0] = mesh->m.topo.nV;
   counts[1] = mesh->m.topo.nE;
   counts[2] = mesh->m.topo.nF;
   counts[3] = mesh->m.topo.nC;
   HYB_CATCH
}

int hyb_mesh_primitive_vertices( const hyb_mesh* mesh, int kind, int id, int* out4 )
{
   HYB_TRY
   require( mesh && out4, "NULL argument" );
   const Topology& t = mesh->m.topo;
   for ( int k = 0; k < 4; ++k ) out4[k] = -1;
   switch ( kind )
   {
   case 0: require( id >= 0 && id < t.nV, "id out of range" ), out4[0] = id; break;
   case 1:
      require( id >= 0 && id < t.nE, "id out of range" );
      for ( int k = 0; k < 2; ++k ) out4[k] = t.ev[id][k];
      break;
   case 2:
      require( id >= 0 && id < t.nF, "id out of range" );
      for ( int k = 0; k < 3; ++k ) out4[k] = t.fv[id][k];
      break;
   case 3:
      require( id >= 0 && id < t.nC, "id out of range" );
      for ( int k = 0; k < 4; ++k ) out4[k] = t.cv[id][k];
      break;
   default: throw std::invalid_argument( "kind must be 0..3" );
   }
   HYB_CATCH
}

int hyb_mesh_vertex_coords( const hyb_mesh* mesh, double* out )
{
   HYB_TRY
   require( mesh && out, "NULL argument" );
   for ( int v = 0; v < mesh->m.topo.nV; ++v )
      for ( int d = 0; d < 3; ++d ) out[3 * v + d] = mesh->m.topo.vx[v][d];
   HYB_CATCH
}

int hyb_mesh_primitive_flag( const hyb_mesh* mesh, int kind, int id, int* flag )
{
   HYB_TRY
   require( mesh && flag, "NULL argument" );
   const Topology& t = mesh->m.topo;
   const std::vector< int >* v = kind == 0 ? &t.flag_v : kind == 1 ? &t.flag_e : kind == 2 ? &t.flag_f : kind == 3 ? &t.flag_c : nullptr;
   require( v != nullptr, "kind must be 0..3" );
   require( id >= 0 && id < int( v->size() ), "id out of range" );
   *flag = ( *v )[id];
   HYB_CATCH
}

int hyb_layout_packed_size( hyb_mesh* mesh, int level, int64_t* size )
{
   HYB_TRY
   require( mesh && size, "NULL argument" );
   require( level >= 0 && level <= 14, "level must be in 0..14" );
   *size = mesh->m.level( level ).packed_size;
   HYB_CATCH
}

int hyb_layout_primitive_offsets( hyb_mesh* mesh, int level, int64_t* offsets, int64_t* sizes )
{
   HYB_TRY
   require( mesh, "mesh is NULL" );
   require( level >= 0 && level <= 14, "level must be in 0..14" );
   const P1Level& P = mesh->m.level( level );
   if ( offsets ) std::copy( P.packed_off.begin(), P.packed_off.end(), offsets );
   if ( sizes ) std::copy( P.psize.begin(), P.psize.end(), sizes );
   HYB_CATCH
}

int64_t hyb_layout_cell_index( int level, int x, int y, int z ) { return cidx( 1 << level, x, y, z ); }
int64_t hyb_layout_face_index( int level, int i, int j ) { return fidx( 1 << level, i, j ); }

// ------------------------------------------------------------------------------------------- functions
int hyb_fn_create( hyb_ctx* ctx, hyb_mesh* mesh, int dtype, int min_level, int max_level, hyb_fn** out )
{
   HYB_TRY
   require( ctx && mesh && out, "NULL argument" );
   require( dtype == F64 || dtype == F32 || dtype == F16, "unknown dtype" );
   require( min_level >= 0 && min_level <= max_level && max_level <= 14, "invalid level range" );
   set_device( ctx->c );
   auto* h    = new hyb_fn();
   h->ctx     = ctx;
   h->f.mesh  = &mesh->m;
   h->f.dtype = dtype;
   h->f.minL  = min_level;
   h->f.maxL  = max_level;
   ctx_ref( ctx );
   mesh_ref( &mesh->m );
   try
   {
      for ( int L = min_level; L <= max_level; ++L )
      {
         void*        p  = nullptr;
         const size_t by = h->f.bytes( L );
         check_cuda( cudaMalloc( &p, by ), "cudaMalloc(function)" );
         h->f.data.push_back( p );
         check_cuda( cudaMemsetAsync( p, 0, by, ctx->c.stream ), "cudaMemset(function)" );
      }
   } catch ( ... )
   {
      delete h;
      throw;
   }
   *out = h;
   HYB_CATCH
}

int hyb_fn_create_p2( hyb_ctx* ctx, hyb_mesh* mesh, int dtype, int min_level, int max_level, hyb_fn** out )
{
   HYB_TRY
   require( min_level >= 0 && min_level <= max_level && max_level <= 13, "invalid level range" );
   // P2 level l has the node set of P1 level l+1: stored there
   const int rc = hyb_fn_create( ctx, mesh, dtype, min_level + 1, max_level + 1, out );
   if ( rc != HYB_OK ) return rc;
   ( *out )->f.lshift = 1;
   HYB_CATCH
}

int hyb_fn_destroy( hyb_fn* fn )
{
   HYB_TRY
   delete fn;
   HYB_CATCH
}

// the context's packed staging buffer, grown to n doubles
static double* stage_buffer( Context& c, int64_t n )
{
   if ( n > c.stage_cap )
   {
      if ( c.d_stage )
      {
         check_cuda( cudaStreamSynchronize( c.stream ), "stage sync" );
         check_cuda( cudaFree( c.d_stage ), "cudaFree(stage)" );
         c.d_stage = nullptr;
      }
      check_cuda( cudaMalloc( &c.d_stage, size_t( n ) * sizeof( double ) ), "cudaMalloc(transfer staging)" );
      c.stage_cap = n;
   }
   return c.d_stage;
}

static void sync_copies( hyb_fn* fn, int L )
{
   PointArgs a{};
   a.op   = PT_SYNC;
   a.flag = kAll;
   a.dst  = fn->f.ptr( L );
   launch_point( &fn->ctx->c, fn->f.mesh, L, fn->f.dtype, a );
}

static void to_device( hyb_fn* fn, int L, const std::vector< double >& padded )
{
   const int64_t count = int64_t( padded.size() );
   if ( fn->f.dtype == F64 )
   {
      check_cuda( cudaMemcpyAsync( fn->f.ptr( L ), padded.data(), count * 8, cudaMemcpyHostToDevice, fn->ctx->c.stream ), "upload" );
      check_cuda( cudaStreamSynchronize( fn->ctx->c.stream ), "upload sync" );
   }
   else
   {
      double* tmp = nullptr;
      check_cuda( cudaMalloc( &tmp, count * 8 ), "cudaMalloc(upload staging)" );
      check_cuda( cudaMemcpyAsync( tmp, padded.data(), count * 8, cudaMemcpyHostToDevice, fn->ctx->c.stream ), "upload" );
      launch_convert( &fn->ctx->c, count, fn->f.dtype, fn->f.ptr( L ), F64, tmp );
      check_cuda( cudaStreamSynchronize( fn->ctx->c.stream ), "upload sync" );
      cudaFree( tmp );
   }
}

static std::vector< double > from_device( hyb_fn* fn, int L )
{
   const int64_t         count = fn->f.mesh->level( L ).size;
   std::vector< double > padded( count );
   if ( fn->f.dtype == F64 )
   {
      check_cuda( cudaMemcpyAsync( padded.data(), fn->f.ptr( L ), count * 8, cudaMemcpyDeviceToHost, fn->ctx->c.stream ), "download" );
      check_cuda( cudaStreamSynchronize( fn->ctx->c.stream ), "download sync" );
   }
   else
   {
      double* tmp = nullptr;
      check_cuda( cudaMalloc( &tmp, count * 8 ), "cudaMalloc(download staging)" );
      launch_convert( &fn->ctx->c, count, F64, tmp, fn->f.dtype, fn->f.ptr( L ) );
      check_cuda( cudaMemcpyAsync( padded.data(), tmp, count * 8, cudaMemcpyDeviceToHost, fn->ctx->c.stream ), "download" );
      check_cuda( cudaStreamSynchronize( fn->ctx->c.stream ), "download sync" );
      cudaFree( tmp );
   }
   return padded;
}

int hyb_fn_upload( hyb_fn* fn, int level, const double* host_packed )
{
   HYB_TRY
   require( fn && host_packed, "NULL argument" );
   level = lv( fn, level );
   require_level( fn->f, level );
   // one contiguous host-to-device copy of the packed vector (full bandwidth from pinned memory),
   // then a device scatter into the padded per-primitive layout and the copy refresh
   Context&      c = fn->ctx->c;
   const int64_t n = fn->f.mesh->level( level ).packed_size;
   double*       st = stage_buffer( c, n );
   check_cuda( cudaMemcpyAsync( st, host_packed, size_t( n ) * sizeof( double ), cudaMemcpyHostToDevice, c.stream ), "upload" );
   launch_repack( &c, fn->f.mesh, level, fn->f.dtype, 1, st, fn->f.ptr( level ) );
   sync_copies( fn, level );
   check_cuda( cudaStreamSynchronize( c.stream ), "upload sync" );
   HYB_CATCH
}

// asynchronous transfers: queued on the function's context stream, with the function's own staging
// buffer, so transfers of different functions on different contexts overlap (one direction each way
// through the copy engines) and with kernels of other streams
static double* fn_stage( hyb_fn* fn, int64_t n )
{
   if ( n > fn->stage_cap )
   {
      if ( fn->stage )
      {
         check_cuda( cudaStreamSynchronize( fn->ctx->c.stream ), "stage sync" );
         check_cuda( cudaFree( fn->stage ), "cudaFree(stage)" );
         fn->stage = nullptr;
      }
      check_cuda( cudaMalloc( &fn->stage, size_t( n ) * sizeof( double ) ), "cudaMalloc(transfer staging)" );
      fn->stage_cap = n;
   }
   return fn->stage;
}

int hyb_fn_upload_async( hyb_fn* fn, int level, const double* host_packed )
{
   HYB_TRY
   require( fn && host_packed, "NULL argument" );
   level = lv( fn, level );
   require_level( fn->f, level );
   Context&      c  = fn->ctx->c;
   const int64_t n  = fn->f.mesh->level( level ).packed_size;
   double*       st = fn_stage( fn, n );
   check_cuda( cudaMemcpyAsync( st, host_packed, size_t( n ) * sizeof( double ), cudaMemcpyHostToDevice, c.stream ), "upload" );
   launch_repack( &c, fn->f.mesh, level, fn->f.dtype, 1, st, fn->f.ptr( level ) );
   sync_copies( fn, level );
   HYB_CATCH
}

int hyb_fn_download_async( hyb_fn* fn, int level, double* host_packed )
{
   HYB_TRY
   require( fn && host_packed, "NULL argument" );
   level = lv( fn, level );
   require_level( fn->f, level );
   Context&      c  = fn->ctx->c;
   const int64_t n  = fn->f.mesh->level( level ).packed_size;
   double*       st = fn_stage( fn, n );
   launch_repack( &c, fn->f.mesh, level, fn->f.dtype, 0, st, fn->f.ptr( level ) );
   check_cuda( cudaMemcpyAsync( host_packed, st, size_t( n ) * sizeof( double ), cudaMemcpyDeviceToHost, c.stream ), "download" );
   HYB_CATCH
}

int hyb_fn_download( hyb_fn* fn, int level, double* host_packed )
{
   HYB_TRY
   require( fn && host_packed, "NULL argument" );
   level = lv( fn, level );
   require_level( fn->f, level );
   // device gather into the packed layout (as doubles), one contiguous device-to-host copy
   Context&      c = fn->ctx->c;
   const int64_t n = fn->f.mesh->level( level ).packed_size;
   double*       st = stage_buffer( c, n );
   launch_repack( &c, fn->f.mesh, level, fn->f.dtype, 0, st, fn->f.ptr( level ) );
   check_cuda( cudaMemcpyAsync( host_packed, st, size_t( n ) * sizeof( double ), cudaMemcpyDeviceToHost, c.stream ), "download" );
   check_cuda( cudaStreamSynchronize( c.stream ), "download sync" );
   HYB_CATCH
}

// L: the caller's level (translated to the storage level here)
// ---------------------------------------------------------------------------------------------
// P2 functions in the reference's own packed layout: the vertex-DoF arrays of level l (the P1
// layout, hyb_layout_*), then every primitive's edge-DoF array (EdgeDoFFunction.cpp:1642-1690 sizes;
// own DoFs at the front: macroedge::index, macroface::index blocks X, XY, Y, macrocell blocks X, Y,
// Z, XY, XZ, YZ, XYZ, EdgeDoFIndexing.hpp:363-373,579-611,922-985).  Every DoF sits on the node set of
// level l+1 where it is stored: vertex DoF v at 2v, the edge DoF of micro-edge (v, v+d) at 2v+d.
// Ghost-layer entries are not maintained and export as zero.
// ---------------------------------------------------------------------------------------------
}  // extern "C"

namespace {
int64_t edge_dof_size( const Topology& t, int kind, int id, int n )
{
   const auto tri  = []( int64_t w ) { return w * ( w + 1 ) / 2; };
   const auto tetw = []( int64_t w ) { return w * ( w + 1 ) * ( w + 2 ) / 6; };
   if ( kind == 0 ) return int64_t( t.v_edges[id].size() + t.v_faces[id].size() );
   if ( kind == 1 )
   {
      const int64_t nf = int64_t( t.e_faces[id].size() ), nc = int64_t( t.e_cells[id].size() );
      return n == 1 ? 1 + 2 * nf + nc : n + nf * ( 3 * n - 1 ) + nc * ( 7 * n - 7 );
   }
   if ( kind == 2 )
   {
      const int64_t nc = int64_t( t.f_cells[id].size() );
      return 3 * tri( n ) + ( nc ? nc * ( 3 * tri( n ) + tri( n - 1 ) + 3 * tri( n - 1 ) ) : 0 );
   }
   return 6 * tetw( n ) + tetw( n - 1 );
}

// visit every own edge DoF of primitive (kind, id) of level l (n = 2^l micro-edges per macro-edge):
// f(index in the primitive's edge-DoF array, storage-local coordinates on level l+1)
template < typename F >
void for_edge_dofs( int kind, int n, F&& f )
{
   if ( kind == 1 )
      for ( int x = 0; x < n; ++x ) f( int64_t( x ), 2 * x + 1, 0, 0 );
   else if ( kind == 2 )
   {
      const int64_t ts = int64_t( n ) * ( n + 1 ) / 2;
      for ( int y = 0; y < n; ++y )
         for ( int x = 0; x + y < n; ++x )
         {
            const int64_t k = fidx( n - 1, x, y );
            f( k, 2 * x + 1, 2 * y, 0 );               // X
            f( ts + k, 2 * x + 1, 2 * y + 1, 0 );      // XY
            f( 2 * ts + k, 2 * x, 2 * y + 1, 0 );      // Y
         }
   }
   else if ( kind == 3 )
   {
      const int64_t tb = tet_size( n );
      for ( int z = 0; z < n; ++z )
         for ( int y = 0; y + z < n; ++y )
            for ( int x = 0; x + y + z < n; ++x )
            {
               const int64_t k = cidx( n - 1, x, y, z );
               f( k, 2 * x + 1, 2 * y, 2 * z );                  // X
               f( tb + k, 2 * x, 2 * y + 1, 2 * z );             // Y
               f( 2 * tb + k, 2 * x, 2 * y, 2 * z + 1 );         // Z
               f( 3 * tb + k, 2 * x + 1, 2 * y + 1, 2 * z );     // XY
               f( 4 * tb + k, 2 * x + 1, 2 * y, 2 * z + 1 );     // XZ
               f( 5 * tb + k, 2 * x, 2 * y + 1, 2 * z + 1 );     // YZ
               if ( x + y + z < n - 1 ) f( 6 * tb + cidx( n - 2, x, y, z ), 2 * x + 1, 2 * y + 1, 2 * z + 1 );  // XYZ
            }
   }
}

// vertex DoFs of the P1 layout of level l: f(index in the primitive's array, storage-local coordinates)
template < typename F >
void for_vertex_dofs( int kind, int n, F&& f )
{
   if ( kind == 0 ) f( int64_t( 0 ), 0, 0, 0 );
   else if ( kind == 1 )
      for ( int x = 0; x <= n; ++x ) f( int64_t( x ), 2 * x, 0, 0 );
   else if ( kind == 2 )
      for ( int y = 0; y <= n; ++y )
         for ( int x = 0; x + y <= n; ++x ) f( fidx( n, x, y ), 2 * x, 2 * y, 0 );
   else
      for ( int z = 0; z <= n; ++z )
         for ( int y = 0; y + z <= n; ++y )
            for ( int x = 0; x + y + z <= n; ++x ) f( cidx( n, x, y, z ), 2 * x, 2 * y, 2 * z );
}

int64_t storage_slot( const P1Level& S, int p, int kind, int X, int Y, int Z )
{
   const int ns = S.n;
   if ( kind == 0 ) return S.off[p];
   if ( kind == 1 ) return S.off[p] + X;
   if ( kind == 2 ) return S.off[p] + fidx( ns, X, Y );
   return S.off[p] + cidx( ns, X, Y, Z );
}

// Slot holding the value of the node at storage-local coordinates (X, Y, Z) of primitive (kind, id).
// Only cell arrays keep copies of every node of their closure, so a lower-dimensional primitive reads
// it from its first neighbour cell: the node's integer barycentric weights on the primitive's
// vertices become cell-local coordinates.
int64_t closure_slot( const Topology& t, const P1Level& S, int kind, int id, int X, int Y, int Z )
{
   const int ns = S.n;
   const int cellbase = t.nV + t.nE + t.nF;
   if ( kind == 3 ) return S.off[cellbase + id] + cidx( ns, X, Y, Z );
   int gv[3], w[3], nv = 0;
   int c = -1;
   if ( kind == 0 )
   {
      gv[0] = id, w[0] = ns, nv = 1;
      c     = t.v_cells[id].empty() ? -1 : t.v_cells[id][0];
   }
   else if ( kind == 1 )
   {
      gv[0] = t.ev[id][0], w[0] = ns - X, gv[1] = t.ev[id][1], w[1] = X, nv = 2;
      c = t.e_cells[id].empty() ? -1 : t.e_cells[id][0];
   }
   else
   {
      gv[0] = t.fv[id][0], w[0] = ns - X - Y, gv[1] = t.fv[id][1], w[1] = X, gv[2] = t.fv[id][2], w[2] = Y, nv = 3;
      c = t.f_cells[id].empty() ? -1 : t.f_cells[id][0];
   }
   require( c >= 0, "primitive without a neighbour cell" );
   int xyz[3] = { 0, 0, 0 };
   for ( int i = 0; i < nv; ++i )
      for ( int d = 1; d < 4; ++d )
         if ( t.cv[c][d] == gv[i] ) xyz[d - 1] = w[i];
   return S.off[cellbase + c] + cidx( ns, xyz[0], xyz[1], xyz[2] );
}

// (kind, id, global primitive index p) in the packed order: vertices, edges, faces, cells
template < typename F >
void for_primitives( const Topology& t, F&& f )
{
   int p = 0;
   for ( int i = 0; i < t.nV; ++i ) f( 0, i, p++ );
   for ( int i = 0; i < t.nE; ++i ) f( 1, i, p++ );
   for ( int i = 0; i < t.nF; ++i ) f( 2, i, p++ );
   for ( int i = 0; i < t.nC; ++i ) f( 3, i, p++ );
}
}  // namespace

extern "C" {

static void pointwise( hyb_fn* dst, int L, uint32_t flag, int op, int n, const double* sc, hyb_fn* const* srcs )
{
   L = lv( dst, L );
   require_level( dst->f, L );
   require( n >= 0 && n <= 3, "at most three source functions" );
   for ( int k = 0; k < n; ++k )
   {
      require( srcs[k] != nullptr, "source function is NULL" );
      same_space( dst, srcs[k] );
      require( srcs[k]->f.mesh == dst->f.mesh, "functions live on different meshes" );
      require( srcs[k]->f.dtype == dst->f.dtype, "functions of different value types (use hyb_fn_copy_from)" );
      require_level( srcs[k]->f, L );
   }
   if ( flag == kAll && op == PT_LINCOMB )
   {
      const void* s[3] = { nullptr, nullptr, nullptr };
      double      a[3] = { 0, 0, 0 };
      for ( int k = 0; k < n; ++k ) s[k] = srcs[k]->f.ptr( L ), a[k] = sc[k];
      if ( n == 0 ) a[0] = sc ? sc[0] : 0.0;
      launch_flat_lincomb( &dst->ctx->c, dst->f.mesh->level( L ).size, dst->f.dtype, dst->f.ptr( L ), n, s, a );
      return;
   }
   PointArgs a{};
   a.op   = op;
   a.flag = flag;
   a.nsrc = n;
   a.s0   = n > 0 ? srcs[0]->f.ptr( L ) : nullptr;
   a.s1   = n > 1 ? srcs[1]->f.ptr( L ) : nullptr;
   a.s2   = n > 2 ? srcs[2]->f.ptr( L ) : nullptr;
   a.dst  = dst->f.ptr( L );
   a.a0   = n > 0 || op == PT_SET ? sc[0] : 0.0;
   a.a1   = n > 1 ? sc[1] : 0.0;
   a.a2   = n > 2 ? sc[2] : 0.0;
   launch_point( &dst->ctx->c, dst->f.mesh, L, dst->f.dtype, a );
}

int hyb_p2_layout_sizes( hyb_mesh* mesh, int level, int64_t* vertex_part, int64_t* edge_part )
{
   HYB_TRY
   require( mesh && vertex_part && edge_part, "NULL argument" );
   require( level >= 0 && level <= 13, "invalid level" );
   *vertex_part = mesh->m.level( level ).packed_size;
   int64_t e    = 0;
   for_primitives( mesh->m.topo, [&]( int kind, int id, int ) { e += edge_dof_size( mesh->m.topo, kind, id, 1 << level ); } );
   *edge_part = e;
   HYB_CATCH
}

int hyb_p2_fn_download_reference( hyb_fn* fn, int level, double* out )
{
   HYB_TRY
   require( fn && out, "NULL argument" );
   require( fn->f.lshift == 1, "not a P2 function" );
   require_level( fn->f, level + 1 );
   const Topology& t  = fn->f.mesh->topo;
   const P1Level&  V  = fn->f.mesh->level( level );      // packed vertex-DoF layout of level l
   const P1Level&  S  = fn->f.mesh->level( level + 1 );  // storage
   const int       n  = 1 << level;
   const auto      st = from_device( fn, level + 1 );
   std::fill( out, out + V.packed_size, 0.0 );
   int64_t eoff = V.packed_size;
   for_primitives( t, [&]( int kind, int id, int p ) {
      const int64_t vb = V.packed_off[p];
      for_vertex_dofs( kind, n, [&]( int64_t k, int X, int Y, int Z ) { out[vb + k] = st[closure_slot( t, S, kind, id, X, Y, Z )]; } );
      const int64_t es = edge_dof_size( t, kind, id, n );
      std::fill( out + eoff, out + eoff + es, 0.0 );
      for_edge_dofs( kind, n, [&]( int64_t k, int X, int Y, int Z ) { out[eoff + k] = st[closure_slot( t, S, kind, id, X, Y, Z )]; } );
      eoff += es;
   } );
   HYB_CATCH
}

int hyb_p2_fn_upload_reference( hyb_fn* fn, int level, const double* in )
{
   HYB_TRY
   require( fn && in, "NULL argument" );
   require( fn->f.lshift == 1, "not a P2 function" );
   require_level( fn->f, level + 1 );
   const Topology& t = fn->f.mesh->topo;
   const P1Level&  V = fn->f.mesh->level( level );
   const P1Level&  S = fn->f.mesh->level( level + 1 );
   const int       n = 1 << level;
   std::vector< double > st( S.size, 0.0 );
   int64_t               eoff = V.packed_size;
   for_primitives( t, [&]( int kind, int id, int p ) {
      const int64_t vb = V.packed_off[p];
      for_vertex_dofs( kind, n, [&]( int64_t k, int X, int Y, int Z ) { st[storage_slot( S, p, kind, X, Y, Z )] = in[vb + k]; } );
      for_edge_dofs( kind, n, [&]( int64_t k, int X, int Y, int Z ) { st[storage_slot( S, p, kind, X, Y, Z )] = in[eoff + k]; } );
      eoff += edge_dof_size( t, kind, id, n );
   } );
   to_device( fn, level + 1, st );
   sync_copies( fn, level + 1 );  // copies in the cell and face arrays take their owners' values
   HYB_CATCH
}

int hyb_fn_interpolate_const( hyb_fn* fn, double value, int level, uint32_t flag )
{
   HYB_TRY
   require( fn, "fn is NULL" );
   level = lv( fn, level );
   require_level( fn->f, level );
   if ( flag == kAll )
   {
      const double a[3] = { value, 0, 0 };
      launch_flat_lincomb( &fn->ctx->c, fn->f.mesh->level( level ).size, fn->f.dtype, fn->f.ptr( level ), 0, nullptr, a );
   }
   else
      pointwise( fn, level - fn->f.lshift, flag, PT_SET, 0, &value, nullptr );  // pointwise takes the caller level
   HYB_CATCH
}

int hyb_fn_interpolate_callback( hyb_fn* fn, double ( *f )( const double*, void* ), void* user, int level, uint32_t flag )
{
   HYB_TRY
   require( fn && f, "NULL argument" );
   level = lv( fn, level );
   require_level( fn->f, level );
   const Topology& t      = fn->f.mesh->topo;
   const P1Level&  P      = fn->f.mesh->level( level );
   const int       n      = P.n;
   auto            padded = from_device( fn, level );
   double          X[3];
   // owned DoFs per primitive, coordinates from the primitive's own map (coordinateFromIndex of
   // VertexDoFMacroVertex/Edge/Face/Cell)
   for ( int v = 0; v < t.nV; ++v )
      if ( t.bc( t.flag_v[v] ) & flag ) padded[P.off[v]] = f( t.vx[v].data(), user );
   for ( int e = 0; e < t.nE; ++e )
   {
      if ( !( t.bc( t.flag_e[e] ) & flag ) ) continue;
      const auto &a = t.vx[t.ev[e][0]], &b = t.vx[t.ev[e][1]];
      for ( int i = 1; i < n; ++i )
      {
         for ( int d = 0; d < 3; ++d ) X[d] = a[d] + ( ( b[d] - a[d] ) * ( 1.0 / n ) ) * i;
         padded[P.off[t.nV + e] + i] = f( X, user );
      }
   }
   for ( int fc = 0; fc < t.nF; ++fc )
   {
      if ( !( t.bc( t.flag_f[fc] ) & flag ) ) continue;
      const auto &a = t.vx[t.fv[fc][0]], &b = t.vx[t.fv[fc][1]], &c = t.vx[t.fv[fc][2]];
      for ( int j = 1; j < n; ++j )
         for ( int i = 1; i + j < n; ++i )
         {
            for ( int d = 0; d < 3; ++d ) X[d] = a[d] + ( ( b[d] - a[d] ) * ( 1.0 / n ) ) * i + ( ( c[d] - a[d] ) * ( 1.0 / n ) ) * j;
            padded[P.off[t.nV + t.nE + fc] + fidx( n, i, j )] = f( X, user );
         }
   }
   for ( int c = 0; c < t.nC; ++c )
   {
      if ( !( t.bc( t.flag_c[c] ) & flag ) ) continue;
      const auto &p0 = t.vx[t.cv[c][0]], &p1 = t.vx[t.cv[c][1]], &p2 = t.vx[t.cv[c][2]], &p3 = t.vx[t.cv[c][3]];
      const int64_t base = P.off[t.nV + t.nE + t.nF + c];
      for ( int z = 1; z < n; ++z )
         for ( int y = 1; y + z < n; ++y )
            for ( int x = 1; x + y + z < n; ++x )
            {
               for ( int d = 0; d < 3; ++d )
                  X[d] = p0[d] + ( ( p1[d] - p0[d] ) * ( 1.0 / n ) ) * x + ( ( p2[d] - p0[d] ) * ( 1.0 / n ) ) * y +
                         ( ( p3[d] - p0[d] ) * ( 1.0 / n ) ) * z;
               padded[base + cidx( n, x, y, z )] = f( X, user );
            }
   }
   to_device( fn, level, padded );
   sync_copies( fn, level );
   HYB_CATCH
}

int hyb_fn_assign( hyb_fn* dst, int n, const double* scalars, hyb_fn* const* srcs, int level, uint32_t flag )
{
   HYB_TRY
   require( dst && ( n == 0 || ( scalars && srcs ) ), "NULL argument" );
   require( n >= 1, "assign needs at least one source" );
   pointwise( dst, level, flag, PT_LINCOMB, n, scalars, srcs );
   HYB_CATCH
}

int hyb_fn_add( hyb_fn* dst, int n, const double* scalars, hyb_fn* const* srcs, int level, uint32_t flag )
{
   HYB_TRY
   require( dst && scalars && srcs && n >= 1, "NULL argument" );
   pointwise( dst, level, flag, PT_ADD, n, scalars, srcs );
   HYB_CATCH
}

int hyb_fn_mult_elementwise( hyb_fn* dst, hyb_fn* a, hyb_fn* b, int level, uint32_t flag )
{
   HYB_TRY
   require( dst && a && b, "NULL argument" );
   hyb_fn* s[2]  = { a, b };
   double  sc[2] = { 1, 1 };
   pointwise( dst, level, flag, PT_MULT, 2, sc, s );
   HYB_CATCH
}

int hyb_fn_invert_elementwise( hyb_fn* fn, int level, uint32_t flag )
{
   HYB_TRY
   require( fn, "fn is NULL" );
   level = lv( fn, level );
   hyb_fn* s[1]  = { fn };
   double  sc[1] = { 1 };
   pointwise( fn, level - fn->f.lshift, flag, PT_INVERT, 1, sc, s );  // pointwise takes the caller level
   HYB_CATCH
}

int hyb_fn_dot( hyb_fn* a, hyb_fn* b, int level, uint32_t flag, double* out )
{
   HYB_TRY
   require( a && b && out, "NULL argument" );
   same_space( a, b );
   level = lv( a, level );
   require( a->f.mesh == b->f.mesh && a->f.dtype == b->f.dtype, "incompatible functions" );
   require_level( a->f, level );
   require_level( b->f, level );
   Context& c = a->ctx->c;
   launch_dot( &c, a->f.mesh, level, a->f.dtype, flag, a->f.ptr( level ), b->f.ptr( level ), c.d_scalars + 32 );
   check_cuda( cudaMemcpyAsync( out, c.d_scalars + 32, sizeof( double ), cudaMemcpyDeviceToHost, c.stream ), "dot readback" );
   check_cuda( cudaStreamSynchronize( c.stream ), "dot sync" );
   HYB_CATCH
}

// Same result as hyb_fn_dot without allocating device memory (fixed static scratch; see
// launch_dot_noalloc for the set-up, the size limit and the overlap rule).
int hyb_fn_dot_noalloc( hyb_fn* a, hyb_fn* b, int level, uint32_t flag, double* out )
{
   HYB_TRY
   require( a && b && out, "NULL argument" );
   same_space( a, b );
   level = lv( a, level );
   require( a->f.mesh == b->f.mesh && a->f.dtype == b->f.dtype, "incompatible functions" );
   require_level( a->f, level );
   require_level( b->f, level );
   set_device( a->ctx->c );
   launch_dot_noalloc( &a->ctx->c, a->f.mesh, level, a->f.dtype, flag, a->f.ptr( level ), b->f.ptr( level ), out );
   HYB_CATCH
}

int hyb_fn_copy_from( hyb_fn* dst, hyb_fn* src, int level )
{
   HYB_TRY
   require( dst && src, "NULL argument" );
   same_space( dst, src );
   level = lv( dst, level );
   require( dst->f.mesh == src->f.mesh, "functions live on different meshes" );
   require_level( dst->f, level );
   require_level( src->f, level );
   launch_convert( &dst->ctx->c, dst->f.mesh->level( level ).size, dst->f.dtype, dst->f.ptr( level ), src->f.dtype,
                   src->f.ptr( level ) );
   HYB_CATCH
}

int hyb_fn_swap( hyb_fn* a, hyb_fn* b, int level )
{
   HYB_TRY
   require( a && b, "NULL argument" );
   same_space( a, b );
   level = lv( a, level );
   require( a->f.mesh == b->f.mesh && a->f.dtype == b->f.dtype, "incompatible functions" );
   require_level( a->f, level );
   require_level( b->f, level );
   std::swap( a->f.data[level - a->f.minL], b->f.data[level - b->f.minL] );
   HYB_CATCH
}

int hyb_fn_device_ptr( hyb_fn* fn, int level, void** ptr, int64_t* nslots )
{
   HYB_TRY
   require( fn, "fn is NULL" );
   level = lv( fn, level );
   require_level( fn->f, level );
   if ( ptr ) *ptr = fn->f.ptr( level );
   if ( nslots ) *nslots = fn->f.mesh->level( level ).size;
   HYB_CATCH
}

int hyb_fn_info( const hyb_fn* fn, int* order, int* dtype, int* min_level, int* max_level )
{
   HYB_TRY
   require( fn, "fn is NULL" );
   if ( order ) *order = 1 + fn->f.lshift;
   if ( dtype ) *dtype = fn->f.dtype;
   if ( min_level ) *min_level = fn->f.minL - fn->f.lshift;
   if ( max_level ) *max_level = fn->f.maxL - fn->f.lshift;
   HYB_CATCH
}

// the host topology of a mesh and the error message of the calling thread, for the data-export file
extern "C" const hyb::Topology* hyb_internal_topology( const hyb_mesh* m ) { return m ? &m->m.topo : nullptr; }
extern "C" const hyb::Topology* hyb_internal_fn_topology( const hyb_fn* fn ) { return &fn->f.mesh->topo; }
extern "C" int64_t hyb_internal_fn_packed_size( const hyb_fn* fn, int level ) { return fn->f.mesh->level( lv( fn, level ) ).packed_size; }
extern "C" void                 hyb_internal_set_error( const char* msg ) { g_err = msg ? msg : ""; }

// ------------------------------------------------------------------------------------------- operators
int hyb_op_create( hyb_ctx* ctx, hyb_mesh* mesh, int kind, int min_level, int max_level, hyb_op** out )
{
   HYB_TRY
   require( ctx && mesh && out, "NULL argument" );
   require( kind == HYB_P1_CONST_LAPLACE || kind == HYB_P1_CONST_MASS || kind == HYB_P2_CONST_LAPLACE, "unknown operator kind" );
   require( min_level >= 0 && min_level <= max_level && max_level <= ( kind == HYB_P2_CONST_LAPLACE ? 13 : 14 ), "invalid level range" );
   set_device( ctx->c );
   const int shift = kind == HYB_P2_CONST_LAPLACE ? 1 : 0;  // P2 level l is stored on storage level l+1
   auto*     h     = new hyb_op();
   h->ctx          = ctx;
   h->o.mesh       = &mesh->m;
   h->o.kind       = kind;
   h->o.order      = 1 + shift;
   h->o.minL       = min_level + shift;
   h->o.maxL       = max_level + shift;
   ctx_ref( ctx );
   mesh_ref( &mesh->m );
   try
   {
      for ( int L = h->o.minL; L <= h->o.maxL; ++L )
      {
         if ( shift ) build_p2_constant_level( &h->o, L );
         else build_operator_level( &h->o, L );
      }
      if ( shift ) ensure_p2_constant_device();
   } catch ( ... )
   {
      op_unref( h );
      throw;
   }
   *out = h;
   HYB_CATCH
}

int hyb_op_create_p2_divkgrad( hyb_ctx* ctx, hyb_mesh* mesh, int min_level, int max_level, const hyb_coeff* k, int blending,
                               hyb_op** out )
{
   HYB_TRY
   require( min_level >= 0 && min_level <= max_level && max_level <= 13, "invalid level range" );
   const int rc = hyb_op_create_divkgrad( ctx, mesh, min_level + 1, max_level + 1, k, blending, out );
   if ( rc != HYB_OK ) return rc;
   ( *out )->o.order = 2;
   ( *out )->o.kind  = HYB_P2_ELEM_DIVKGRAD;
   ensure_p2_constants();
   HYB_CATCH
}

int hyb_op_create_p2_divkgrad_nodal( hyb_ctx* ctx, hyb_mesh* mesh, int min_level, int max_level, const hyb_coeff* k, int blending,
                                     hyb_op** out )
{
   HYB_TRY
   const int rc = hyb_op_create_p2_divkgrad( ctx, mesh, min_level, max_level, k, blending, out );
   if ( rc != HYB_OK ) return rc;
   hyb_op* h     = *out;
   h->o.nodal_k  = true;
   try
   {
      for ( int L = h->o.minL; L <= h->o.maxL; ++L ) set_p2_nodal_coefficient( &ctx->c, &h->o, L, nullptr );
   } catch ( ... )
   {
      *out = nullptr;
      op_unref( h );
      throw;
   }
   HYB_CATCH
}

int hyb_op_create_p2_divkgrad_fn( hyb_ctx* ctx, hyb_mesh* mesh, int min_level, int max_level, hyb_fn* k, int blending, hyb_op** out )
{
   HYB_TRY
   require( ctx && mesh && k && out, "NULL argument" );
   require( k->f.lshift == 1, "the coefficient must be a P2 function" );
   require( k->f.dtype == HYB_F64, "the coefficient function must hold FP64 values" );
   require( &mesh->m == k->f.mesh, "coefficient function and operator live on different meshes" );
   for ( int L = min_level; L <= max_level; ++L ) require_level( k->f, L + 1 );
   const int rc = hyb_op_create_p2_divkgrad( ctx, mesh, min_level, max_level, nullptr, blending, out );
   if ( rc != HYB_OK ) return rc;
   hyb_op* h    = *out;
   h->o.nodal_k = true;
   try
   {
      for ( int L = h->o.minL; L <= h->o.maxL; ++L )
         set_p2_nodal_coefficient( &ctx->c, &h->o, L, static_cast< const double* >( k->f.ptr( L ) ) );
   } catch ( ... )
   {
      *out = nullptr;
      op_unref( h );
      throw;
   }
   HYB_CATCH
}

int hyb_op_store_element_matrices( hyb_op* op )
{
   HYB_TRY
   require( op, "NULL argument" );
   require( op->o.elementwise, "only elementwise operators store element matrices" );
   op->o.store_matrices = true;
   HYB_CATCH
}

int hyb_op_create_divkgrad( hyb_ctx* ctx, hyb_mesh* mesh, int min_level, int max_level, const hyb_coeff* k, int blending,
                            hyb_op** out )
{
   HYB_TRY
   require( ctx && mesh && out, "NULL argument" );
   require( min_level >= 0 && min_level <= max_level && max_level <= 14, "invalid level range" );
   require( blending == HYB_BLEND_NONE || blending == HYB_BLEND_SHELL, "unknown blending" );
   require( !k || k->kind == HYB_COEFF_CONSTANT || k->kind == HYB_COEFF_EXPSIN || k->kind == HYB_COEFF_RADIAL_EXP,
            "unknown coefficient kind" );
   require( !k || k->kind != HYB_COEFF_RADIAL_EXP || k->freq != 0.0, "radial coefficient needs a non-zero scale" );
   set_device( ctx->c );
   auto* h          = new hyb_op();
   h->ctx           = ctx;
   h->o.mesh        = &mesh->m;
   h->o.kind        = HYB_P1_ELEM_DIVKGRAD;
   h->o.minL        = min_level;
   h->o.maxL        = max_level;
   h->o.elementwise = true;
   h->o.blending    = blending;
   if ( k )
   {
      h->o.coeff.kind  = k->kind;
      h->o.coeff.value = k->value;
      h->o.coeff.amp   = k->amp;
      h->o.coeff.freq  = k->freq;
      for ( int d = 0; d < 3; ++d ) h->o.coeff.phase[d] = k->phase[d];
   }
   ctx_ref( ctx );
   mesh_ref( &mesh->m );
   try
   {
      build_elementwise_operator( &h->o );
   } catch ( ... )
   {
      op_unref( h );
      throw;
   }
   *out = h;
   HYB_CATCH
}

int hyb_op_destroy( hyb_op* op )
{
   HYB_TRY
   op_unref( op );
   HYB_CATCH
}

static void check_op_fn( hyb_op* op, hyb_fn* f, int L )
{
   require( f != nullptr, "function is NULL" );
   require( f->f.mesh == op->o.mesh, "function and operator live on different meshes" );
   require( f->f.lshift == op->o.order - 1, "P1 function given to a P2 operator or the other way round" );
   require_level( f->f, L );
   require( L >= op->o.minL && L <= op->o.maxL, "level outside the operator's level range" );
   require( op->o.kind != HYB_P2P1_DIV && op->o.kind != HYB_P2_FULL_VISCOUS,
            "block operators are applied through their own entry points (hyb_p2p1_div_apply, hyb_p2_full_viscous_apply)" );
}

static void stencil( hyb_op* op, int L, int dtype, int code, uint32_t flag, int copy_unflagged, const void* src, const void* v1,
                     void* v2, void* dst, double a0 = 0, double a1 = 0 )
{
   StencilArgs a{};
   a.op             = code;
   a.flag           = flag;
   a.copy_unflagged = copy_unflagged;
   a.src            = src;
   a.v1             = v1;
   a.v2             = v2;
   a.dst            = dst;
   a.a0             = a0;
   a.a1             = a1;
   launch_stencil( &op->ctx->c, op->o.mesh, &op->o, L, dtype, a );
}

int hyb_op_apply( hyb_op* op, hyb_fn* src, hyb_fn* dst, int level, uint32_t flag, int update )
{
   HYB_TRY
   require( op, "op is NULL" );
   level += op->o.order - 1;  // P2 level l is stored on storage level l+1
   check_op_fn( op, src, level );
   check_op_fn( op, dst, level );
   require( src != dst, "src and dst must differ" );
   require( src->f.dtype == dst->f.dtype, "src and dst value types differ" );
   require( update == HYB_REPLACE || update == HYB_ADD, "update must be HYB_REPLACE or HYB_ADD" );
   stencil( op, level, src->f.dtype, update == HYB_ADD ? OP_APPLY_ADD : OP_APPLY, flag, 0, src->f.ptr( level ), nullptr, nullptr,
            dst->f.ptr( level ) );
   HYB_CATCH
}

int hyb_op_smooth_sor( hyb_op* op, hyb_fn* dst, hyb_fn* rhs, double relax, int level, uint32_t flag, int backwards )
{
   HYB_TRY
   require( op, "op is NULL" );
   level += op->o.order - 1;
   check_op_fn( op, dst, level );
   check_op_fn( op, rhs, level );
   require( dst != rhs, "dst and rhs must differ" );
   require( dst->f.dtype == rhs->f.dtype, "value types differ" );
   require( !op->o.elementwise && op->o.order == 1, "Gauss-Seidel / SOR is provided for P1 constant-stencil operators" );
   launch_sor( &op->ctx->c, op->o.mesh, &op->o, level, dst->f.dtype, flag, dst->f.ptr( level ), rhs->f.ptr( level ), relax,
               backwards != 0 );
   HYB_CATCH
}

int hyb_op_smooth_jac( hyb_op* op, hyb_fn* dst, hyb_fn* rhs, hyb_fn* src, double relax, int level, uint32_t flag )
{
   HYB_TRY
   require( op, "op is NULL" );
   level += op->o.order - 1;  // P2 level l is stored on storage level l+1
   check_op_fn( op, dst, level );
   check_op_fn( op, rhs, level );
   check_op_fn( op, src, level );
   require( src != dst, "src and dst must differ" );
   require( src->f.dtype == dst->f.dtype && rhs->f.dtype == dst->f.dtype, "value types differ" );
   stencil( op, level, dst->f.dtype, OP_JAC, flag, 0, src->f.ptr( level ), rhs->f.ptr( level ), nullptr, dst->f.ptr( level ),
            relax );
   HYB_CATCH
}

int hyb_op_inverse_diagonal( hyb_op* op, hyb_fn* out, int level, uint32_t flag )
{
   HYB_TRY
   require( op, "op is NULL" );
   level += op->o.order - 1;  // P2 level l is stored on storage level l+1
   check_op_fn( op, out, level );
   if ( op->o.elementwise )
   {
      ensure_elementwise_level( &op->ctx->c, &op->o, level, F64 );
      const int64_t cnt = op->o.mesh->level( level ).size;
      launch_convert( &op->ctx->c, cnt, out->f.dtype, out->f.ptr( level ), F64, op->o.el[level].d_invd[F64] );
      sync_copies( out, level );
      return HYB_OK;
   }
   if ( op->o.kind == HYB_P2_CONST_LAPLACE )
   {
      auto padded = from_device( out, level );
      p2_constant_inverse_diagonal( &op->o, level, flag, padded );
      to_device( out, level, padded );
      sync_copies( out, level );
      return HYB_OK;
   }
   const OpLevel&  ol = op->o.lv.at( level );
   const P1Level&  P  = op->o.mesh->level( level );
   const Topology& t  = op->o.mesh->topo;
   auto            padded = from_device( out, level );
   const int       n      = P.n;
   for ( const auto& tk : P.tasks )
   {
      const int b = tk[0];
      uint32_t  bc = b < t.nV ? t.bc( t.flag_v[b] ) : b < t.nV + t.nE ? t.bc( t.flag_e[b - t.nV] ) : t.bc( t.flag_f[b - t.nV - t.nE] );
      if ( !( bc & flag ) ) continue;
      const int64_t o = P.off[b] + ( b < t.nV ? 0 : b < t.nV + t.nE ? tk[1] : fidx( n, tk[1], tk[2] ) );
      padded[o]       = ol.invd_b[b];
   }
   for ( int c = 0; c < t.nC; ++c )
   {
      if ( !( t.bc( t.flag_c[c] ) & flag ) ) continue;
      const int64_t base = P.off[P.nB + c];
      for ( int z = 1; z < n; ++z )
         for ( int y = 1; y + z < n; ++y )
            for ( int x = 1; x + y + z < n; ++x ) padded[base + cidx( n, x, y, z )] = ol.invd_c[c];
   }
   to_device( out, level, padded );
   sync_copies( out, level );
   HYB_CATCH
}

int hyb_op_stencil( hyb_op* op, int level, int cell, int cls, double* out15 )
{
   HYB_TRY
   require( op && out15, "NULL argument" );
   require( !op->o.elementwise && op->o.order == 1, "only P1 constant-stencil operators have a 15-point stencil" );
   require( level >= op->o.minL && level <= op->o.maxL, "level outside the operator's level range" );
   require( cell >= 0 && cell < op->o.mesh->topo.nC && cls >= 0 && cls < kNumClasses, "cell or class out of range" );
   const OpLevel& ol = op->o.lv.at( level );
   std::copy( ol.W.begin() + ( size_t( cell ) * kNumClasses + cls ) * kNumDirs,
              ol.W.begin() + ( size_t( cell ) * kNumClasses + cls + 1 ) * kNumDirs, out15 );
   HYB_CATCH
}

// ------------------------------------------------------------------------------------------- transfer
int hyb_restrict( hyb_fn* fn, int source_level, uint32_t flag )
{
   HYB_TRY
   require( fn, "fn is NULL" );
   source_level = lv( fn, source_level );
   require_level( fn->f, source_level );
   require_level( fn->f, source_level - 1 );
   if ( fn->f.lshift )
      launch_p2_restrict( &fn->ctx->c, fn->f.mesh, source_level, fn->f.dtype, flag, fn->f.ptr( source_level ),
                          fn->f.ptr( source_level - 1 ) );
   else
      launch_restrict( &fn->ctx->c, fn->f.mesh, source_level, fn->f.dtype, flag, fn->f.ptr( source_level ),
                       fn->f.ptr( source_level - 1 ) );
   HYB_CATCH
}

int hyb_prolongate( hyb_fn* fn, int source_level, uint32_t flag, int update )
{
   HYB_TRY
   require( fn, "fn is NULL" );
   source_level = lv( fn, source_level );
   require_level( fn->f, source_level );
   require_level( fn->f, source_level + 1 );
   require( update == HYB_REPLACE || update == HYB_ADD, "update must be HYB_REPLACE or HYB_ADD" );
   if ( fn->f.lshift )
      launch_p2_prolongate( &fn->ctx->c, fn->f.mesh, source_level, fn->f.dtype, flag, fn->f.ptr( source_level ),
                            fn->f.ptr( source_level + 1 ), update == HYB_ADD );
   else
      launch_prolongate( &fn->ctx->c, fn->f.mesh, source_level, fn->f.dtype, flag, fn->f.ptr( source_level ),
                         fn->f.ptr( source_level + 1 ), update == HYB_ADD );
   HYB_CATCH
}

}  // extern "C"

// =============================================================================================
// solvers
// =============================================================================================
namespace hyb {

struct FnHolder
{
   hyb_fn* h = nullptr;
   ~FnHolder() { hyb_fn_destroy( h ); }
};

static hyb_fn* new_fn( hyb_ctx* ctx, Mesh* m, int dtype, int minL, int maxL )
{
   hyb_fn* h  = new hyb_fn();
   h->ctx     = ctx;
   h->f.mesh  = m;
   h->f.dtype = dtype;
   h->f.minL  = minL;
   h->f.maxL  = maxL;
   ctx_ref( ctx );
   mesh_ref( m );
   for ( int L = minL; L <= maxL; ++L )
   {
      void* p = nullptr;
      check_cuda( cudaMalloc( &p, h->f.bytes( L ) ), "cudaMalloc(solver temporary)" );
      check_cuda( cudaMemsetAsync( p, 0, h->f.bytes( L ), ctx->c.stream ), "cudaMemset" );
      h->f.data.push_back( p );
   }
   return h;
}

constexpr uint32_t kSolveFlag = kInner | kNeumann | kFreeslip;

// CG on the device; all control scalars stay on the device so the loop can be graph-captured.
struct CGState
{
   hyb_fn* p  = nullptr;
   hyb_fn* ap = nullptr;
   hyb_fn* r  = nullptr;
   double* st = nullptr;  // 16 doubles
};

static void cg_run( hyb_op* op, CGState& s, hyb_fn* x, hyb_fn* b, int L, int maxit, double rtol, double atol, bool host_checks )
{
   Context& c  = op->ctx->c;
   const int dt = x->f.dtype;
   for ( hyb_fn* f : { s.p, s.ap, s.r } )
      check_cuda( cudaMemsetAsync( f->f.ptr( L ), 0, f->f.bytes( L ), c.stream ), "cudaMemset(cg)" );
   // init (CGSolver::init): r = b - A x ; p = r ; prsold = r.r
   stencil( op, L, dt, OP_RESID, kSolveFlag, 0, x->f.ptr( L ), b->f.ptr( L ), nullptr, s.r->f.ptr( L ) );
   {
      PointArgs a{};
      a.op   = PT_LINCOMB;
      a.flag = kSolveFlag;
      a.nsrc = 1;
      a.s0   = s.r->f.ptr( L );
      a.dst  = s.p->f.ptr( L );
      a.a0   = 1.0;
      launch_point( &c, op->o.mesh, L, dt, a );
   }
   launch_dot( &c, op->o.mesh, L, dt, kSolveFlag, s.r->f.ptr( L ), s.r->f.ptr( L ), s.st + 3 );
   launch_cg_scalar( &c, s.st, 0, rtol, atol );
   for ( int it = 0; it < maxit; ++it )
   {
      if ( host_checks && ( it % 8 ) == 0 )
      {
         double done = 0;
         check_cuda( cudaMemcpyAsync( &done, s.st + 6, sizeof( double ), cudaMemcpyDeviceToHost, c.stream ), "cg readback" );
         check_cuda( cudaStreamSynchronize( c.stream ), "cg sync" );
         if ( done != 0.0 ) break;
      }
      stencil( op, L, dt, OP_APPLY, kSolveFlag, 0, s.p->f.ptr( L ), nullptr, nullptr, s.ap->f.ptr( L ) );
      launch_dot( &c, op->o.mesh, L, dt, kSolveFlag, s.p->f.ptr( L ), s.ap->f.ptr( L ), s.st + 2 );
      launch_cg_scalar( &c, s.st, 1, rtol, atol );
      PointArgs a{};
      a.op          = PT_CG_XR;
      a.flag        = kSolveFlag;
      a.s0          = x->f.ptr( L );
      a.s1          = s.p->f.ptr( L );
      a.s2          = s.ap->f.ptr( L );
      a.dst         = s.r->f.ptr( L );
      a.dev_scalars = s.st;
      launch_point( &c, op->o.mesh, L, dt, a );
      launch_dot( &c, op->o.mesh, L, dt, kSolveFlag, s.r->f.ptr( L ), s.r->f.ptr( L ), s.st + 3 );
      launch_cg_scalar( &c, s.st, 2, rtol, atol );
      PointArgs q{};
      q.op          = PT_CG_P;
      q.flag        = kSolveFlag;
      q.s0          = s.r->f.ptr( L );
      q.dst         = s.p->f.ptr( L );
      q.dev_scalars = s.st;
      launch_point( &c, op->o.mesh, L, dt, q );
   }
}

std::vector< double > chebyshev_coefficients( int order, double lower, double upper )
{
   // error polynomial e(t) = T_k((theta - t)/delta) / T_k(theta/delta); x += p(D^-1 A) D^-1 r with
   // 1 - t p(t) = e(t), i.e. p_i = -e_{i+1} (same coefficients as
   // ChebyshevSmoother::setupCoefficientsInternal, ChebyshevSmoother.hpp:329-555)
   if ( order < 1 || order > 16 ) throw std::invalid_argument( "Chebyshev order must be 1..16" );
   if ( !( upper > lower ) || !( lower > 0 ) ) throw std::invalid_argument( "Chebyshev bounds must satisfy 0 < lower < upper" );
   const double theta = 0.5 * ( upper + lower ), delta = 0.5 * ( upper - lower );
   std::vector< std::vector< double > > T = { { 1.0 }, { 0.0, 1.0 } };
   for ( int k = 2; k <= order; ++k )
   {
      std::vector< double > t( k + 1, 0.0 );
      for ( size_t i = 0; i < T[k - 1].size(); ++i ) t[i + 1] += 2 * T[k - 1][i];
      for ( size_t i = 0; i < T[k - 2].size(); ++i ) t[i] -= T[k - 2][i];
      T.push_back( t );
   }
   const auto&           Tk = T[order];
   std::vector< double > poly( order + 1, 0.0 ), pw = { 1.0 };
   for ( int k = 0; k <= order; ++k )
   {
      for ( size_t i = 0; i < pw.size(); ++i ) poly[i] += Tk[k] * pw[i];
      std::vector< double > nx( pw.size() + 1, 0.0 );
      for ( size_t i = 0; i < pw.size(); ++i )
      {
         nx[i] += pw[i] * ( theta / delta );
         nx[i + 1] += pw[i] * ( -1.0 / delta );
      }
      pw = nx;
   }
   double norm = 0, s = theta / delta, sp = 1;
   for ( int k = 0; k <= order; ++k ) norm += Tk[k] * sp, sp *= s;
   std::vector< double > out( order );
   for ( int i = 0; i < order; ++i ) out[i] = -poly[i + 1] / norm;
   return out;
}

}  // namespace hyb

struct hyb_gmg
{
   hyb_ctx*                             ctx = nullptr;
   hyb_op*                              op  = nullptr;
   hyb_gmg_params                       p{};
   int                                  dtype = -1;
   hyb_fn*                              tmp   = nullptr;  // residual per level
   hyb_fn*                              jt    = nullptr;  // Jacobi ping-pong partner of x
   hyb_fn*                              z0    = nullptr;  // Chebyshev temporaries
   hyb_fn*                              z1    = nullptr;
   hyb::CGState                         cg;
   hyb::CGState                         cg64;   // FP64 coarse solve for low-precision hierarchies
   hyb_fn*                              cgx64 = nullptr;
   hyb_fn*                              cgb64 = nullptr;
   // mixed-precision refinement temporaries (inner dtype r and c, fp64 residual)
   hyb_fn*                              mx_r = nullptr;
   hyb_fn*                              mx_c = nullptr;
   hyb_fn*                              mx_t = nullptr;
   std::vector< double >                radii;
   std::vector< std::vector< double > > coeff;
   std::vector< int >                   swaps;  // Jacobi swaps per level in the current cycle
   // CG iterations unrolled into a captured cycle (measured by coarse_probe; -1: not yet)
   int coarse_cap = -1;
   // graph cache
   cudaGraphExec_t gexec   = nullptr;
   void*           g_x     = nullptr;
   void*           g_b     = nullptr;
   int             g_level = -1;
   ~hyb_gmg()
   {
      if ( gexec ) cudaGraphExecDestroy( gexec );
      hyb_fn_destroy( tmp );
      hyb_fn_destroy( jt );
      hyb_fn_destroy( z0 );
      hyb_fn_destroy( z1 );
      hyb_fn_destroy( cg.p );
      hyb_fn_destroy( cg.ap );
      hyb_fn_destroy( cg.r );
      cudaFree( cg.st );
      hyb_fn_destroy( cg64.p );
      hyb_fn_destroy( cg64.ap );
      hyb_fn_destroy( cg64.r );
      cudaFree( cg64.st );
      hyb_fn_destroy( cgx64 );
      hyb_fn_destroy( cgb64 );
      hyb_fn_destroy( mx_r );
      hyb_fn_destroy( mx_c );
      hyb_fn_destroy( mx_t );
      hyb_op*  o = op;
      hyb_ctx* c = ctx;
      op_unref( o );
      ctx_unref( c );
   }
};

namespace hyb {

static void gmg_alloc( hyb_gmg* g, int dtype )
{
   if ( g->dtype == dtype ) return;
   if ( g->dtype >= 0 ) throw std::invalid_argument( "a multigrid solver instance serves one value type" );
   Mesh*     m = g->op->o.mesh;
   const int a = g->p.min_level, b = g->p.max_level;
   g->tmp      = new_fn( g->ctx, m, dtype, a, b );
   if ( g->p.smoother == HYB_SMOOTHER_JACOBI ) g->jt = new_fn( g->ctx, m, dtype, a, b );
   else
   {
      g->z0 = new_fn( g->ctx, m, dtype, a, b );
      g->z1 = new_fn( g->ctx, m, dtype, a, b );
   }
   g->cg.p  = new_fn( g->ctx, m, dtype, a, a );
   g->cg.ap = new_fn( g->ctx, m, dtype, a, a );
   g->cg.r  = new_fn( g->ctx, m, dtype, a, a );
   check_cuda( cudaMalloc( &g->cg.st, 16 * sizeof( double ) ), "cudaMalloc(cg state)" );
   check_cuda( cudaMemsetAsync( g->cg.st, 0, 16 * sizeof( double ), g->ctx->c.stream ), "cudaMemset" );
   if ( dtype != F64 && g->p.coarse_fp64 )
   {
      g->cg64.p  = new_fn( g->ctx, m, F64, a, a );
      g->cg64.ap = new_fn( g->ctx, m, F64, a, a );
      g->cg64.r  = new_fn( g->ctx, m, F64, a, a );
      g->cgx64   = new_fn( g->ctx, m, F64, a, a );
      g->cgb64   = new_fn( g->ctx, m, F64, a, a );
      check_cuda( cudaMalloc( &g->cg64.st, 16 * sizeof( double ) ), "cudaMalloc(cg state)" );
      check_cuda( cudaMemsetAsync( g->cg64.st, 0, 16 * sizeof( double ), g->ctx->c.stream ), "cudaMemset" );
   }
   g->dtype = dtype;
}

static void smooth( hyb_gmg* g, hyb_fn* x, hyb_fn* b, int L )
{
   hyb_op* op = g->op;
   const int dt = x->f.dtype;
   if ( g->p.smoother == HYB_SMOOTHER_GAUSS_SEIDEL || g->p.smoother == HYB_SMOOTHER_SOR )
   {
      // GaussSeidelSmoother::solve -> smooth_gs (relax 1), SORSmoother::solve -> smooth_sor
      const double relax = g->p.smoother == HYB_SMOOTHER_SOR ? g->p.jacobi_relax : 1.0;
      launch_sor( &g->ctx->c, op->o.mesh, &op->o, L, dt, kSolveFlag, x->f.ptr( L ), b->f.ptr( L ), relax, 0 );
      return;
   }
   if ( g->p.smoother == HYB_SMOOTHER_JACOBI )
   {
      // WeightedJacobiSmoother::solve: tmp <- x (All); x <- tmp + w D^-1 (b - A tmp).  The copy is
      // replaced by exchanging the storage of x and its partner; unflagged DoFs are carried over by
      // the sweep itself.
      std::swap( x->f.data[L - x->f.minL], g->jt->f.data[L - g->jt->f.minL] );
      g->swaps[L - g->p.min_level] ^= 1;
      stencil( op, L, dt, OP_JAC, kSolveFlag, 1, g->jt->f.ptr( L ), b->f.ptr( L ), nullptr, x->f.ptr( L ), g->p.jacobi_relax );
      return;
   }
   // ChebyshevSmoother::solve (ChebyshevSmoother.hpp:112-240), fused: step 0 z0 = D^-1 (b - A x),
   // step m z_m = D^-1 A z_{m-1} with x += c_{m-1} z_{m-1}, last step adds c_{k-1} z_{k-1} too.
   const auto& c     = g->coeff.at( L - g->p.min_level );
   const int   order = int( c.size() );
   hyb_fn*     za = g->z0, *zb = g->z1;
   stencil( op, L, dt, OP_CHEB0, kSolveFlag, 1, x->f.ptr( L ), b->f.ptr( L ), nullptr, za->f.ptr( L ) );
   if ( order == 1 )
   {
      PointArgs a{};
      a.op   = PT_ADD;
      a.flag = kSolveFlag;
      a.nsrc = 1;
      a.s0   = za->f.ptr( L );
      a.dst  = x->f.ptr( L );
      a.a0   = c[0];
      launch_point( &g->ctx->c, op->o.mesh, L, dt, a );
      return;
   }
   for ( int m = 1; m < order; ++m )
   {
      if ( m < order - 1 )
      {
         stencil( op, L, dt, OP_CHEBI, kSolveFlag, 1, za->f.ptr( L ), nullptr, x->f.ptr( L ), zb->f.ptr( L ), c[m - 1] );
         std::swap( za, zb );
      }
      else
         stencil( op, L, dt, OP_CHEBL, kSolveFlag, 0, za->f.ptr( L ), nullptr, x->f.ptr( L ), nullptr, c[m - 1], c[m] );
   }
}

// A captured coarse solve launches the kernels of every unrolled iteration even after the
// device-side stopping test has ended it, so captured cycles unroll only the probed iteration
// count (with margin); cycles run with host checks stop on their own and keep coarse_max_iter.
static int coarse_iterations( const hyb_gmg* g, bool host_checks )
{
   return ( host_checks || g->coarse_cap < 0 ) ? g->p.coarse_max_iter : g->coarse_cap;
}

static void cycle_rec( hyb_gmg* g, hyb_fn* x, hyb_fn* b, int L, int invoked, bool host_checks )
{
   hyb_op*   op = g->op;
   Context&  cx = g->ctx->c;
   const int dt = x->f.dtype;
   if ( L == g->p.min_level )
   {
      if ( g->cgx64 )
      {
         // coarse-grid solve in FP64 for a low-precision hierarchy
         const int64_t cnt = x->f.mesh->level( L ).size;
         launch_convert( &cx, cnt, F64, g->cgb64->f.ptr( L ), dt, b->f.ptr( L ) );
         check_cuda( cudaMemsetAsync( g->cgx64->f.ptr( L ), 0, g->cgx64->f.bytes( L ), cx.stream ), "cudaMemset" );
         cg_run( op, g->cg64, g->cgx64, g->cgb64, L, coarse_iterations( g, host_checks ), g->p.coarse_rtol, g->p.coarse_atol,
                 host_checks );
         launch_convert( &cx, cnt, dt, x->f.ptr( L ), F64, g->cgx64->f.ptr( L ) );
      }
      else
         cg_run( op, g->cg, x, b, L, coarse_iterations( g, host_checks ), g->p.coarse_rtol, g->p.coarse_atol, host_checks );
      return;
   }
   const int pre = g->p.pre_smooth + g->p.smooth_increment * ( invoked - L );
   for ( int i = 0; i < pre; ++i ) smooth( g, x, b, L );
   // residual, restricted straight into b on level L-1 (b.assign({1},{tmp},L-1,flag) of the reference)
   stencil( op, L, dt, OP_RESID, kSolveFlag, 0, x->f.ptr( L ), b->f.ptr( L ), nullptr, g->tmp->f.ptr( L ) );
   if ( op->o.order == 2 ) launch_p2_restrict( &cx, op->o.mesh, L, dt, kSolveFlag, g->tmp->f.ptr( L ), b->f.ptr( L - 1 ) );
   else launch_restrict( &cx, op->o.mesh, L, dt, kSolveFlag, g->tmp->f.ptr( L ), b->f.ptr( L - 1 ) );
   check_cuda( cudaMemsetAsync( x->f.ptr( L - 1 ), 0, x->f.bytes( L - 1 ), cx.stream ), "x.interpolate(0)" );
   cycle_rec( g, x, b, L - 1, invoked, host_checks );
   if ( g->p.cycle == HYB_WCYCLE ) cycle_rec( g, x, b, L - 1, invoked, host_checks );
   if ( op->o.order == 2 ) launch_p2_prolongate( &cx, op->o.mesh, L - 1, dt, kSolveFlag, x->f.ptr( L - 1 ), x->f.ptr( L ), 1 );
   else launch_prolongate( &cx, op->o.mesh, L - 1, dt, kSolveFlag, x->f.ptr( L - 1 ), x->f.ptr( L ), 1 );
   const int post = g->p.post_smooth + g->p.smooth_increment * ( invoked - L );
   for ( int i = 0; i < post; ++i ) smooth( g, x, b, L );
}

static void one_cycle( hyb_gmg* g, hyb_fn* x, hyb_fn* b, int L, bool host_checks )
{
   std::fill( g->swaps.begin(), g->swaps.end(), 0 );
   cycle_rec( g, x, b, L, L, host_checks );
   // restore the storage assignment of x so that every cycle (and a captured graph) starts alike
   for ( int l = g->p.min_level; l <= L; ++l )
      if ( g->swaps[l - g->p.min_level] )
      {
         const int64_t count = x->f.mesh->level( l ).size;
         const void*   s[1]  = { x->f.ptr( l ) };
         const double  a[3]  = { 1, 0, 0 };
         launch_flat_lincomb( &g->ctx->c, count, x->f.dtype, g->jt->f.ptr( l ), 1, s, a );
         std::swap( x->f.data[l - x->f.minL], g->jt->f.data[l - g->jt->f.minL] );
      }
}

static void run_cycle( hyb_gmg* g, hyb_fn* x, hyb_fn* b, int L )
{
   Context& cx = g->ctx->c;
   if ( !g->p.use_graph )
   {
      one_cycle( g, x, b, L, true );
      return;
   }
   if ( !( g->gexec && g->g_x == x->f.ptr( L ) && g->g_b == b->f.ptr( L ) && g->g_level == L ) )
   {
      // every lazily created device table must exist before the capture starts
      prepare_device( &cx, g->op->o.mesh, &g->op->o, g->p.min_level, L, x->f.dtype );
      if ( g->gexec ) cudaGraphExecDestroy( g->gexec ), g->gexec = nullptr;
      cudaGraph_t graph;
      check_cuda( cudaStreamBeginCapture( cx.stream, cudaStreamCaptureModeThreadLocal ), "begin capture" );
      try
      {
         one_cycle( g, x, b, L, false );
      } catch ( ... )
      {
         cudaStreamEndCapture( cx.stream, &graph );
         throw;
      }
      check_cuda( cudaStreamEndCapture( cx.stream, &graph ), "end capture" );
      check_cuda( cudaGraphInstantiate( &g->gexec, graph, 0 ), "graph instantiate" );
      cudaGraphDestroy( graph );
      g->g_x     = x->f.ptr( L );
      g->g_b     = b->f.ptr( L );
      g->g_level = L;
   }
   check_cuda( cudaGraphLaunch( g->gexec, cx.stream ), "graph launch" );
   cx.launches += 1;
}

static double residual_norm( hyb_op* op, hyb_fn* x, hyb_fn* b, hyb_fn* tmp, int L, uint32_t flag )
{
   Context& c = op->ctx->c;
   stencil( op, L, x->f.dtype, OP_RESID, flag, 0, x->f.ptr( L ), b->f.ptr( L ), nullptr, tmp->f.ptr( L ) );
   launch_dot( &c, op->o.mesh, L, x->f.dtype, flag, tmp->f.ptr( L ), tmp->f.ptr( L ), c.d_scalars + 40 );
   double r = 0;
   check_cuda( cudaMemcpyAsync( &r, c.d_scalars + 40, sizeof( double ), cudaMemcpyDeviceToHost, c.stream ), "readback" );
   check_cuda( cudaStreamSynchronize( c.stream ), "sync" );
   return std::sqrt( r );
}

static double power_iteration( hyb_op* op, hyb_fn* x, hyb_fn* aux, int L, int iters )
{
   // estimateSpectralRadiusWithPowerIteration on D^-1 A with flag All (SpectrumEstimation.hpp:56-84)
   Context& c  = op->ctx->c;
   const int dt = x->f.dtype;
   const int64_t count = op->o.mesh->level( L ).size;
   auto dot = [&]( hyb_fn* a, hyb_fn* b ) {
      launch_dot( &c, op->o.mesh, L, dt, kAll, a->f.ptr( L ), b->f.ptr( L ), c.d_scalars + 48 );
      double r = 0;
      check_cuda( cudaMemcpyAsync( &r, c.d_scalars + 48, sizeof( double ), cudaMemcpyDeviceToHost, c.stream ), "readback" );
      check_cuda( cudaStreamSynchronize( c.stream ), "sync" );
      return r;
   };
   auto scale = [&]( hyb_fn* dst, hyb_fn* src, double s ) {
      const void*  p[1] = { src->f.ptr( L ) };
      const double a[3] = { s, 0, 0 };
      launch_flat_lincomb( &c, count, dt, dst->f.ptr( L ), 1, p, a );
   };
   double norm = std::sqrt( dot( x, x ) );
   scale( x, x, 1.0 / norm );
   stencil( op, L, dt, OP_DINV_APPLY, kAll, 0, x->f.ptr( L ), nullptr, nullptr, aux->f.ptr( L ) );
   double radius = 0;
   for ( int it = 1; it <= iters; ++it )
   {
      norm = std::sqrt( dot( aux, aux ) );
      scale( x, aux, 1.0 / norm );
      stencil( op, L, dt, OP_DINV_APPLY, kAll, 0, x->f.ptr( L ), nullptr, nullptr, aux->f.ptr( L ) );
      radius = dot( x, aux );
   }
   return radius;
}

static void set_coefficients( hyb_gmg* g )
{
   g->coeff.clear();
   for ( size_t i = 0; i < g->radii.size(); ++i )
   {
      // the multigrid solver's coarsest level is solved by CG, never smoothed; a smoother user that
      // does smooth it (the Stokes velocity smoother) gets its coefficients when the radius is valid
      const double r = g->radii[i];
      if ( i == 0 && !( r > 0 && std::isfinite( r ) ) )
      {
         g->coeff.push_back( {} );
         continue;
      }
      if ( !( r > 0 ) || !std::isfinite( r ) )
         throw std::runtime_error( "spectral radius estimate of level " + std::to_string( g->p.min_level + int( i ) ) +
                                   " is not positive: " + std::to_string( r ) );
      g->coeff.push_back( chebyshev_coefficients( g->p.cheb_order, g->p.cheb_lower_factor * r, g->p.cheb_upper_factor * r ) );
   }
   if ( g->gexec ) cudaGraphExecDestroy( g->gexec ), g->gexec = nullptr;
}

// seeded start vector for the power iteration: uniform in [-1, 1] on every owned DoF
static void seeded_vector( hyb_fn* x, int L, uint64_t seed )
{
   const P1Level&                           P = x->f.mesh->level( L );
   std::vector< double >                    packed( P.packed_size, 0.0 );
   std::mt19937_64                          rng( seed );
   std::uniform_real_distribution< double > U( -1.0, 1.0 );
   for ( auto& v : packed ) v = U( rng );
   hyb_fn_upload( x, L, packed.data() );
}

// Iterations the coarse CG takes to reach coarse_rtol on this hierarchy, measured once on a seeded
// right-hand side (CG iteration counts on a fixed matrix barely depend on the right-hand side);
// captured cycles unroll twice that plus ten, at most coarse_max_iter, and none when the probe
// needed none.
static void coarse_probe( hyb_gmg* g, int dt )
{
   const int L   = g->p.min_level;
   const int pdt = g->cgx64 ? F64 : dt;
   hyb_fn*   xp  = new_fn( g->ctx, g->op->o.mesh, pdt, L, L );
   hyb_fn*   bp  = new_fn( g->ctx, g->op->o.mesh, pdt, L, L );
   try
   {
      seeded_vector( bp, L, 4242u );
      CGState& st = g->cgx64 ? g->cg64 : g->cg;
      cg_run( g->op, st, xp, bp, L, g->p.coarse_max_iter, g->p.coarse_rtol, g->p.coarse_atol, true );
      double   it = 0;
      Context& c  = g->ctx->c;
      check_cuda( cudaMemcpyAsync( &it, st.st + 7, sizeof( double ), cudaMemcpyDeviceToHost, c.stream ), "cg readback" );
      check_cuda( cudaStreamSynchronize( c.stream ), "cg sync" );
      // a coarse problem that is solved before the first iteration (no unknowns, e.g. every
      // coarse DoF on the Dirichlet boundary) needs no unrolled iterations at all
      g->coarse_cap = it == 0.0 ? 0 : std::min( g->p.coarse_max_iter, 2 * int( it ) + 10 );
   } catch ( ... )
   {
      hyb_fn_destroy( xp );
      hyb_fn_destroy( bp );
      throw;
   }
   hyb_fn_destroy( xp );
   hyb_fn_destroy( bp );
}

}  // namespace hyb

extern "C" {

int hyb_gmg_params_default( hyb_gmg_params* p )
{
   HYB_TRY
   require( p, "NULL argument" );
   *p                       = hyb_gmg_params{};
   p->min_level             = 0;
   p->max_level             = 0;
   p->pre_smooth            = 3;
   p->post_smooth           = 3;
   p->smooth_increment      = 0;
   p->cycle                 = HYB_VCYCLE;
   p->smoother              = HYB_SMOOTHER_JACOBI;
   p->jacobi_relax          = 2.0 / 3.0;
   p->cheb_order            = 3;
   p->cheb_upper_factor     = 1.2;
   p->cheb_lower_factor     = 0.3;
   p->cheb_power_iterations = 50;
   p->coarse_max_iter       = 1000;
   p->coarse_rtol           = 1e-14;
   p->coarse_atol           = 1e-16;
   p->use_graph             = 1;
   p->coarse_fp64           = 1;
   HYB_CATCH
}

int hyb_gmg_create( hyb_ctx* ctx, hyb_op* op, const hyb_gmg_params* params, hyb_gmg** out )
{
   HYB_TRY
   require( ctx && op && params && out, "NULL argument" );
   hyb_gmg_params p = *params;
   p.min_level += op->o.order - 1;  // P2 levels are stored one storage level up
   p.max_level += op->o.order - 1;
   require( p.min_level >= op->o.minL && p.max_level <= op->o.maxL && p.min_level <= p.max_level,
            "multigrid levels outside the operator's level range" );
   require( p.smoother == HYB_SMOOTHER_JACOBI || p.smoother == HYB_SMOOTHER_CHEBYSHEV || p.smoother == HYB_SMOOTHER_GAUSS_SEIDEL ||
                p.smoother == HYB_SMOOTHER_SOR,
            "unknown smoother" );
   require( ( p.smoother != HYB_SMOOTHER_GAUSS_SEIDEL && p.smoother != HYB_SMOOTHER_SOR ) || ( !op->o.elementwise && op->o.order == 1 ),
            "Gauss-Seidel / SOR smoothing is provided for P1 constant-stencil operators" );
   require( p.cycle == HYB_VCYCLE || p.cycle == HYB_WCYCLE, "unknown cycle type" );
   require( p.pre_smooth >= 0 && p.post_smooth >= 0 && p.smooth_increment >= 0, "negative smoothing steps" );
   require( p.coarse_max_iter >= 0, "negative coarse iteration count" );
   auto* g = new hyb_gmg();
   g->ctx  = ctx;
   g->op   = op;
   ctx_ref( ctx );
   ++op->refs;
   g->p    = p;
   g->swaps.assign( p.max_level - p.min_level + 1, 0 );
   *out = g;
   HYB_CATCH
}

int hyb_gmg_destroy( hyb_gmg* gmg )
{
   HYB_TRY
   if ( gmg ) cudaStreamSynchronize( gmg->ctx->c.stream );
   delete gmg;
   HYB_CATCH
}

int hyb_gmg_set_radii( hyb_gmg* g, const double* radii )
{
   HYB_TRY
   require( g && radii, "NULL argument" );
   g->radii.assign( radii, radii + ( g->p.max_level - g->p.min_level + 1 ) );
   set_coefficients( g );
   HYB_CATCH
}

// the setup a solver derives from its operator alone (Chebyshev radii, coarse iteration cap),
// copied to another solver of the same operator kind, level range and precision: the copy skips the
// power iterations and the coarse probe and runs the same cycles bit for bit
int hyb_internal_gmg_copy_setup( hyb_gmg* dst, const hyb_gmg* src )
{
   HYB_TRY
   require( dst && src, "NULL argument" );
   require( dst->p.min_level == src->p.min_level && dst->p.max_level == src->p.max_level, "level ranges differ" );
   if ( !src->radii.empty() )
   {
      dst->radii = src->radii;
      set_coefficients( dst );
   }
   dst->coarse_cap = src->coarse_cap;
   HYB_CATCH
}

int hyb_gmg_get_radii( hyb_gmg* g, double* radii )
{
   HYB_TRY
   require( g && radii, "NULL argument" );
   require( !g->radii.empty(), "radii not set yet" );
   std::copy( g->radii.begin(), g->radii.end(), radii );
   HYB_CATCH
}

static void gmg_prepare( hyb_gmg* g, hyb_fn* x, hyb_fn* b, int level )
{
   require( g && x && b, "NULL argument" );
   require( x != b, "x and b must differ" );
   require( x->f.mesh == g->op->o.mesh && b->f.mesh == g->op->o.mesh, "functions live on another mesh" );
   require( x->f.dtype == b->f.dtype, "x and b value types differ" );
   require( level >= g->p.min_level && level <= g->p.max_level, "level outside the multigrid range" );
   require( x->f.minL <= g->p.min_level && x->f.maxL >= level && b->f.minL <= g->p.min_level && b->f.maxL >= level,
            "x and b must hold every level from the coarse level up to `level`" );
   gmg_alloc( g, x->f.dtype );
   if ( g->p.smoother == HYB_SMOOTHER_CHEBYSHEV && g->radii.empty() )
   {
      hyb_fn* v   = new_fn( g->ctx, g->op->o.mesh, x->f.dtype, g->p.min_level, g->p.max_level );
      hyb_fn* aux = new_fn( g->ctx, g->op->o.mesh, x->f.dtype, g->p.min_level, g->p.max_level );
      for ( int L = g->p.min_level; L <= g->p.max_level; ++L )
      {
         seeded_vector( v, L, 1234567u + L );
         g->radii.push_back( power_iteration( g->op, v, aux, L, g->p.cheb_power_iterations ) );
      }
      hyb_fn_destroy( v );
      hyb_fn_destroy( aux );
      set_coefficients( g );
   }
   if ( g->p.use_graph && g->coarse_cap < 0 ) coarse_probe( g, x->f.dtype );
}

int hyb_gmg_solve( hyb_gmg* g, hyb_fn* x, hyb_fn* b, int level )
{
   HYB_TRY
   require( g && x && b, "NULL argument" );
   require( x->f.lshift == g->op->o.order - 1 && b->f.lshift == x->f.lshift, "P1 and P2 objects mixed" );
   level += g->op->o.order - 1;
   gmg_prepare( g, x, b, level );
   run_cycle( g, x, b, level );
   HYB_CATCH
}

int hyb_gmg_smooth( hyb_gmg* g, hyb_fn* x, hyb_fn* b, int level, int iterations )
{
   HYB_TRY
   require( g && x && b, "NULL argument" );
   require( x->f.lshift == g->op->o.order - 1 && b->f.lshift == x->f.lshift, "P1 and P2 objects mixed" );
   require( iterations >= 0, "negative iteration count" );
   level += g->op->o.order - 1;
   gmg_prepare( g, x, b, level );
   require( level > g->p.min_level, "the smoother runs on the levels above the coarsest one" );
   const int li = level - g->p.min_level;
   g->swaps[li] = 0;
   for ( int i = 0; i < iterations; ++i ) smooth( g, x, b, level );
   if ( g->swaps[li] )
   {
      // the last Jacobi sweep wrote the partner buffer: copy back so that x keeps its storage
      const int64_t count = x->f.mesh->level( level ).size;
      const void*   s[1]  = { x->f.ptr( level ) };
      const double  a[3]  = { 1, 0, 0 };
      launch_flat_lincomb( &g->ctx->c, count, x->f.dtype, g->jt->f.ptr( level ), 1, s, a );
      std::swap( x->f.data[level - x->f.minL], g->jt->f.data[level - g->jt->f.minL] );
      g->swaps[li] = 0;
   }
   HYB_CATCH
}

int hyb_gmg_solve_cycles( hyb_gmg* g, hyb_fn* x, hyb_fn* b, int level, int max_cycles, double rtol, double* res_history,
                          int* cycles_done )
{
   HYB_TRY
   require( g && x && b, "NULL argument" );
   require( x->f.lshift == g->op->o.order - 1 && b->f.lshift == x->f.lshift, "P1 and P2 objects mixed" );
   level += g->op->o.order - 1;
   gmg_prepare( g, x, b, level );
   require( max_cycles >= 0, "negative cycle count" );
   double r0   = residual_norm( g->op, x, b, g->tmp, level, kSolveFlag );
   if ( res_history ) res_history[0] = r0;
   int k = 0;
   for ( ; k < max_cycles; ++k )
   {
      run_cycle( g, x, b, level );
      const double r = residual_norm( g->op, x, b, g->tmp, level, kSolveFlag );
      if ( res_history ) res_history[k + 1] = r;
      if ( !std::isfinite( r ) ) throw std::runtime_error( "multigrid diverged: residual is not finite" );
      if ( r0 > 0 && r / r0 < rtol )
      {
         ++k;
         break;
      }
   }
   if ( cycles_done ) *cycles_done = k;
   HYB_CATCH
}

int hyb_estimate_radius( hyb_op* op, hyb_fn* x, hyb_fn* tmp, int level, int iterations, double* radius )
{
   HYB_TRY
   require( op && x && tmp && radius, "NULL argument" );
   level += op->o.order - 1;
   check_op_fn( op, x, level );
   check_op_fn( op, tmp, level );
   require( iterations >= 1, "iterations must be >= 1" );
   *radius = power_iteration( op, x, tmp, level, iterations );
   HYB_CATCH
}

int hyb_chebyshev_coefficients( int order, double lower, double upper, double* out )
{
   HYB_TRY
   require( out, "NULL argument" );
   auto c = chebyshev_coefficients( order, lower, upper );
   std::copy( c.begin(), c.end(), out );
   HYB_CATCH
}

int hyb_cg_solve( hyb_op* op, hyb_fn* x, hyb_fn* b, int level, int max_iter, double rtol, double atol, int* iterations )
{
   HYB_TRY
   require( op && x && b, "NULL argument" );
   level += op->o.order - 1;
   check_op_fn( op, x, level );
   check_op_fn( op, b, level );
   require( x->f.dtype == b->f.dtype, "value types differ" );
   CGState s;
   FnHolder hp, ha, hr;
   hp.h = s.p  = new_fn( op->ctx, op->o.mesh, x->f.dtype, level, level );
   ha.h = s.ap = new_fn( op->ctx, op->o.mesh, x->f.dtype, level, level );
   hr.h = s.r  = new_fn( op->ctx, op->o.mesh, x->f.dtype, level, level );
   check_cuda( cudaMalloc( &s.st, 16 * sizeof( double ) ), "cudaMalloc(cg state)" );
   try
   {
      cg_run( op, s, x, b, level, max_iter, rtol, atol, true );
      double st[16];
      check_cuda( cudaMemcpyAsync( st, s.st, sizeof( st ), cudaMemcpyDeviceToHost, op->ctx->c.stream ), "readback" );
      check_cuda( cudaStreamSynchronize( op->ctx->c.stream ), "sync" );
      if ( iterations ) *iterations = int( st[7] );
   } catch ( ... )
   {
      cudaFree( s.st );
      throw;
   }
   cudaFree( s.st );
   HYB_CATCH
}

int hyb_residual_norm( hyb_op* op, hyb_fn* x, hyb_fn* b, hyb_fn* tmp, int level, uint32_t flag, double* out )
{
   HYB_TRY
   require( op, "op is NULL" );
   level += op->o.order - 1;
   require( op && x && b && tmp && out, "NULL argument" );
   check_op_fn( op, x, level );
   check_op_fn( op, b, level );
   check_op_fn( op, tmp, level );
   *out = residual_norm( op, x, b, tmp, level, flag );
   HYB_CATCH
}

}  // extern "C"

// =============================================================================================
// mixed-precision iterative refinement
// =============================================================================================
namespace hyb {

static double count_owned( Mesh* m, int L, uint32_t flag )
{
   const P1Level&  P = m->level( L );
   const Topology& t = m->topo;
   double          n = 0;
   for ( const auto& tk : P.tasks )
   {
      const int b  = tk[0];
      uint32_t  bc = b < t.nV ? t.bc( t.flag_v[b] ) : b < t.nV + t.nE ? t.bc( t.flag_e[b - t.nV] ) : t.bc( t.flag_f[b - t.nV - t.nE] );
      if ( bc & flag ) n += 1;
   }
   for ( int c = 0; c < t.nC; ++c )
      if ( t.bc( t.flag_c[c] ) & flag ) n += double( P.n_owned_cell );
   return n;
}

}  // namespace hyb

extern "C" int hyb_mixed_solve( hyb_gmg* g, int inner_dtype, hyb_op* op, hyb_fn* x, hyb_fn* b, int level, int inner_cycles,
                                int max_outer, double rtol, double* res_history, int* outer_iters )
{
   HYB_TRY
   require( g && op && x && b, "NULL argument" );
   require( inner_dtype == F32 || inner_dtype == F16 || inner_dtype == F64, "unknown inner dtype" );
   require( x->f.dtype == F64 && b->f.dtype == F64, "x and b must hold FP64 values" );
   require( g->op == op || g->op->o.mesh == op->o.mesh, "inner solver lives on another mesh" );
   require( inner_cycles >= 1 && max_outer >= 0, "invalid iteration counts" );
   require( op->o.order == g->op->o.order, "inner solver and operator of different orders" );
   level += op->o.order - 1;
   check_op_fn( op, x, level );
   check_op_fn( op, b, level );
   require( level >= g->p.min_level && level <= g->p.max_level, "level outside the inner multigrid range" );
   Mesh* m = op->o.mesh;
   if ( !g->mx_r || g->mx_r->f.maxL < level || g->mx_r->f.dtype != inner_dtype )
   {
      hyb_fn_destroy( g->mx_r );
      hyb_fn_destroy( g->mx_c );
      hyb_fn_destroy( g->mx_t );
      g->mx_r = new_fn( g->ctx, m, inner_dtype, g->p.min_level, level );
      g->mx_c = new_fn( g->ctx, m, inner_dtype, g->p.min_level, level );
      g->mx_t = new_fn( g->ctx, m, F64, level, level );
   }
   gmg_prepare( g, g->mx_c, g->mx_r, level );
   Context&      cx    = g->ctx->c;
   const int64_t cnt   = m->level( level ).size;
   const double  nown  = std::max( 1.0, count_owned( m, level, kSolveFlag ) );
   double        r0    = residual_norm( op, x, b, g->mx_t, level, kSolveFlag );
   double        rn    = r0;
   if ( res_history ) res_history[0] = r0;
   int k = 0;
   for ( ; k < max_outer; ++k )
   {
      if ( r0 == 0.0 || rn / r0 < rtol ) break;
      // r (fp64, written by residual_norm into mx_t) -> inner precision, scaled to unit RMS
      const double s = std::sqrt( nown ) / rn;
      launch_convert( &cx, cnt, inner_dtype, g->mx_r->f.ptr( level ), F64, g->mx_t->f.ptr( level ), s );
      check_cuda( cudaMemsetAsync( g->mx_c->f.ptr( level ), 0, g->mx_c->f.bytes( level ), cx.stream ), "cudaMemset" );
      for ( int c = 0; c < inner_cycles; ++c ) run_cycle( g, g->mx_c, g->mx_r, level );
      launch_axpy_to_f64( &cx, cnt, (double*) x->f.ptr( level ), inner_dtype, g->mx_c->f.ptr( level ), 1.0 / s );
      rn = residual_norm( op, x, b, g->mx_t, level, kSolveFlag );
      if ( res_history ) res_history[k + 1] = rn;
      if ( !std::isfinite( rn ) ) throw std::runtime_error( "mixed-precision refinement diverged: residual is not finite" );
   }
   if ( outer_iters ) *outer_iters = k;
   HYB_CATCH
}

// =============================================================================================
// asynchronous pieces used by the serving loop (not part of the public header)
// =============================================================================================
// r = b - A x over the solve flag into tmp, ||r||^2 into d_out (device); no host synchronisation
extern "C" int hyb_internal_residual_async( hyb_op* op, hyb_fn* x, hyb_fn* b, hyb_fn* tmp, int level, double* d_out )
{
   HYB_TRY
   Context& c = op->ctx->c;
   stencil( op, level, x->f.dtype, OP_RESID, kSolveFlag, 0, x->f.ptr( level ), b->f.ptr( level ), nullptr, tmp->f.ptr( level ) );
   launch_dot( &c, op->o.mesh, level, x->f.dtype, kSolveFlag, tmp->f.ptr( level ), tmp->f.ptr( level ), d_out );
   HYB_CATCH
}

// ---------------------------------------------------------------------------------------------
// Replicated meshes: R disjoint copies of one macro mesh as one mesh, so that one launch of every
// multigrid kernel serves the solves of R same-shaped problems (the serving loop's batches).  The
// copy r of vertex v is vertex r nV + v; since edges and faces are ordered by their sorted vertex
// ids and cells by their vertex tuples, the copy r of primitive i of a kind has index r n_kind + i,
// which hyb_internal_mesh_replicate checks.
// ---------------------------------------------------------------------------------------------
extern "C" int hyb_internal_mesh_replicate( hyb_mesh* m, int R, hyb_mesh** out )
{
   HYB_TRY
   require( m && out && R >= 1, "bad arguments" );
   const Topology&                        t = m->m.topo;
   std::vector< std::array< double, 3 > > c;
   std::vector< std::array< int, 4 > >    tets;
   c.reserve( size_t( R ) * t.nV );
   tets.reserve( size_t( R ) * t.nC );
   for ( int r = 0; r < R; ++r )
   {
      for ( int v = 0; v < t.nV; ++v ) c.push_back( t.vx[v] );
      for ( int k = 0; k < t.nC; ++k )
      {
         const auto& cv = t.cv[k];
         tets.push_back( { cv[0] + r * t.nV, cv[1] + r * t.nV, cv[2] + r * t.nV, cv[3] + r * t.nV } );
      }
   }
   make_mesh( static_cast< hyb_ctx* >( m->m.owner_ctx ), c, tets, out );  // throws on failure
   Topology& u = ( *out )->m.topo;
   bool      same = u.nV == R * t.nV && u.nE == R * t.nE && u.nF == R * t.nF && u.nC == R * t.nC;
   for ( int r = 0; r < R && same; ++r )
   {
      for ( int i = 0; i < t.nE && same; ++i ) same = u.ev[r * t.nE + i][0] == t.ev[i][0] + r * t.nV && u.ev[r * t.nE + i][1] == t.ev[i][1] + r * t.nV;
      for ( int i = 0; i < t.nF && same; ++i )
         for ( int k = 0; k < 3; ++k ) same = same && u.fv[r * t.nF + i][k] == t.fv[i][k] + r * t.nV;
      for ( int i = 0; i < t.nC && same; ++i )
         for ( int k = 0; k < 4; ++k ) same = same && u.cv[r * t.nC + i][k] == t.cv[i][k] + r * t.nV;
   }
   if ( !same )
   {
      hyb_mesh_destroy( *out );
      *out = nullptr;
      throw std::logic_error( "replicated mesh does not keep the primitive order copy by copy" );
   }
   for ( int r = 0; r < R; ++r )
   {
      for ( int i = 0; i < t.nV; ++i ) u.flag_v[r * t.nV + i] = t.flag_v[i];
      for ( int i = 0; i < t.nE; ++i ) u.flag_e[r * t.nE + i] = t.flag_e[i];
      for ( int i = 0; i < t.nF; ++i ) u.flag_f[r * t.nF + i] = t.flag_f[i];
      for ( int i = 0; i < t.nC; ++i ) u.flag_c[r * t.nC + i] = t.flag_c[i];
   }
   u.bc_of_flag = t.bc_of_flag;
   u.blending   = t.blending;
   u.shell_rmin = t.shell_rmin;
   u.shell_rmax = t.shell_rmax;
   HYB_CATCH
}

// Maps of copy r of a replicated mesh at storage level Ls: *d_poff the np packed primitive offsets of
// the original mesh, *d_off R x np padded offsets of each copy's primitives in the replicated mesh's
// buffer, *d_tasks the replicated mesh's boundary tasks regrouped copy by copy, each copy padded to
// *tpad tasks (a multiple of 256; padding tasks have x = -1).  Device arrays, freed with cudaFree.
extern "C" int hyb_internal_replica_maps( hyb_mesh* orig, hyb_mesh* uni, int R, int Ls, void** d_poff, void** d_off, void** d_tasks,
                                          int* np_out, int64_t* count, int* tpad_out )
{
   HYB_TRY
   require( orig && uni && R >= 1 && d_poff && d_off && d_tasks && np_out && count && tpad_out, "bad arguments" );
   const Topology& t  = orig->m.topo;
   const Topology& u  = uni->m.topo;
   require( u.nC == R * t.nC, "not a replicated mesh of this copy count" );
   const P1Level&  Po = orig->m.level( Ls );
   const P1Level&  Pu = uni->m.level( Ls );
   const int       np = t.nV + t.nE + t.nF + t.nC;
   const int       kn[4] = { t.nV, t.nE, t.nF, t.nC }, kb[4] = { 0, u.nV, u.nV + u.nE, u.nV + u.nE + u.nF };
   std::vector< int64_t > poff( Po.packed_off.begin(), Po.packed_off.begin() + np ), off( size_t( R ) * np );
   for ( int r = 0; r < R; ++r )
   {
      int j = 0;
      for ( int k = 0; k < 4; ++k )
         for ( int i = 0; i < kn[k]; ++i, ++j ) off[size_t( r ) * np + j] = Pu.off[kb[k] + r * kn[k] + i];
   }
   auto copy_of = [&]( int b ) {
      if ( b < u.nV ) return b / t.nV;
      if ( b < u.nV + u.nE ) return ( b - u.nV ) / t.nE;
      return ( b - u.nV - u.nE ) / t.nF;
   };
   std::vector< std::vector< int4 > > per( R );
   for ( const auto& q : Pu.tasks ) per[copy_of( q[0] )].push_back( make_int4( q[0], q[1], q[2], 0 ) );
   size_t tmax = 0;
   for ( const auto& v : per ) tmax = std::max( tmax, v.size() );
   const int tpad = int( std::max< size_t >( 256, ( tmax + 255 ) / 256 * 256 ) );
   std::vector< int4 > tasks( size_t( R ) * tpad, make_int4( -1, 0, 0, 0 ) );
   for ( int r = 0; r < R; ++r ) std::copy( per[r].begin(), per[r].end(), tasks.begin() + size_t( r ) * tpad );
   auto up = [&]( void** dst, const void* src, size_t bytes ) {
      check_cuda( cudaMalloc( dst, std::max< size_t >( bytes, 16 ) ), "cudaMalloc(replica maps)" );
      check_cuda( cudaMemcpy( *dst, src, bytes, cudaMemcpyHostToDevice ), "upload replica maps" );
   };
   up( d_poff, poff.data(), poff.size() * sizeof( int64_t ) );
   up( d_off, off.data(), off.size() * sizeof( int64_t ) );
   up( d_tasks, tasks.data(), tasks.size() * sizeof( int4 ) );
   *np_out   = np;
   *count    = Po.packed_size;
   *tpad_out = tpad;
   HYB_CATCH
}

// copy r of a function on a replicated mesh <-> a packed device vector in the original mesh's layout
extern "C" int hyb_internal_replica_copy( hyb_fn* ufn, int level, int to_union, const void* d_poff, const void* d_off_r, int np,
                                          int64_t count, double* d_packed )
{
   HYB_TRY
   require( ufn && d_poff && d_off_r && d_packed, "NULL argument" );
   const int Ls = lv( ufn, level );
   require_level( ufn->f, Ls );
   launch_repack_map( &ufn->ctx->c, count, np, static_cast< const int64_t* >( d_poff ), static_cast< const int64_t* >( d_off_r ), ufn->f.dtype,
                      to_union, d_packed, ufn->f.ptr( Ls ) );
   HYB_CATCH
}

// a function's level as a packed device vector and back (no host transfer)
extern "C" int hyb_internal_fn_packed_device( hyb_fn* fn, int level, int to_padded, double* d_packed )
{
   HYB_TRY
   require( fn && d_packed, "NULL argument" );
   const int Ls = lv( fn, level );
   require_level( fn->f, Ls );
   launch_repack( &fn->ctx->c, fn->f.mesh, Ls, fn->f.dtype, to_padded, d_packed, fn->f.ptr( Ls ) );
   HYB_CATCH
}

// residual r = b - A x (flagged DoFs) into tmp and its squared norm per copy into d_out[R]; with x
// NULL, the squared norms of b itself (the initial residual of a zero guess)
extern "C" int hyb_internal_residual_replicas_async( hyb_op* op, hyb_fn* x, hyb_fn* b, hyb_fn* tmp, int level, int R, const void* d_tasks,
                                                     int tpad, double* d_out )
{
   HYB_TRY
   Context&   c  = op->ctx->c;
   const int  dt = b->f.dtype;
   const void* v = b->f.ptr( level );
   if ( x )
   {
      stencil( op, level, dt, OP_RESID, kSolveFlag, 0, x->f.ptr( level ), b->f.ptr( level ), nullptr, tmp->f.ptr( level ) );
      v = tmp->f.ptr( level );
   }
   launch_dot_replicas( &c, op->o.mesh, level, dt, kSolveFlag, v, v, R, static_cast< const int4* >( d_tasks ), tpad, d_out );
   HYB_CATCH
}

// one defect-correction step with the residual already in g->mx_t (FP64) and its norm rn on the
// host: scale and convert, one inner cycle, FP64 update, new residual into g->mx_t and ||r||^2
// into d_out
extern "C" int hyb_internal_mixed_step_async( hyb_gmg* g, int inner_dtype, hyb_op* op, hyb_fn* x, hyb_fn* b, int level, double rn,
                                              double* d_out )
{
   HYB_TRY
   Mesh* m = op->o.mesh;
   if ( !g->mx_r || g->mx_r->f.maxL < level || g->mx_r->f.dtype != inner_dtype )
   {
      hyb_fn_destroy( g->mx_r );
      hyb_fn_destroy( g->mx_c );
      hyb_fn_destroy( g->mx_t );
      g->mx_r = new_fn( g->ctx, m, inner_dtype, g->p.min_level, level );
      g->mx_c = new_fn( g->ctx, m, inner_dtype, g->p.min_level, level );
      g->mx_t = new_fn( g->ctx, m, F64, level, level );
   }
   gmg_prepare( g, g->mx_c, g->mx_r, level );
   Context&      cx  = g->ctx->c;
   const int64_t cnt = m->level( level ).size;
   if ( rn > 0 )
   {
      const double s = std::sqrt( std::max( 1.0, count_owned( m, level, kSolveFlag ) ) ) / rn;
      launch_convert( &cx, cnt, inner_dtype, g->mx_r->f.ptr( level ), F64, g->mx_t->f.ptr( level ), s );
      check_cuda( cudaMemsetAsync( g->mx_c->f.ptr( level ), 0, g->mx_c->f.bytes( level ), cx.stream ), "cudaMemset" );
      run_cycle( g, g->mx_c, g->mx_r, level );
      launch_axpy_to_f64( &cx, cnt, (double*) x->f.ptr( level ), inner_dtype, g->mx_c->f.ptr( level ), 1.0 / s );
   }
   stencil( op, level, F64, OP_RESID, kSolveFlag, 0, x->f.ptr( level ), b->f.ptr( level ), nullptr, g->mx_t->f.ptr( level ) );
   launch_dot( &cx, m, level, F64, kSolveFlag, g->mx_t->f.ptr( level ), g->mx_t->f.ptr( level ), d_out );
   HYB_CATCH
}

// fill every owned DoF (and its copies) of one level with seeded uniform values in [-1, 1]
extern "C" int hyb_fn_fill_random( hyb_fn* fn, int level, uint64_t seed )
{
   HYB_TRY
   require( fn, "fn is NULL" );
   level = lv( fn, level );
   require_level( fn->f, level );
   launch_fill_uniform( &fn->ctx->c, fn->f.mesh->level( level ).size, fn->f.dtype, fn->f.ptr( level ), seed );
   sync_copies( fn, level );
   HYB_CATCH
}

// =============================================================================================
// P2-P1 Taylor-Hood Stokes: coupling blocks, pressure scaling and Uzawa multigrid
// =============================================================================================
extern "C" {

int hyb_op_create_p2p1_div( hyb_ctx* ctx, hyb_mesh* mesh, int min_level, int max_level, int blending, hyb_op** out )
{
   HYB_TRY
   require( min_level >= 0 && min_level <= max_level && max_level <= 12, "invalid level range" );
   const int rc = hyb_op_create_divkgrad( ctx, mesh, min_level + 1, max_level + 1, nullptr, blending, out );
   if ( rc != HYB_OK ) return rc;
   ( *out )->o.order = 2;
   ( *out )->o.kind  = HYB_P2P1_DIV;
   ensure_stokes_constants();
   HYB_CATCH
}

static void stokes_blocks_check( hyb_op* d, hyb_fn* const* u, hyb_fn* p, int level )
{
   require( d && u && p && u[0] && u[1] && u[2], "NULL argument" );
   require( d->o.kind == HYB_P2P1_DIV, "not a P2-P1 coupling operator" );
   require( p->f.lshift == 0, "the pressure must be a P1 function" );
   for ( int k = 0; k < 3; ++k )
   {
      require( u[k]->f.lshift == 1, "velocity components must be P2 functions" );
      require( u[k]->f.dtype == p->f.dtype, "velocity and pressure value types differ" );
      require( u[k]->f.mesh == &d->o.mesh[0] || u[k]->f.mesh == d->o.mesh, "functions live on another mesh" );
      require_level( u[k]->f, level + 1 );
   }
   require_level( p->f, level );
   require( level + 1 >= d->o.minL && level + 1 <= d->o.maxL, "level outside the operator's range" );
}

int hyb_p2p1_div_apply( hyb_op* d, hyb_fn* const* u, hyb_fn* p, int level, uint32_t flag, int update )
{
   HYB_TRY
   stokes_blocks_check( d, u, p, level );
   const void* uu[3] = { u[0]->f.ptr( level + 1 ), u[1]->f.ptr( level + 1 ), u[2]->f.ptr( level + 1 ) };
   launch_stokes_div( &d->ctx->c, &d->o, level, p->f.dtype, 0, uu, nullptr, nullptr, p->f.ptr( level ), flag, update == HYB_ADD );
   HYB_CATCH
}

int hyb_p1p2_divt_apply( hyb_op* d, hyb_fn* p, hyb_fn* const* u, int level, uint32_t flag, int update )
{
   HYB_TRY
   stokes_blocks_check( d, u, p, level );
   void* uu[3] = { u[0]->f.ptr( level + 1 ), u[1]->f.ptr( level + 1 ), u[2]->f.ptr( level + 1 ) };
   launch_stokes_div( &d->ctx->c, &d->o, level, p->f.dtype, 1, nullptr, p->f.ptr( level ), uu, nullptr, flag, update == HYB_ADD );
   HYB_CATCH
}

int hyb_op_create_p2_full_viscous( hyb_ctx* ctx, hyb_mesh* mesh, int min_level, int max_level, const hyb_coeff* viscosity, int blending,
                                   hyb_op** out )
{
   HYB_TRY
   require( min_level >= 0 && min_level <= max_level && max_level <= 12, "invalid level range" );
   const int rc = hyb_op_create_divkgrad( ctx, mesh, min_level + 1, max_level + 1, viscosity, blending, out );
   if ( rc != HYB_OK ) return rc;
   ( *out )->o.order = 2;
   ( *out )->o.kind  = HYB_P2_FULL_VISCOUS;
   HYB_CATCH
}

static void visc_fns_check( hyb_op* op, hyb_fn* const* u, int level )
{
   require( op && u && u[0] && u[1] && u[2], "NULL argument" );
   require( op->o.kind == HYB_P2_FULL_VISCOUS, "not a full viscous operator" );
   for ( int k = 0; k < 3; ++k )
   {
      require( u[k]->f.lshift == 1, "velocity components must be P2 functions" );
      require( u[k]->f.dtype == u[0]->f.dtype, "component value types differ" );
      require( u[k]->f.mesh == op->o.mesh, "functions live on another mesh" );
      require_level( u[k]->f, level + 1 );
   }
   require( level + 1 >= op->o.minL && level + 1 <= op->o.maxL, "level outside the operator's range" );
}

int hyb_p2_full_viscous_apply( hyb_op* op, hyb_fn* const* src, hyb_fn* const* dst, int level, uint32_t flag, int update )
{
   HYB_TRY
   visc_fns_check( op, src, level );
   visc_fns_check( op, dst, level );
   require( src[0]->f.dtype == dst[0]->f.dtype, "src and dst value types differ" );
   require( update == HYB_REPLACE || update == HYB_ADD, "update must be HYB_REPLACE or HYB_ADD" );
   for ( int i = 0; i < 3; ++i )
      for ( int j = 0; j < 3; ++j ) require( src[i] != dst[j], "src and dst must differ" );
   const int   Ls    = level + 1;
   const void* u[3]  = { src[0]->f.ptr( Ls ), src[1]->f.ptr( Ls ), src[2]->f.ptr( Ls ) };
   void*       d[3]  = { dst[0]->f.ptr( Ls ), dst[1]->f.ptr( Ls ), dst[2]->f.ptr( Ls ) };
   launch_full_viscous( &op->ctx->c, &op->o, level, src[0]->f.dtype, 0, u, d, flag, update == HYB_ADD );
   HYB_CATCH
}

int hyb_p2_full_viscous_inverse_diagonal( hyb_op* op, hyb_fn* const* out, int level )
{
   HYB_TRY
   visc_fns_check( op, out, level );
   const int     Ls  = level + 1;
   ElemLevel&    e   = op->o.el[Ls];
   const int64_t cnt = op->o.mesh->level( Ls ).size;
   if ( !e.d_invd[F64] )
   {
      // the inverse diagonals of the three diagonal blocks, FP64, computed once per level
      void* p = nullptr;
      check_cuda( cudaMalloc( &p, size_t( 3 * cnt ) * sizeof( double ) ), "cudaMalloc(inverse diagonal)" );
      e.d_invd[F64] = p;
      double* dd    = reinterpret_cast< double* >( p );
      void*   d[3]  = { dd, dd + cnt, dd + 2 * cnt };
      launch_full_viscous( &op->ctx->c, &op->o, level, F64, 1, nullptr, d, kAll, 0 );
   }
   const double* dd = reinterpret_cast< const double* >( e.d_invd[F64] );
   for ( int k = 0; k < 3; ++k )
   {
      launch_convert( &op->ctx->c, cnt, out[k]->f.dtype, out[k]->f.ptr( Ls ), F64, dd + k * cnt );
      sync_copies( out[k], Ls );
   }
   HYB_CATCH
}

int hyb_op_create_p1_pspg( hyb_ctx* ctx, hyb_mesh* mesh, int min_level, int max_level, hyb_op** out )
{
   HYB_TRY
   hyb_coeff k{};
   const int rc = hyb_op_create_divkgrad( ctx, mesh, min_level, max_level, nullptr, HYB_BLEND_NONE, out );
   if ( rc != HYB_OK ) return rc;
   ( *out )->o.coeff.kind = kCoeffPSPG;
   ( *out )->o.kind       = HYB_P1_PSPG;
   (void) k;
   HYB_CATCH
}

}  // extern "C"

namespace {
// a nested entry point's failure, rethrown with its message
void ok_rc( int rc )
{
   if ( rc == HYB_EINVAL ) throw std::invalid_argument( g_err );
   if ( rc != HYB_OK ) throw std::runtime_error( g_err );
}

// dot product of two functions on user level l (flagged owned DoFs), read back to the host
double dot_host( hyb_fn* a, hyb_fn* b, int l, uint32_t flag )
{
   double r = 0;
   ok_rc( hyb_fn_dot( a, b, l, flag, &r ) );
   return r;
}
}  // namespace

struct hyb_stokes
{
   hyb_ctx*          ctx  = nullptr;
   hyb_mesh*         mesh = nullptr;
   hyb_stokes_params p{};
   hyb_op*           A    = nullptr;  // velocity block, one component: P2 -div(eta grad)
   hyb_op*           D    = nullptr;  // div / divT
   hyb_op*           S    = nullptr;  // P1 PSPG, for its inverted diagonal
   hyb_gmg*          vel  = nullptr;  // Chebyshev velocity smoother (radii, coefficients, work vectors)
   hyb_fn*           ru[3] = { nullptr, nullptr, nullptr };
   hyb_fn*           rp    = nullptr;
   hyb_fn*           sinv  = nullptr;  // inverted PSPG diagonal on every level
   int               dtype = -1;
   // full viscous velocity block (velocity_block 1): the coupled operator, Chebyshev on it with the
   // inverse diagonals of its diagonal blocks, work vectors z and t, radii and coefficients per level
   hyb_op*                              V = nullptr;
   hyb_fn*                              vz[3]    = { nullptr, nullptr, nullptr };
   hyb_fn*                              vt[3]    = { nullptr, nullptr, nullptr };
   hyb_fn*                              vinvd[3] = { nullptr, nullptr, nullptr };
   std::vector< double >                vradii;
   std::vector< std::vector< double > > vcoef;
   // captured V-cycle: the graph of the last (functions, level) key, captured on the key's second
   // cycle (the first one creates every lazily allocated buffer outside the capture)
   cudaGraphExec_t              gexec = nullptr;
   std::vector< const void* >   gkey;
   // defect correction: the inner solver's iterate and right-hand side (u0-2, bu0-2, p, bp), kept
   // between calls with the same inner solver, level and value type so that its captured cycle stays valid
   hyb_fn*     mx[8]    = { nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr };
   hyb_stokes* mx_inner = nullptr;
   int         mx_dtype = -1, mx_level = -1;
   ~hyb_stokes()
   {
      if ( gexec ) cudaGraphExecDestroy( gexec );
      for ( hyb_fn* f : mx ) hyb_fn_destroy( f );
      for ( hyb_fn* f : ru ) hyb_fn_destroy( f );
      for ( int k = 0; k < 3; ++k )
      {
         hyb_fn_destroy( vz[k] );
         hyb_fn_destroy( vt[k] );
         hyb_fn_destroy( vinvd[k] );
      }
      hyb_fn_destroy( rp );
      hyb_fn_destroy( sinv );
      if ( vel ) hyb_gmg_destroy( vel );
      op_unref( V );
      op_unref( A );
      op_unref( D );
      op_unref( S );
      if ( ctx ) ctx_unref( ctx );
   }
};

namespace {
void stokes_fns_check( hyb_stokes* s, hyb_fn* const* u, hyb_fn* p, int level )
{
   require( s && u && p, "NULL argument" );
   for ( int k = 0; k < 3; ++k )
   {
      require( u[k] && u[k]->f.lshift == 1, "velocity components must be P2 functions" );
      require( u[k]->f.mesh == &s->mesh->m, "functions live on another mesh" );
      require( u[k]->f.dtype == p->f.dtype, "value types differ" );
      require( u[k]->f.minL <= s->p.min_level + 1 && u[k]->f.maxL >= level + 1, "velocity must hold the multigrid levels" );
   }
   require( p->f.lshift == 0 && p->f.mesh == &s->mesh->m, "the pressure must be a P1 function on the solver's mesh" );
   require( p->f.minL <= s->p.min_level && p->f.maxL >= level, "pressure must hold the multigrid levels" );
   require( level >= s->p.min_level && level <= s->p.max_level, "level outside the multigrid range" );
}

// Chebyshev coefficients of the coupled velocity block from per-level radii (bounds 0.3 and 1.2
// times the radius, as the scalar smoother)
void visc_set_radii( hyb_stokes* s, const double* radii )
{
   const int nl = s->p.max_level - s->p.min_level + 1;
   s->vradii.assign( radii, radii + nl );
   s->vcoef.clear();
   for ( int i = 0; i < nl; ++i )
   {
      const double r = s->vradii[i];
      if ( !( r > 0 ) || !std::isfinite( r ) )
         throw std::runtime_error( "spectral radius estimate of level " + std::to_string( s->p.min_level + i ) + " is not positive" );
      s->vcoef.push_back( chebyshev_coefficients( s->p.cheb_order, 0.3 * r, 1.2 * r ) );
   }
}

// D^-1 A of the coupled block on all DoFs (flag All), x -> aux
void visc_dinv_apply( hyb_stokes* s, hyb_fn* const* x, hyb_fn* const* aux, int l )
{
   const int   Ls    = l + 1;
   const void* xx[3] = { x[0]->f.ptr( Ls ), x[1]->f.ptr( Ls ), x[2]->f.ptr( Ls ) };
   void*       aa[3] = { aux[0]->f.ptr( Ls ), aux[1]->f.ptr( Ls ), aux[2]->f.ptr( Ls ) };
   launch_full_viscous( &s->ctx->c, &s->V->o, l, x[0]->f.dtype, 0, xx, aa, kAll, 0 );
   const double one[2] = { 1.0, 1.0 };
   for ( int k = 0; k < 3; ++k )
   {
      hyb_fn* src[2] = { s->vinvd[k], aux[k] };
      pointwise( aux[k], l, kAll, PT_MULT, 2, one, src );
   }
}

// spectral radius of D^-1 A of the coupled block: the scalar power iteration (SpectrumEstimation.hpp:
// 56-84, flag All) with norms and Rayleigh quotient summed over the three components; seeded start
void visc_power_iteration_impl( hyb_stokes* s, int l, int iters, double* out )
{
   hyb_fn** x = s->vz;
   hyb_fn** a = s->vt;
   for ( int k = 0; k < 3; ++k ) ok_rc( hyb_fn_fill_random( x[k], l, 7001u + 31u * uint64_t( l ) + uint64_t( k ) ) );
   auto vdot = [&]( hyb_fn** p, hyb_fn** q ) {
      double r = 0;
      for ( int k = 0; k < 3; ++k ) r += dot_host( p[k], q[k], l, kAll );
      return r;
   };
   auto scale = [&]( hyb_fn** dst, hyb_fn** src, double f ) {
      const double c[1] = { f };
      for ( int k = 0; k < 3; ++k )
      {
         hyb_fn* sr[1] = { src[k] };
         pointwise( dst[k], l, kAll, PT_LINCOMB, 1, c, sr );
      }
   };
   double norm = std::sqrt( vdot( x, x ) );
   scale( x, x, 1.0 / norm );
   visc_dinv_apply( s, x, a, l );
   double radius = 0;
   for ( int it = 1; it <= iters; ++it )
   {
      norm = std::sqrt( vdot( a, a ) );
      scale( x, a, 1.0 / norm );
      visc_dinv_apply( s, x, a, l );
      radius = vdot( x, a );
   }
   *out = radius;
}

double visc_power_iteration( hyb_stokes* s, int l, int iters )
{
   double r = 0;
   visc_power_iteration_impl( s, l, iters, &r );
   return r;
}

// ChebyshevSmoother::solve on the coupled velocity block: z = D^-1 (r - A u), u += c_0 z, then
// z = D^-1 A z, u += c_m z; z starts as a copy of u so that its unflagged entries are u's
void visc_smooth( hyb_stokes* s, hyb_fn* const* u, hyb_fn* const* r, int l )
{
   Context&     cx = s->ctx->c;
   const int    Ls = l + 1, dt = u[0]->f.dtype;
   const auto&  c  = s->vcoef.at( l - s->p.min_level );
   const double one[2] = { 1.0, 1.0 }, pm[2] = { 1.0, -1.0 };
   void*        tt[3]  = { s->vt[0]->f.ptr( Ls ), s->vt[1]->f.ptr( Ls ), s->vt[2]->f.ptr( Ls ) };
   const void*  uu[3]  = { u[0]->f.ptr( Ls ), u[1]->f.ptr( Ls ), u[2]->f.ptr( Ls ) };
   const void*  zz[3]  = { s->vz[0]->f.ptr( Ls ), s->vz[1]->f.ptr( Ls ), s->vz[2]->f.ptr( Ls ) };
   for ( int k = 0; k < 3; ++k )
   {
      hyb_fn* src[1] = { u[k] };
      pointwise( s->vz[k], l, kAll, PT_LINCOMB, 1, one, src );
   }
   launch_full_viscous( &cx, &s->V->o, l, dt, 0, uu, tt, kSolveFlag, 0 );
   for ( int k = 0; k < 3; ++k )
   {
      hyb_fn* d[2] = { r[k], s->vt[k] };
      pointwise( s->vt[k], l, kSolveFlag, PT_LINCOMB, 2, pm, d );
      hyb_fn* q[2] = { s->vinvd[k], s->vt[k] };
      pointwise( s->vz[k], l, kSolveFlag, PT_MULT, 2, one, q );
      const double c0[1] = { c[0] };
      hyb_fn*      z[1]  = { s->vz[k] };
      pointwise( u[k], l, kSolveFlag, PT_ADD, 1, c0, z );
   }
   for ( size_t m = 1; m < c.size(); ++m )
   {
      launch_full_viscous( &cx, &s->V->o, l, dt, 0, zz, tt, kSolveFlag, 0 );
      for ( int k = 0; k < 3; ++k )
      {
         hyb_fn* q[2] = { s->vinvd[k], s->vt[k] };
         pointwise( s->vz[k], l, kSolveFlag, PT_MULT, 2, one, q );
         const double cm[1] = { c[m] };
         hyb_fn*      z[1]  = { s->vz[k] };
         pointwise( u[k], l, kSolveFlag, PT_ADD, 1, cm, z );
      }
   }
}

// work vectors and the solver setup in the value type of the functions
void stokes_prepare( hyb_stokes* s, hyb_fn* u0, hyb_fn* b0, int dt )
{
   if ( s->dtype == dt ) return;
   require( s->dtype < 0, "a Stokes solver serves one value type" );
   Mesh* m = &s->mesh->m;
   for ( int k = 0; k < 3; ++k )
   {
      s->ru[k]           = new_fn( s->ctx, m, dt, s->p.min_level + 1, s->p.max_level + 1 );
      s->ru[k]->f.lshift = 1;
   }
   s->rp   = new_fn( s->ctx, m, dt, s->p.min_level, s->p.max_level );
   s->sinv = new_fn( s->ctx, m, dt, s->p.min_level, s->p.max_level );
   for ( int L = s->p.min_level; L <= s->p.max_level; ++L ) ok_rc( hyb_op_inverse_diagonal( s->S, s->sinv, L, kAll ) );
   if ( s->V )
   {
      for ( int k = 0; k < 3; ++k )
      {
         hyb_fn** f[3] = { &s->vz[k], &s->vt[k], &s->vinvd[k] };
         for ( hyb_fn** g : f )
         {
            *g             = new_fn( s->ctx, m, dt, s->p.min_level + 1, s->p.max_level + 1 );
            ( *g )->f.lshift = 1;
         }
      }
      for ( int L = s->p.min_level; L <= s->p.max_level; ++L ) ok_rc( hyb_p2_full_viscous_inverse_diagonal( s->V, s->vinvd, L ) );
      if ( s->vradii.empty() )
      {
         std::vector< double > r;
         for ( int L = s->p.min_level; L <= s->p.max_level; ++L ) r.push_back( visc_power_iteration( s, L, s->p.power_iterations ) );
         visc_set_radii( s, r.data() );
      }
      s->dtype = dt;
      return;
   }
   // radii of the velocity block (power iteration on D^-1 A per level, once)
   gmg_prepare( s->vel, u0, b0, s->p.max_level + 1 );
   s->dtype = dt;
}

// UzawaSmoother::uzawaSmooth, block-Laplace variant without stabilisation (UzawaSmoother.hpp:
// 321-441): r_u = b_u - divT p; velocity smoothing on A with r_u; r_p = b_p - div u; p += omega
// S^-1 r_p with S^-1 the inverted PSPG diagonal
void uzawa_smooth( hyb_stokes* s, hyb_fn* const* u, hyb_fn* p, hyb_fn* const* bu, hyb_fn* bp, int l )
{
   Context&  cx = s->ctx->c;
   const int Ls = l + 1, dt = p->f.dtype;
   void*     rr[3] = { s->ru[0]->f.ptr( Ls ), s->ru[1]->f.ptr( Ls ), s->ru[2]->f.ptr( Ls ) };
   launch_stokes_div( &cx, &s->D->o, l, dt, 1, nullptr, p->f.ptr( l ), rr, nullptr, kSolveFlag, 0 );
   const double sc[2] = { 1.0, -1.0 };
   for ( int k = 0; k < 3; ++k )
   {
      hyb_fn* src[2] = { bu[k], s->ru[k] };
      pointwise( s->ru[k], l, kSolveFlag, PT_LINCOMB, 2, sc, src );
   }
   for ( int it = 0; it < s->p.velocity_sweeps; ++it )
   {
      if ( s->V )
      {
         visc_smooth( s, u, s->ru, l );
         continue;
      }
      for ( int k = 0; k < 3; ++k ) smooth( s->vel, u[k], s->ru[k], Ls );
   }
   const void* uu[3] = { u[0]->f.ptr( Ls ), u[1]->f.ptr( Ls ), u[2]->f.ptr( Ls ) };
   launch_stokes_div( &cx, &s->D->o, l, dt, 0, uu, nullptr, nullptr, s->rp->f.ptr( l ), kAll, 0 );
   {
      hyb_fn* src[2] = { bp, s->rp };
      pointwise( s->rp, l, kAll, PT_LINCOMB, 2, sc, src );
   }
   {
      const double one[2]  = { 1.0, 1.0 };  // PT_MULT reads no scalar, but the argument block is filled from the array
      hyb_fn*      src[2] = { s->sinv, s->rp };
      pointwise( s->rp, l, kAll, PT_MULT, 2, one, src );
   }
   {
      const double om[1]  = { s->p.omega };
      hyb_fn*      src[1] = { s->rp };
      pointwise( p, l, kAll, PT_ADD, 1, om, src );
   }
}

// residual of the saddle-point system into ru / rp: r_u = b_u - A u - divT p, r_p = b_p - div u
void stokes_residual( hyb_stokes* s, hyb_fn* const* u, hyb_fn* p, hyb_fn* const* bu, hyb_fn* bp, int l )
{
   Context&  cx = s->ctx->c;
   const int Ls = l + 1, dt = p->f.dtype;
   void*     rr[3] = { s->ru[0]->f.ptr( Ls ), s->ru[1]->f.ptr( Ls ), s->ru[2]->f.ptr( Ls ) };
   if ( s->V )
   {
      const void*  uu[3] = { u[0]->f.ptr( Ls ), u[1]->f.ptr( Ls ), u[2]->f.ptr( Ls ) };
      const double pm[2] = { 1.0, -1.0 };
      launch_full_viscous( &cx, &s->V->o, l, dt, 0, uu, rr, kSolveFlag, 0 );
      for ( int k = 0; k < 3; ++k )
      {
         hyb_fn* d[2] = { bu[k], s->ru[k] };
         pointwise( s->ru[k], l, kSolveFlag, PT_LINCOMB, 2, pm, d );
      }
   }
   else
      for ( int k = 0; k < 3; ++k )
         stencil( s->A, Ls, dt, OP_RESID, kSolveFlag, 0, u[k]->f.ptr( Ls ), bu[k]->f.ptr( Ls ), nullptr, rr[k] );
   // r_u -= divT p: divT into rp's partner is not available, so subtract through a scaled add
   const double sc[2] = { 1.0, -1.0 };
   {
      // p_neg = -p is not stored: divT is linear, so r_u += divT(-p) == r_u - divT p; use the
      // pressure work vector for -p
      const double m1[1]  = { -1.0 };
      hyb_fn*      src[1] = { p };
      pointwise( s->rp, l, kAll, PT_LINCOMB, 1, m1, src );
      launch_stokes_div( &cx, &s->D->o, l, dt, 1, nullptr, s->rp->f.ptr( l ), rr, nullptr, kSolveFlag, 1 );
   }
   const void* uu[3] = { u[0]->f.ptr( Ls ), u[1]->f.ptr( Ls ), u[2]->f.ptr( Ls ) };
   launch_stokes_div( &cx, &s->D->o, l, dt, 0, uu, nullptr, nullptr, s->rp->f.ptr( l ), kAll, 0 );
   hyb_fn* src[2] = { bp, s->rp };
   pointwise( s->rp, l, kAll, PT_LINCOMB, 2, sc, src );
}

void stokes_vcycle( hyb_stokes* s, hyb_fn* const* u, hyb_fn* p, hyb_fn* const* bu, hyb_fn* bp, int l )
{
   Context&  cx = s->ctx->c;
   const int dt = p->f.dtype;
   Mesh*     m  = &s->mesh->m;
   if ( l == s->p.min_level )
   {
      for ( int it = 0; it < s->p.coarse_sweeps; ++it ) uzawa_smooth( s, u, p, bu, bp, l );
      return;
   }
   for ( int it = 0; it < s->p.pre_smooth; ++it ) uzawa_smooth( s, u, p, bu, bp, l );
   stokes_residual( s, u, p, bu, bp, l );
   for ( int k = 0; k < 3; ++k )
   {
      launch_p2_restrict( &cx, m, l + 1, dt, kSolveFlag, s->ru[k]->f.ptr( l + 1 ), bu[k]->f.ptr( l ) );
      check_cuda( cudaMemsetAsync( u[k]->f.ptr( l ), 0, u[k]->f.bytes( l ), cx.stream ), "u.interpolate(0)" );
   }
   launch_restrict( &cx, m, l, dt, kAll, s->rp->f.ptr( l ), bp->f.ptr( l - 1 ) );
   check_cuda( cudaMemsetAsync( p->f.ptr( l - 1 ), 0, p->f.bytes( l - 1 ), cx.stream ), "p.interpolate(0)" );
   stokes_vcycle( s, u, p, bu, bp, l - 1 );
   for ( int k = 0; k < 3; ++k ) launch_p2_prolongate( &cx, m, l, dt, kSolveFlag, u[k]->f.ptr( l ), u[k]->f.ptr( l + 1 ), 1 );
   launch_prolongate( &cx, m, l - 1, dt, kAll, p->f.ptr( l - 1 ), p->f.ptr( l ), 1 );
   for ( int it = 0; it < s->p.post_smooth; ++it ) uzawa_smooth( s, u, p, bu, bp, l );
}

// one V-cycle through a CUDA graph: the cycle's thousands of small launches (the coarsest level's
// Uzawa steps above all) become one graph launch; the key is every level pointer of u, p, bu, bp
void stokes_cycle( hyb_stokes* s, hyb_fn* const* u, hyb_fn* p, hyb_fn* const* bu, hyb_fn* bp, int l )
{
   Context&                   cx = s->ctx->c;
   std::vector< const void* > key;
   key.push_back( reinterpret_cast< const void* >( intptr_t( l ) ) );
   for ( int L = s->p.min_level; L <= l; ++L )
   {
      for ( int k = 0; k < 3; ++k )
      {
         key.push_back( u[k]->f.ptr( L + 1 ) );
         key.push_back( bu[k]->f.ptr( L + 1 ) );
      }
      key.push_back( p->f.ptr( L ) );
      key.push_back( bp->f.ptr( L ) );
   }
   if ( key != s->gkey )
   {
      if ( s->gexec ) cudaGraphExecDestroy( s->gexec ), s->gexec = nullptr;
      s->gkey = key;
      stokes_vcycle( s, u, p, bu, bp, l );
      return;
   }
   if ( !s->gexec )
   {
      cudaGraph_t graph = nullptr;
      check_cuda( cudaStreamBeginCapture( cx.stream, cudaStreamCaptureModeThreadLocal ), "begin capture" );
      try
      {
         stokes_vcycle( s, u, p, bu, bp, l );
      } catch ( ... )
      {
         cudaStreamEndCapture( cx.stream, &graph );
         if ( graph ) cudaGraphDestroy( graph );
         s->gkey.clear();
         throw;
      }
      check_cuda( cudaStreamEndCapture( cx.stream, &graph ), "end capture" );
      const cudaError_t e = cudaGraphInstantiate( &s->gexec, graph, 0 );
      cudaGraphDestroy( graph );
      check_cuda( e, "graph instantiate" );
   }
   check_cuda( cudaGraphLaunch( s->gexec, cx.stream ), "graph launch" );
   cx.launches += 1;
}

double stokes_residual_norm( hyb_stokes* s, hyb_fn* const* u, hyb_fn* p, hyb_fn* const* bu, hyb_fn* bp, int l )
{
   stokes_residual( s, u, p, bu, bp, l );
   double r2 = 0;
   for ( int k = 0; k < 3; ++k ) r2 += dot_host( s->ru[k], s->ru[k], l, kSolveFlag );
   r2 += dot_host( s->rp, s->rp, l, kAll );
   return std::sqrt( r2 );
}
}  // namespace

extern "C" {

int hyb_stokes_params_default( hyb_stokes_params* p )
{
   if ( !p ) return HYB_EINVAL;
   *p                  = hyb_stokes_params{};
   p->min_level        = 0;
   p->max_level        = 2;
   // measured on the cube (eta = 1) and the blended shell (radial viscosity): asymptotic
   // residual-reduction factors 0.63-0.73 per V-cycle; omega = 1 diverged on the cube, fewer
   // velocity sweeps or pre/post steps diverged or stalled
   p->pre_smooth       = 3;
   p->post_smooth      = 3;
   p->velocity_sweeps  = 3;
   p->cheb_order       = 3;
   p->power_iterations = 20;
   p->omega            = 0.7;
   p->coarse_sweeps    = 30;
   p->velocity_block   = 0;
   p->pressure_scaling = 0;
   return HYB_OK;
}

int hyb_stokes_create( hyb_ctx* ctx, hyb_mesh* mesh, const hyb_coeff* viscosity, int blending, const hyb_stokes_params* params,
                       hyb_stokes** out )
{
   HYB_TRY
   require( ctx && mesh && params && out, "NULL argument" );
   require( params->min_level >= 0 && params->min_level <= params->max_level && params->max_level <= 10, "invalid level range" );
   require( params->pre_smooth >= 0 && params->post_smooth >= 0 && params->velocity_sweeps >= 1 && params->coarse_sweeps >= 1,
            "invalid smoothing counts" );
   require( params->cheb_order >= 1 && params->cheb_order <= 16, "Chebyshev order must be 1..16" );
   require( params->velocity_block == 0 || params->velocity_block == 1, "velocity_block must be 0 (per component) or 1 (full viscous)" );
   require( params->pressure_scaling == 0 || params->pressure_scaling == 1,
            "pressure_scaling must be 0 (PSPG diagonal) or 1 (lumped mass weighted by 1/eta)" );
   auto* s = new hyb_stokes();
   s->ctx  = ctx;
   ctx_ref( ctx );
   s->mesh = mesh;
   s->p    = *params;
   try
   {
      ok_rc( hyb_op_create_p2p1_div( ctx, mesh, params->min_level, params->max_level, blending, &s->D ) );
      if ( params->pressure_scaling == 1 )
      {
         ok_rc( hyb_op_create_divkgrad( ctx, mesh, params->min_level, params->max_level, viscosity, blending, &s->S ) );
         s->S->o.coeff.element = kElemLumpedMassInvK;
      }
      else ok_rc( hyb_op_create_p1_pspg( ctx, mesh, params->min_level, params->max_level, &s->S ) );
      if ( params->velocity_block == 1 )
      {
         ok_rc( hyb_op_create_p2_full_viscous( ctx, mesh, params->min_level, params->max_level, viscosity, blending, &s->V ) );
         *out = s;
         return HYB_OK;
      }
      ok_rc( hyb_op_create_p2_divkgrad( ctx, mesh, params->min_level, params->max_level, viscosity, blending, &s->A ) );
      // the velocity block is applied some hundred times per cycle: its element matrices are stored
      ok_rc( hyb_op_store_element_matrices( s->A ) );
      hyb_gmg_params gp;
      hyb_gmg_params_default( &gp );
      gp.min_level             = params->min_level;
      gp.max_level             = params->max_level;
      gp.smoother              = HYB_SMOOTHER_CHEBYSHEV;
      gp.cheb_order            = params->cheb_order;
      gp.cheb_power_iterations = params->power_iterations;
      gp.use_graph             = 0;
      ok_rc( hyb_gmg_create( ctx, s->A, &gp, &s->vel ) );
   } catch ( ... )
   {
      delete s;
      throw;
   }
   *out = s;
   HYB_CATCH
}

int hyb_stokes_destroy( hyb_stokes* s )
{
   HYB_TRY
   delete s;
   HYB_CATCH
}

int hyb_stokes_set_velocity_radii( hyb_stokes* s, const double* radii )
{
   HYB_TRY
   require( s && radii, "NULL argument" );
   // the captured cycle holds the Chebyshev coefficients of the old radii
   if ( s->gexec ) cudaGraphExecDestroy( s->gexec ), s->gexec = nullptr;
   s->gkey.clear();
   if ( s->V )
   {
      visc_set_radii( s, radii );
      return HYB_OK;
   }
   return hyb_gmg_set_radii( s->vel, radii );
   HYB_CATCH
}

int hyb_stokes_set_omega( hyb_stokes* s, double omega )
{
   HYB_TRY
   require( s, "NULL argument" );
   require( omega > 0.0 && std::isfinite( omega ), "omega must be positive" );
   // the captured cycle holds the old omega as a kernel argument
   if ( s->gexec ) cudaGraphExecDestroy( s->gexec ), s->gexec = nullptr;
   s->gkey.clear();
   s->p.omega = omega;
   HYB_CATCH
}

int hyb_stokes_estimate_relaxation( hyb_stokes* s, int level, int iterations, int velocity_sweeps, double* rho )
{
   HYB_TRY
   require( s && rho, "NULL argument" );
   require( level >= s->p.min_level && level <= s->p.max_level, "level outside the solver's level range" );
   require( iterations >= 1 && velocity_sweeps >= 1, "iterations and velocity_sweeps must be positive" );
   require( s->dtype < 0 || s->dtype == HYB_F64, "the estimate runs in FP64: call it on the FP64 solver" );
   Mesh*     m = &s->mesh->m;
   const int l = level, Ls = level + 1, dt = HYB_F64;
   FnHolder  uh[3], bh, xh, yh;
   hyb_fn*   u[3];
   for ( int k = 0; k < 3; ++k )
   {
      uh[k].h           = new_fn( s->ctx, m, dt, s->p.min_level + 1, s->p.max_level + 1 );
      uh[k].h->f.lshift = 1;
      u[k]              = uh[k].h;
   }
   bh.h           = new_fn( s->ctx, m, dt, s->p.min_level + 1, s->p.max_level + 1 );
   bh.h->f.lshift = 1;
   xh.h           = new_fn( s->ctx, m, dt, s->p.min_level, s->p.max_level );
   yh.h           = new_fn( s->ctx, m, dt, s->p.min_level, s->p.max_level );
   hyb_fn *x = xh.h, *y = yh.h;
   stokes_prepare( s, u[0], bh.h, dt );
   Context&     cx     = s->ctx->c;
   const double one[2] = { 1.0, 1.0 };
   // y = |S|^-1 B A~^-1 B^T x (P2P1UzawaDampingFactorEstimationOperator::apply with the solver's own
   // velocity smoother and pressure scaling; S^-1 is negative, hence the sign)
   auto E = [&]() {
      void* rr[3] = { s->ru[0]->f.ptr( Ls ), s->ru[1]->f.ptr( Ls ), s->ru[2]->f.ptr( Ls ) };
      launch_stokes_div( &cx, &s->D->o, l, dt, 1, nullptr, x->f.ptr( l ), rr, nullptr, kSolveFlag, 0 );
      for ( int k = 0; k < 3; ++k ) check_cuda( cudaMemsetAsync( u[k]->f.ptr( Ls ), 0, u[k]->f.bytes( Ls ), cx.stream ), "u = 0" );
      for ( int it = 0; it < velocity_sweeps; ++it )
      {
         if ( s->V )
         {
            visc_smooth( s, u, s->ru, l );
            continue;
         }
         for ( int k = 0; k < 3; ++k ) smooth( s->vel, u[k], s->ru[k], Ls );
      }
      const void* uu[3] = { u[0]->f.ptr( Ls ), u[1]->f.ptr( Ls ), u[2]->f.ptr( Ls ) };
      launch_stokes_div( &cx, &s->D->o, l, dt, 0, uu, nullptr, nullptr, s->rp->f.ptr( l ), kAll, 0 );
      hyb_fn* src[2] = { s->sinv, s->rp };
      pointwise( y, l, kAll, PT_MULT, 2, one, src );
      const double m1[1] = { -1.0 };
      hyb_fn*      ys[1] = { y };
      pointwise( y, l, kAll, PT_LINCOMB, 1, m1, ys );
   };
   auto scale_into = [&]( hyb_fn* dst, hyb_fn* src_fn, double f ) {
      const double c[1]  = { f };
      hyb_fn*      sr[1] = { src_fn };
      pointwise( dst, l, kAll, PT_LINCOMB, 1, c, sr );
   };
   // estimateSpectralRadiusWithPowerIteration (SpectrumEstimation.hpp:56-84): x random and normalised,
   // then x = y / |y|, y = E x; the radius is the Rayleigh quotient x . y
   ok_rc( hyb_fn_fill_random( x, l, 42u ) );
   scale_into( x, x, 1.0 / std::sqrt( dot_host( x, x, l, kAll ) ) );
   E();
   double radius = 0;
   for ( int it = 1; it <= iterations; ++it )
   {
      scale_into( x, y, 1.0 / std::sqrt( dot_host( y, y, l, kAll ) ) );
      E();
      radius = dot_host( x, y, l, kAll );
   }
   *rho = radius;
   HYB_CATCH
}

int hyb_stokes_apply( hyb_stokes* s, hyb_fn* const* u, hyb_fn* p, hyb_fn* const* du, hyb_fn* dp, int level )
{
   HYB_TRY
   stokes_fns_check( s, u, p, level );
   stokes_fns_check( s, du, dp, level );
   const int Ls = level + 1, dt = p->f.dtype;
   void*     dd[3] = { du[0]->f.ptr( Ls ), du[1]->f.ptr( Ls ), du[2]->f.ptr( Ls ) };
   if ( s->V )
   {
      const void* uu[3] = { u[0]->f.ptr( Ls ), u[1]->f.ptr( Ls ), u[2]->f.ptr( Ls ) };
      launch_full_viscous( &s->ctx->c, &s->V->o, level, dt, 0, uu, dd, kSolveFlag, 0 );
   }
   else
      for ( int k = 0; k < 3; ++k ) stencil( s->A, Ls, dt, OP_APPLY, kSolveFlag, 0, u[k]->f.ptr( Ls ), nullptr, nullptr, dd[k] );
   launch_stokes_div( &s->ctx->c, &s->D->o, level, dt, 1, nullptr, p->f.ptr( level ), dd, nullptr, kSolveFlag, 1 );
   const void* uu[3] = { u[0]->f.ptr( Ls ), u[1]->f.ptr( Ls ), u[2]->f.ptr( Ls ) };
   launch_stokes_div( &s->ctx->c, &s->D->o, level, dt, 0, uu, nullptr, nullptr, dp->f.ptr( level ), kAll, 0 );
   HYB_CATCH
}

int hyb_stokes_uzawa_smooth( hyb_stokes* s, hyb_fn* const* u, hyb_fn* p, hyb_fn* const* bu, hyb_fn* bp, int level )
{
   HYB_TRY
   stokes_fns_check( s, u, p, level );
   stokes_fns_check( s, bu, bp, level );
   stokes_prepare( s, u[0], bu[0], p->f.dtype );
   uzawa_smooth( s, u, p, bu, bp, level );
   HYB_CATCH
}

int hyb_stokes_residual_norm( hyb_stokes* s, hyb_fn* const* u, hyb_fn* p, hyb_fn* const* bu, hyb_fn* bp, int level, double* out )
{
   HYB_TRY
   require( out, "NULL argument" );
   stokes_fns_check( s, u, p, level );
   stokes_fns_check( s, bu, bp, level );
   stokes_prepare( s, u[0], bu[0], p->f.dtype );
   *out = stokes_residual_norm( s, u, p, bu, bp, level );
   HYB_CATCH
}

// mixedPrecisionIterativeRefinement for the Stokes system: the FP64 residual of `outer`, scaled to unit
// RMS and rounded to the inner solver's value type, one inner V-cycle from a zero correction, the
// correction added to the FP64 iterate.  `inner` is a second solver of the same levels whose work
// vectors hold FP32 or FP16.
int hyb_stokes_mixed_solve( hyb_stokes* outer, hyb_stokes* inner, int inner_dtype, hyb_fn* const* u, hyb_fn* p, hyb_fn* const* bu,
                            hyb_fn* bp, int level, int max_outer, double rtol, double* history, int* iterations )
{
   HYB_TRY
   require( outer && inner && outer != inner, "two solver instances are needed" );
   // FP16 is refused: the inverted PSPG diagonal (of order h^-3) leaves the FP16 range
   require( inner_dtype == F32 || inner_dtype == F64, "inner dtype must be FP32 or FP64 (FP16 overflows the pressure scaling)" );
   stokes_fns_check( outer, u, p, level );
   stokes_fns_check( outer, bu, bp, level );
   require( p->f.dtype == F64, "the iterate must hold FP64 values" );
   require( inner->mesh == outer->mesh && inner->p.min_level == outer->p.min_level && level <= inner->p.max_level,
            "inner solver of another mesh or level range" );
   require( ( inner->V != nullptr ) == ( outer->V != nullptr ), "inner and outer solvers have different velocity blocks" );
   require( max_outer >= 0, "max_outer must be >= 0" );
   stokes_prepare( outer, u[0], bu[0], F64 );
   Mesh*         m   = &outer->mesh->m;
   const int     lo  = outer->p.min_level;
   // inner iterate and right-hand side on every level (P2 velocity, P1 pressure), kept by the outer
   // solver for later calls with the same inner solver, level and value type
   if ( outer->mx_inner != inner || outer->mx_dtype != inner_dtype || outer->mx_level != level || !outer->mx[0] ||
        outer->mx[0]->ctx != inner->ctx )
   {
      for ( hyb_fn*& f : outer->mx ) hyb_fn_destroy( f ), f = nullptr;
      for ( int k = 0; k < 6; ++k )
      {
         outer->mx[k]           = new_fn( inner->ctx, m, inner_dtype, lo + 1, level + 1 );
         outer->mx[k]->f.lshift = 1;
      }
      outer->mx[6]    = new_fn( inner->ctx, m, inner_dtype, lo, level );
      outer->mx[7]    = new_fn( inner->ctx, m, inner_dtype, lo, level );
      outer->mx_inner = inner;
      outer->mx_dtype = inner_dtype;
      outer->mx_level = level;
   }
   hyb_fn* iu[3]  = { outer->mx[0], outer->mx[1], outer->mx[2] };
   hyb_fn* ibu[3] = { outer->mx[3], outer->mx[4], outer->mx[5] };
   hyb_fn* ip     = outer->mx[6];
   hyb_fn* ibp    = outer->mx[7];
   stokes_prepare( inner, iu[0], ibu[0], inner_dtype );
   Context&  cx = outer->ctx->c;
   const int Ls = level + 1;
   // owned entries of the residual (velocity inner DoFs, all pressure DoFs) for the unit-RMS scaling
   double nown = 0;
   {
      const P1Level& PU = m->level( Ls );
      const P1Level& PP = m->level( level );
      nown = 3.0 * double( PU.packed_size ) + double( PP.packed_size );
   }
   double r0 = stokes_residual_norm( outer, u, p, bu, bp, level );
   double rn = r0;
   if ( history ) history[0] = r0;
   int it = 0;
   for ( ; it < max_outer; ++it )
   {
      if ( r0 == 0.0 || rn / r0 < rtol ) break;
      const double sc = std::sqrt( nown ) / rn;
      for ( int k = 0; k < 3; ++k )
      {
         launch_convert( &cx, m->level( Ls ).size, inner_dtype, ibu[k]->f.ptr( Ls ), F64, outer->ru[k]->f.ptr( Ls ), sc );
         check_cuda( cudaMemsetAsync( iu[k]->f.ptr( Ls ), 0, iu[k]->f.bytes( Ls ), cx.stream ), "cudaMemset" );
      }
      launch_convert( &cx, m->level( level ).size, inner_dtype, ibp->f.ptr( level ), F64, outer->rp->f.ptr( level ), sc );
      check_cuda( cudaMemsetAsync( ip->f.ptr( level ), 0, ip->f.bytes( level ), cx.stream ), "cudaMemset" );
      if ( inner->ctx != outer->ctx ) check_cuda( cudaStreamSynchronize( cx.stream ), "sync" );
      stokes_cycle( inner, iu, ip, ibu, ibp, level );
      if ( inner->ctx != outer->ctx ) check_cuda( cudaStreamSynchronize( inner->ctx->c.stream ), "sync" );
      for ( int k = 0; k < 3; ++k )
         launch_axpy_to_f64( &cx, m->level( Ls ).size, (double*) u[k]->f.ptr( Ls ), inner_dtype, iu[k]->f.ptr( Ls ), 1.0 / sc );
      launch_axpy_to_f64( &cx, m->level( level ).size, (double*) p->f.ptr( level ), inner_dtype, ip->f.ptr( level ), 1.0 / sc );
      rn = stokes_residual_norm( outer, u, p, bu, bp, level );
      if ( history ) history[it + 1] = rn;
   }
   if ( iterations ) *iterations = it;
   HYB_CATCH
}

int hyb_stokes_solve( hyb_stokes* s, hyb_fn* const* u, hyb_fn* p, hyb_fn* const* bu, hyb_fn* bp, int level, int max_cycles, double rtol,
                      double* history, int* cycles_done )
{
   HYB_TRY
   stokes_fns_check( s, u, p, level );
   stokes_fns_check( s, bu, bp, level );
   require( max_cycles >= 0, "max_cycles must be >= 0" );
   stokes_prepare( s, u[0], bu[0], p->f.dtype );
   const double r0 = stokes_residual_norm( s, u, p, bu, bp, level );
   if ( history ) history[0] = r0;
   int c = 0;
   for ( ; c < max_cycles; ++c )
   {
      stokes_cycle( s, u, p, bu, bp, level );
      const double r = stokes_residual_norm( s, u, p, bu, bp, level );
      if ( history ) history[c + 1] = r;
      if ( rtol > 0 && r <= rtol * r0 )
      {
         ++c;
         break;
      }
   }
   if ( cycles_done ) *cycles_done = c;
   HYB_CATCH
}

}  // extern "C"
