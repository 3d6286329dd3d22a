/*
 * hyteg_b200.hpp — C++ adaptor over the C ABI of include/hyteg_b200.h that keeps the reference's
 * class and method names, so HyTeG application code (tutorials/full-apps/FA.01_GeometricMultigrid,
 * the convergence tests under tests/hyteg/convergence) can switch to the B200 path by changing types,
 * not calls.
 *
 * Reference interfaces mirrored (paths relative to the hyteg source tree):
 *   P1Function<ValueType>                p1functionspace/P1Function.hpp, VertexDoFFunction.hpp
 *   P1ConstantLaplaceOperator            constant_stencil_operator/P1ConstantOperator.hpp:167
 *     ::apply(src, dst, level, flag, updateType)  operators/Operator.hpp:74-81
 *     ::smooth_jac(dst, rhs, tmp, relax, level, flag)  solvers/Smoothables.hpp:33-40
 *   P1toP1LinearRestriction / P1toP1LinearProlongation  gridtransferoperators/
 *   CGSolver(storage, minLevel, maxLevel, maxIter, relTol, absTol)  solvers/CGSolver.hpp:44-75
 *   GeometricMultigridSolver::solve(A, x, b, level)  solvers/GeometricMultigridSolver.hpp:180-305
 *   VTKOutput(dir, filename, storage, writeFrequency)  dataexport/VTKOutput/VTKOutput.hpp:44-139
 *
 * Errors: the reference aborts the process (WALBERLA_ABORT / WALBERLA_CHECK); here every failing
 * call goes to one error handler, by default throwing hyteg::b200::Error with the library's message.
 * setErrorHandler() replaces it (for example with a handler that logs and aborts, as the reference
 * does).  Objects own their handles (RAII); copies are disabled, moves transfer ownership.
 */
#pragma once

#include <array>
#include <cstdint>
#include <functional>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "hyteg_b200.h"

namespace hyteg {

// DoFType (types/types.hpp:29-43) and UpdateType (types/types.hpp:88-92)
enum DoFType : uint32_t
{
   Inner            = HYB_INNER,
   DirichletBoundary = HYB_DIRICHLET,
   NeumannBoundary  = HYB_NEUMANN,
   FreeslipBoundary = HYB_FREESLIP,
   All              = HYB_ALL,
};
inline DoFType operator|( DoFType a, DoFType b ) { return DoFType( uint32_t( a ) | uint32_t( b ) ); }
enum UpdateType
{
   Replace = HYB_REPLACE,
   Add     = HYB_ADD,
};

namespace b200 {

struct Error : std::runtime_error
{
   int status;
   Error( int rc, const std::string& what )
   : std::runtime_error( what )
   , status( rc )
   {}
};

using ErrorHandler = std::function< void( int status, const char* message ) >;

inline ErrorHandler& errorHandler()
{
   static ErrorHandler h = []( int rc, const char* msg ) { throw Error( rc, std::string( "hyteg_b200: " ) + msg ); };
   return h;
}
inline void setErrorHandler( ErrorHandler h ) { errorHandler() = std::move( h ); }
inline void check( int rc )
{
   if ( rc != HYB_OK ) errorHandler()( rc, hyb_last_error() );
}

// a device and the stream the library issues its work on
class Context
{
 public:
   explicit Context( int device = 0, void* stream = nullptr ) { check( hyb_ctx_create( device, stream, &h_ ) ); }
   ~Context() { if ( h_ ) hyb_ctx_destroy( h_ ); }
   Context( const Context& )            = delete;
   Context& operator=( const Context& ) = delete;
   hyb_ctx* get() const { return h_; }
   void     synchronize() const { check( hyb_ctx_synchronize( h_ ) ); }

 private:
   hyb_ctx* h_ = nullptr;
};

}  // namespace b200

// MeshInfo + SetupPrimitiveStorage + PrimitiveStorage in one object (mesh/MeshInfo.hpp,
// primitivestorage/SetupPrimitiveStorage.hpp:45, primitivestorage/PrimitiveStorage.hpp:116)
class PrimitiveStorage
{
 public:
   // MeshInfo::meshCuboid (mesh/MeshGenCuboid.cpp:35-172)
   static PrimitiveStorage cuboid( b200::Context& c, const std::array< double, 3 >& lo, const std::array< double, 3 >& hi,
                                   int nx, int ny, int nz )
   {
      PrimitiveStorage s;
      b200::check( hyb_mesh_create_cuboid( c.get(), lo.data(), hi.data(), nx, ny, nz, &s.h_ ) );
      return s;
   }
   // MeshInfo::meshSphericalShell (mesh/MeshGenSphericalShell.cpp:642-765)
   static PrimitiveStorage sphericalShell( b200::Context& c, int ntan, int nrad, double rmin, double rmax )
   {
      PrimitiveStorage s;
      b200::check( hyb_mesh_create_spherical_shell( c.get(), ntan, nrad, rmin, rmax, &s.h_ ) );
      return s;
   }
   // vertex coordinates in id order, tetrahedra in the mesh's own vertex order
   static PrimitiveStorage fromTetrahedra( b200::Context& c, const std::vector< double >& coords, const std::vector< int >& tets )
   {
      PrimitiveStorage s;
      b200::check( hyb_mesh_create( c.get(), int( coords.size() / 3 ), coords.data(), int( tets.size() / 4 ), tets.data(), &s.h_ ) );
      return s;
   }
   PrimitiveStorage( PrimitiveStorage&& o ) noexcept
   : h_( std::exchange( o.h_, nullptr ) )
   {}
   ~PrimitiveStorage() { if ( h_ ) hyb_mesh_destroy( h_ ); }
   PrimitiveStorage( const PrimitiveStorage& )            = delete;
   PrimitiveStorage& operator=( const PrimitiveStorage& ) = delete;
   hyb_mesh*         get() const { return h_; }
   int64_t           packedSize( uint_fast32_t level ) const
   {
      int64_t n = 0;
      b200::check( hyb_layout_packed_size( h_, int( level ), &n ) );
      return n;
   }

 private:
   PrimitiveStorage() = default;
   hyb_mesh* h_       = nullptr;
};

template < typename ValueType >
struct ValueTypeCode;
template <>
struct ValueTypeCode< double >
{
   static constexpr int value = HYB_F64;
};
template <>
struct ValueTypeCode< float >
{
   static constexpr int value = HYB_F32;
};

// P1Function<ValueType> (p1functionspace/P1Function.hpp); host values are exchanged as doubles in
// the packed per-primitive layout of the reference (VertexDoFMemory.hpp:39-60)
template < typename ValueType >
class P1Function
{
 public:
   P1Function( const std::string& name, b200::Context& c, const PrimitiveStorage& storage, uint_fast32_t minLevel,
               uint_fast32_t maxLevel )
   : name_( name )
   {
      b200::check( hyb_fn_create( c.get(), storage.get(), ValueTypeCode< ValueType >::value, int( minLevel ), int( maxLevel ), &h_ ) );
   }
   ~P1Function() { if ( h_ ) hyb_fn_destroy( h_ ); }
   P1Function( const P1Function& )            = delete;
   P1Function& operator=( const P1Function& ) = delete;
   hyb_fn*     get() const { return h_; }
   const std::string& getFunctionName() const { return name_; }

   void interpolate( double constant, uint_fast32_t level, DoFType flag = All ) const
   {
      b200::check( hyb_fn_interpolate_const( h_, constant, int( level ), flag ) );
   }
   // interpolate(std::function<real_t(const Point3D&)>, level, flag)
   void interpolate( const std::function< double( const double* xyz ) >& f, uint_fast32_t level, DoFType flag = All ) const
   {
      auto tramp = []( const double* xyz, void* user ) -> double { return ( *static_cast< const std::function< double( const double* ) >* >( user ) )( xyz ); };
      b200::check( hyb_fn_interpolate_callback( h_, tramp, const_cast< void* >( static_cast< const void* >( &f ) ), int( level ), flag ) );
   }
   void assign( const std::vector< double >& scalars, const std::vector< const P1Function* >& fns, uint_fast32_t level,
                DoFType flag = All ) const
   {
      std::vector< hyb_fn* > hs;
      for ( auto* f : fns ) hs.push_back( f->get() );
      b200::check( hyb_fn_assign( h_, int( hs.size() ), scalars.data(), hs.data(), int( level ), flag ) );
   }
   void add( const std::vector< double >& scalars, const std::vector< const P1Function* >& fns, uint_fast32_t level,
             DoFType flag = All ) const
   {
      std::vector< hyb_fn* > hs;
      for ( auto* f : fns ) hs.push_back( f->get() );
      b200::check( hyb_fn_add( h_, int( hs.size() ), scalars.data(), hs.data(), int( level ), flag ) );
   }
   double dotGlobal( const P1Function& other, uint_fast32_t level, DoFType flag = All ) const
   {
      double r = 0;
      b200::check( hyb_fn_dot( h_, other.get(), int( level ), flag, &r ) );
      return r;
   }
   template < typename Other >
   void copyFrom( const P1Function< Other >& other, uint_fast32_t level ) const
   {
      b200::check( hyb_fn_copy_from( h_, other.get(), int( level ) ) );
   }
   void upload( uint_fast32_t level, const std::vector< double >& packed ) const
   {
      b200::check( hyb_fn_upload( h_, int( level ), packed.data() ) );
   }
   std::vector< double > download( uint_fast32_t level, int64_t packedSize ) const
   {
      std::vector< double > out( static_cast< size_t >( packedSize ) );
      b200::check( hyb_fn_download( h_, int( level ), out.data() ) );
      return out;
   }

 private:
   std::string name_;
   hyb_fn*     h_ = nullptr;
};

// the operator kinds of include/hyteg_b200.h behind one class template
template < int Kind >
class P1ConstantOperatorB200
{
 public:
   P1ConstantOperatorB200( b200::Context& c, const PrimitiveStorage& storage, uint_fast32_t minLevel, uint_fast32_t maxLevel )
   {
      b200::check( hyb_op_create( c.get(), storage.get(), Kind, int( minLevel ), int( maxLevel ), &h_ ) );
   }
   ~P1ConstantOperatorB200() { if ( h_ ) hyb_op_destroy( h_ ); }
   P1ConstantOperatorB200( const P1ConstantOperatorB200& )            = delete;
   P1ConstantOperatorB200& operator=( const P1ConstantOperatorB200& ) = delete;
   hyb_op*                 get() const { return h_; }

   template < typename V >
   void apply( const P1Function< V >& src, const P1Function< V >& dst, uint_fast32_t level, DoFType flag,
               UpdateType updateType = Replace ) const
   {
      b200::check( hyb_op_apply( h_, src.get(), dst.get(), int( level ), flag, int( updateType ) ) );
   }
   template < typename V >
   void smooth_jac( const P1Function< V >& dst, const P1Function< V >& rhs, const P1Function< V >& tmp, double relax,
                    uint_fast32_t level, DoFType flag ) const
   {
      b200::check( hyb_op_smooth_jac( h_, dst.get(), rhs.get(), tmp.get(), relax, int( level ), flag ) );
   }
   template < typename V >
   void smooth_gs( const P1Function< V >& dst, const P1Function< V >& rhs, uint_fast32_t level, DoFType flag ) const
   {
      b200::check( hyb_op_smooth_sor( h_, dst.get(), rhs.get(), 1.0, int( level ), flag, 0 ) );
   }

 private:
   hyb_op* h_ = nullptr;
};
using P1ConstantLaplaceOperator = P1ConstantOperatorB200< HYB_P1_CONST_LAPLACE >;
using P1ConstantMassOperator    = P1ConstantOperatorB200< HYB_P1_CONST_MASS >;

class P1toP1LinearRestriction
{
 public:
   template < typename V >
   void restrict( const P1Function< V >& function, uint_fast32_t sourceLevel, DoFType flag ) const
   {
      b200::check( hyb_restrict( function.get(), int( sourceLevel ), flag ) );
   }
};

class P1toP1LinearProlongation
{
 public:
   template < typename V >
   void prolongate( const P1Function< V >& function, uint_fast32_t sourceLevel, DoFType flag ) const
   {
      b200::check( hyb_prolongate( function.get(), int( sourceLevel ), flag, HYB_REPLACE ) );
   }
   template < typename V >
   void prolongateAndAdd( const P1Function< V >& function, uint_fast32_t sourceLevel, DoFType flag ) const
   {
      b200::check( hyb_prolongate( function.get(), int( sourceLevel ), flag, HYB_ADD ) );
   }
};

// CGSolver (solvers/CGSolver.hpp:44-75,94-206), identity preconditioner
template < typename Operator >
class CGSolver
{
 public:
   CGSolver( uint_fast32_t maxIter = 1000000, double relativeTolerance = 1e-16, double absoluteTolerance = 1e-16 )
   : maxIter_( maxIter )
   , rtol_( relativeTolerance )
   , atol_( absoluteTolerance )
   {}
   template < typename V >
   void solve( const Operator& A, const P1Function< V >& x, const P1Function< V >& b, uint_fast32_t level )
   {
      b200::check( hyb_cg_solve( A.get(), x.get(), b.get(), int( level ), int( maxIter_ ), rtol_, atol_, &iterations_ ) );
   }
   int iterations() const { return iterations_; }

 private:
   uint_fast32_t maxIter_;
   double        rtol_, atol_;
   int           iterations_ = 0;
};

// GeometricMultigridSolver (solvers/GeometricMultigridSolver.hpp:61-162) with the smoother and the CG
// coarse solver on the device; parameters as hyb_gmg_params (hyb_gmg_params_default gives the
// reference's defaults: Chebyshev 1.2 / 0.3 bounds, CG coarse solve)
template < typename Operator >
class GeometricMultigridSolver
{
 public:
   static hyb_gmg_params defaultParameters()
   {
      hyb_gmg_params p;
      b200::check( hyb_gmg_params_default( &p ) );
      return p;
   }
   GeometricMultigridSolver( b200::Context& c, const Operator& A, const hyb_gmg_params& p )
   {
      b200::check( hyb_gmg_create( c.get(), A.get(), &p, &h_ ) );
   }
   ~GeometricMultigridSolver() { if ( h_ ) hyb_gmg_destroy( h_ ); }
   GeometricMultigridSolver( const GeometricMultigridSolver& )            = delete;
   GeometricMultigridSolver& operator=( const GeometricMultigridSolver& ) = delete;

   // Solver::solve(A, x, b, level): one cycle (solvers/Solver.hpp:31-35)
   template < typename V >
   void solve( const Operator&, const P1Function< V >& x, const P1Function< V >& b, uint_fast32_t level )
   {
      b200::check( hyb_gmg_solve( h_, x.get(), b.get(), int( level ) ) );
   }
   // cycles until ||r|| / ||r_0|| < rtol; returns ||r_0||, ..., ||r_k||
   template < typename V >
   std::vector< double > solveCycles( const P1Function< V >& x, const P1Function< V >& b, uint_fast32_t level, int maxCycles,
                                      double rtol )
   {
      std::vector< double > hist( size_t( maxCycles ) + 1 );
      int                   done = 0;
      b200::check( hyb_gmg_solve_cycles( h_, x.get(), b.get(), int( level ), maxCycles, rtol, hist.data(), &done ) );
      hist.resize( size_t( done ) + 1 );
      return hist;
   }
   void setRadii( const std::vector< double >& radii ) { b200::check( hyb_gmg_set_radii( h_, radii.data() ) ); }

 private:
   hyb_gmg* h_ = nullptr;
};

// VTKOutput (dataexport/VTKOutput/VTKOutput.hpp:44-139): add() functions, write( level, timestep )
// writes <dir>/<filename>_VertexDoF_level<L>_ts<T>.vtu when timestep % writeFrequency == 0;
// setParameter( "vtkDataFormat", "ASCII" | "BINARY" ).  Added functions must outlive the writer's
// write() calls (they are downloaded at write time).
class VTKOutput
{
 public:
   VTKOutput( const std::string& dir, const std::string& filename, const PrimitiveStorage& storage, uint_fast32_t writeFrequency = 1 )
   {
      b200::check( hyb_vtk_create( storage.get(), dir.c_str(), filename.c_str(), int( writeFrequency ), &h_ ) );
   }
   ~VTKOutput() { if ( h_ ) hyb_vtk_destroy( h_ ); }
   VTKOutput( const VTKOutput& )            = delete;
   VTKOutput& operator=( const VTKOutput& ) = delete;

   template < typename Function >
   void add( const Function& function )
   {
      b200::check( hyb_vtk_add( h_, function.get(), function.getFunctionName().c_str() ) );
   }
   template < typename Function >
   void remove( const Function& function )
   {
      b200::check( hyb_vtk_remove( h_, function.get() ) );
   }
   void setParameter( const std::string& key, const std::string& value )
   {
      b200::check( hyb_vtk_set_parameter( h_, key.c_str(), value.c_str() ) );
   }
   void write( uint_fast32_t level, uint_fast32_t timestep = 0 ) const { b200::check( hyb_vtk_write( h_, int( level ), int( timestep ) ) ); }

 private:
   hyb_vtk* h_ = nullptr;
};

}  // namespace hyteg
