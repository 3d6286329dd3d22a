// Stand-in for hyteg/primitivestorage/SetupPrimitiveStorage.hpp in the oracle's shell-map library:
// the few queries IcosahedralShellMap makes (cell coordinates, neighbour vertices / faces / cells,
// lookups by id), over a macro mesh given as vertex coordinates and tetrahedra, and the MPI buffer
// types its (de)serialisation names.  Primitive ids: vertices 0..nV-1, faces from 1e6, cells from
// 2e6.  Cell-local faces in the reference's order 012, 013, 023, 123 (SetupPrimitiveStorage.cpp
// :305-315).  Test infrastructure only.
#pragma once
#include <algorithm>
#include <array>
#include <cstdint>
#include <limits>
#include <map>
#include <memory>
#include <vector>

#include "core/DataTypes.h"
#include "hyteg/types/PointMatrixForwardDeclare.hpp"

#define WALBERLA_ABORT( msg ) std::abort()
#define WALBERLA_ASSERT_EQUAL( a, b )
#define WALBERLA_ASSERT_GREATER( a, b )
#define WALBERLA_UNUSED( x ) (void) ( x )

namespace walberla {
namespace mpi {
template < typename T >
class GenericRecvBuffer
{
 public:
   std::vector< double > data;
   size_t                pos = 0;
   GenericRecvBuffer&    operator>>( double& v )
   {
      v = data.at( pos++ );
      return *this;
   }
   GenericRecvBuffer& operator>>( hyteg::Point3D& p )
   {
      for ( int i = 0; i < 3; ++i ) p[i] = data.at( pos++ );
      return *this;
   }
};
struct OptimalGrowth
{};
template < typename T, typename G >
class GenericSendBuffer
{
 public:
   template < typename X >
   GenericSendBuffer& operator<<( const X& )
   {
      return *this;
   }
};
}  // namespace mpi
}  // namespace walberla

namespace hyteg {
using walberla::real_t;
using walberla::uint_t;

class GeometryMap;

class PrimitiveID
{
 public:
   PrimitiveID() = default;
   explicit PrimitiveID( int64_t i )
   : id_( i )
   {}
   bool    operator==( const PrimitiveID& o ) const { return id_ == o.id_; }
   bool    operator!=( const PrimitiveID& o ) const { return id_ != o.id_; }
   bool    operator<( const PrimitiveID& o ) const { return id_ < o.id_; }
   int64_t id() const { return id_; }

 private:
   int64_t id_ = -1;
};

class Primitive
{
 public:
   PrimitiveID                getID() const { return id; }
   void                       getNeighborVertices( std::vector< PrimitiveID >& v ) const { v = vertices; }
   void                       getNeighborFaces( std::vector< PrimitiveID >& v ) const { v = faces; }
   void                       getNeighborCells( std::vector< PrimitiveID >& v ) const { v = cells; }
   PrimitiveID                id;
   std::vector< PrimitiveID > vertices, faces, cells;
};

class Cell : public Primitive
{
 public:
   const std::array< Point3D, 4 >& getCoordinates() const { return coords; }
   uint_t                          getLocalVertexID( const PrimitiveID& v ) const
   {
      return uint_t( std::find( vertices.begin(), vertices.end(), v ) - vertices.begin() );
   }
   std::array< Point3D, 4 > coords;
};
class Face : public Primitive
{};
class Edge : public Primitive
{};

class SetupPrimitiveStorage
{
 public:
   SetupPrimitiveStorage( int nv, const double* xyz, int nc, const int* tets )
   {
      std::map< std::array< int, 3 >, int64_t > face_id;
      for ( int c = 0; c < nc; ++c )
      {
         auto cell = std::make_shared< Cell >();
         cell->id  = PrimitiveID( 2000000 + c );
         for ( int k = 0; k < 4; ++k )
         {
            const int v = tets[4 * c + k];
            cell->vertices.push_back( PrimitiveID( v ) );
            cell->coords[k] = Point3D( xyz[3 * v], xyz[3 * v + 1], xyz[3 * v + 2] );
         }
         static const int lf[4][3] = { { 0, 1, 2 }, { 0, 1, 3 }, { 0, 2, 3 }, { 1, 2, 3 } };
         for ( const auto& f : lf )
         {
            std::array< int, 3 > key = { tets[4 * c + f[0]], tets[4 * c + f[1]], tets[4 * c + f[2]] };
            std::sort( key.begin(), key.end() );
            auto it = face_id.find( key );
            if ( it == face_id.end() )
            {
               const int64_t id = 1000000 + int64_t( face_id.size() );
               it               = face_id.emplace( key, id ).first;
               auto face        = std::make_shared< Face >();
               face->id         = PrimitiveID( id );
               for ( int v : key ) face->vertices.push_back( PrimitiveID( v ) );
               faces_[face->id] = face;
            }
            cell->faces.push_back( PrimitiveID( it->second ) );
            faces_[PrimitiveID( it->second )]->cells.push_back( cell->id );
         }
         cells_[cell->id] = cell;
      }
      (void) nv;
   }
   std::shared_ptr< Cell >       getCell( const PrimitiveID& id ) const { return cells_.at( id ); }
   std::shared_ptr< const Face > getFace( const PrimitiveID& id ) const { return faces_.at( id ); }
   const std::map< PrimitiveID, std::shared_ptr< Cell > >& getCells() const { return cells_; }
   const std::map< PrimitiveID, std::shared_ptr< Face > >& getFaces() const { return faces_; }
   const std::map< PrimitiveID, std::shared_ptr< Edge > >& getEdges() const { return edges_; }
   void setGeometryMap( const PrimitiveID&, const std::shared_ptr< GeometryMap >& ) {}

 private:
   std::map< PrimitiveID, std::shared_ptr< Cell > > cells_;
   std::map< PrimitiveID, std::shared_ptr< Face > > faces_;
   std::map< PrimitiveID, std::shared_ptr< Edge > > edges_;
};

}  // namespace hyteg
