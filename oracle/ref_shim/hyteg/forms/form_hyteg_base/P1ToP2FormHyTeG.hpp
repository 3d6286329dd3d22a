// Minimal stand-in for the P1ToP2FormHyTeG base class of the reference's generated mixed forms (P2
// test functions, P1 trial functions).  Test infrastructure only.
#pragma once
#include "hyteg/geometry/GeometryMap.hpp"

namespace hyteg {
class P1ToP2FormHyTeG
{
 public:
   virtual ~P1ToP2FormHyTeG() = default;
   virtual void integrateAll( const std::array< Point3D, 3 >&, Matrix< real_t, 6, 3 >& ) const {}
   virtual void integrateAll( const std::array< Point3D, 4 >&, Matrix< real_t, 10, 4 >& ) const {}
   virtual void integrateRow0( const std::array< Point3D, 3 >&, Matrix< real_t, 1, 3 >& ) const {}
   virtual void integrateRow0( const std::array< Point3D, 4 >&, Matrix< real_t, 1, 4 >& ) const {}
   void         setGeometryMap( const std::shared_ptr< GeometryMap >& m ) const { geometryMap_ = m; }

 protected:
   mutable std::shared_ptr< GeometryMap > geometryMap_;
};
}  // namespace hyteg
