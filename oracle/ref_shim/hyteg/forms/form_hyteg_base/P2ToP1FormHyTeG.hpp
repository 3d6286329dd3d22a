// Minimal stand-in for the P2ToP1FormHyTeG base class of the reference's generated mixed forms (P1
// test functions, P2 trial functions): the integration interface and the blending map member.
// Test infrastructure only.
#pragma once
#include "hyteg/geometry/GeometryMap.hpp"

namespace hyteg {
class P2ToP1FormHyTeG
{
 public:
   virtual ~P2ToP1FormHyTeG() = default;
   virtual void integrateAll( const std::array< Point3D, 3 >&, Matrix< real_t, 3, 6 >& ) const {}
   virtual void integrateAll( const std::array< Point3D, 4 >&, Matrix< real_t, 4, 10 >& ) const {}
   virtual void integrateRow0( const std::array< Point3D, 3 >&, Matrix< real_t, 1, 6 >& ) const {}
   virtual void integrateRow0( const std::array< Point3D, 4 >&, Matrix< real_t, 1, 10 >& ) const {}
   void         setGeometryMap( const std::shared_ptr< GeometryMap >& m ) const { geometryMap_ = m; }

 protected:
   mutable std::shared_ptr< GeometryMap > geometryMap_;
};
}  // namespace hyteg
