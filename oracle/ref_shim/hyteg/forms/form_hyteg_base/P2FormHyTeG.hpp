// Minimal stand-in for the P2FormHyTeG base class of the reference's generated forms: the
// virtual integration interface and the blending map member.  Test infrastructure only.
#pragma once
#include "hyteg/geometry/GeometryMap.hpp"

namespace hyteg {
class P2FormHyTeG
{
 public:
   virtual ~P2FormHyTeG() = default;
   virtual void integrateAll( const std::array< Point3D, 3 >&, Matrix< real_t, 6, 6 >& ) const {}
   virtual void integrateRow0( const std::array< Point3D, 3 >&, Matrix< real_t, 1, 6 >& ) const {}
   virtual void integrateAll( const std::array< Point3D, 4 >&, Matrix< real_t, 10, 10 >& ) const {}
   virtual void integrateRow0( const std::array< Point3D, 4 >&, Matrix< real_t, 1, 10 >& ) const {}
   void         setGeometryMap( const std::shared_ptr< GeometryMap >& m ) const { geometryMap_ = m; }

 protected:
   mutable std::shared_ptr< GeometryMap > geometryMap_;
};
}  // namespace hyteg
