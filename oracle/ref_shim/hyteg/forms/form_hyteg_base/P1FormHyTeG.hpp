// Minimal stand-in for the P1FormHyTeG base class of the reference's generated forms: the
// virtual integration interface and the blending map member.  Test infrastructure only.
#pragma once
#include "hyteg/geometry/GeometryMap.hpp"

namespace hyteg {
class P1FormHyTeG
{
 public:
   virtual ~P1FormHyTeG() = default;
   virtual void integrateAll( const std::array< Point3D, 3 >&, Matrix< real_t, 3, 3 >& ) const {}
   virtual void integrateRow0( const std::array< Point3D, 3 >&, Matrix< real_t, 1, 3 >& ) const {}
   virtual void integrateAll( const std::array< Point3D, 4 >&, Matrix< real_t, 4, 4 >& ) const {}
   virtual void integrateRow0( const std::array< Point3D, 4 >&, Matrix< real_t, 1, 4 >& ) const {}
   void         setGeometryMap( const std::shared_ptr< GeometryMap >& m ) const { geometryMap_ = m; }

 protected:
   mutable std::shared_ptr< GeometryMap > geometryMap_;
};
}  // namespace hyteg
