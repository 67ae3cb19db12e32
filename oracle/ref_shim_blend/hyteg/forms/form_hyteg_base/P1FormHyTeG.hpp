// Shim (ours): the form base class of the generated P1 forms, reduced to the integration
// interface and the geometry map the generated code calls.
#pragma once
#include <array>
#include <functional>
#include <memory>

#include "hyteg/geometry/GeometryMap.hpp"

namespace hyteg {
class P1FormHyTeG
{
 public:
   virtual ~P1FormHyTeG() {}
   virtual void integrateAll( const std::array< Point3D, 3 >& coords, Matrix< real_t, 3, 3 >& elMat ) const  = 0;
   virtual void integrateRow0( const std::array< Point3D, 3 >& coords, Matrix< real_t, 1, 3 >& elMat ) const = 0;
   virtual void integrateAll( const std::array< Point3D, 4 >& coords, Matrix< real_t, 4, 4 >& elMat ) const  = 0;
   virtual void integrateRow0( const std::array< Point3D, 4 >& coords, Matrix< real_t, 1, 4 >& elMat ) const = 0;
   void         setGeometryMap( std::shared_ptr< GeometryMap > map ) { geometryMap_ = std::move( map ); }

 protected:
   std::shared_ptr< GeometryMap > geometryMap_;
};
} // namespace hyteg
