// Minimal stand-in for hyteg/indexing/Common.hpp: a 3-component logical index
// that can key a std::map (the generated kernels receive stencils as
// std::map<Index, double> and look weights up by brace-initialised offsets).
#pragma once
#include <cstdint>
#include "core/DataTypes.h"
namespace hyteg {
using idx_t = std::int64_t;
namespace indexing {
struct Index
{
   idx_t v[3];
   Index() : v{ 0, 0, 0 } {}
   Index( idx_t x, idx_t y, idx_t z ) : v{ x, y, z } {}
   idx_t x() const { return v[0]; }
   idx_t y() const { return v[1]; }
   idx_t z() const { return v[2]; }
   bool  operator<( const Index& o ) const
   {
      if ( v[0] != o.v[0] ) return v[0] < o.v[0];
      if ( v[1] != o.v[1] ) return v[1] < o.v[1];
      return v[2] < o.v[2];
   }
};
} // namespace indexing
} // namespace hyteg
