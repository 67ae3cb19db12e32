// Minimal stand-in for waLBerla's core/DataTypes.h: the generated kernels only
// need the fixed-width integer names.
#pragma once
#include <cstddef>
#include <cstdint>
namespace walberla {
using uint_t   = std::size_t;
using real_t   = double;
using int32_t  = std::int32_t;
using int64_t  = std::int64_t;
using uint32_t = std::uint32_t;
using uint64_t = std::uint64_t;
} // namespace walberla
