// Shim (ours): a 3-vector with the operations the compiled reference headers use.
#pragma once
#include <cmath>
#include <cstddef>

#include "hyteg/types/Matrix.hpp"

namespace hyteg {
struct Point3D
{
   real_t v[3] = { 0, 0, 0 };
   Point3D() = default;
   Point3D( real_t a, real_t b, real_t c )
   : v{ a, b, c }
   {}
   real_t&       operator[]( std::size_t i ) { return v[i]; }
   const real_t& operator[]( std::size_t i ) const { return v[i]; }
   real_t        dot( const Point3D& o ) const { return v[0] * o.v[0] + v[1] * o.v[1] + v[2] * o.v[2]; }
   real_t        squaredNorm() const { return dot( *this ); }
   real_t        norm() const { return std::sqrt( squaredNorm() ); }
   Point3D&      operator/=( real_t s )
   {
      v[0] /= s;
      v[1] /= s;
      v[2] /= s;
      return *this;
   }
   Point3D& operator*=( real_t s )
   {
      v[0] *= s;
      v[1] *= s;
      v[2] *= s;
      return *this;
   }
};
inline Point3D operator-( const Point3D& a, const Point3D& b ) { return { a[0] - b[0], a[1] - b[1], a[2] - b[2] }; }
inline Point3D operator+( const Point3D& a, const Point3D& b ) { return { a[0] + b[0], a[1] + b[1], a[2] + b[2] }; }
inline Point3D operator*( real_t s, const Point3D& a ) { return { s * a[0], s * a[1], s * a[2] }; }
inline Point3D operator*( const Point3D& a, real_t s ) { return { s * a[0], s * a[1], s * a[2] }; }
inline Point3D crossProduct( const Point3D& a, const Point3D& b )
{
   return { a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0] };
}
} // namespace hyteg
