// Shim (ours): fixed-size row-major matrices with operator()(i, j), the scalar types and
// the serialisation buffer types the compiled reference headers name.
#pragma once
#include <cstddef>
#include <memory>

namespace walberla {
using real_t = double;
using uint_t = std::size_t;
template < typename T >
inline real_t real_c( T x )
{
   return real_t( x );
}
namespace mpi {
struct SendBuffer
{
   template < typename T >
   SendBuffer& operator<<( const T& )
   {
      return *this;
   }
};
struct RecvBuffer
{
   template < typename T >
   RecvBuffer& operator>>( T& )
   {
      return *this;
   }
};
} // namespace mpi
} // namespace walberla

namespace hyteg {
using walberla::real_t;
using walberla::uint_t;
template < typename T, int M, int N >
struct Matrix
{
   T        a[M][N] = {};
   T&       operator()( int i, int j ) { return a[i][j]; }
   const T& operator()( int i, int j ) const { return a[i][j]; }
};
using Matrix2r = Matrix< real_t, 2, 2 >;
using Matrix3r = Matrix< real_t, 3, 3 >;
} // namespace hyteg
