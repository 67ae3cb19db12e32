// C ABI (ours) over the reference's IcosahedralShellMap and the p1_div_k_grad_blending_q3 and
// p1_div_k_grad_affine_q3 forms, compiled unchanged from the reference source tree against
// the shims in ref_shim_blend/.
// TEST INFRASTRUCTURE ONLY: it pins the oracle's restatement of the shell map, of the
// blended element matrix (tests/test_blend_oracle.py, tests/golden/make_blend_golden.py) and
// of the affine div-k-grad element matrix (tests/test_divkgrad_oracle.py,
// tests/golden/make_divkgrad_golden.py).
//
// The mesh is given as arrays (vertex coordinates, cell vertex lists); the storage shim is
// filled the way SetupPrimitiveStorage orders it (src/hyteg/primitivestorage/
// SetupPrimitiveStorage.cpp:244-300): a cell's faces are (v0 v1 v2), (v0 v1 v3), (v0 v2 v3),
// (v1 v2 v3), and a face lists its cells in cell order.
#include <algorithm>
#include <cmath>

#include "hyteg/geometry/IcosahedralShellMap.hpp"
#include "hyteg/forms/form_hyteg_generated/p1/p1_div_k_grad_affine_q3.hpp"
#include "hyteg/forms/form_hyteg_generated/p1/p1_div_k_grad_blending_q3.hpp"

bool hyteg::GeometryMap::verifyPointPairing( const Point3D&, const Point3D&, real_t ) const
{
   return true;
}

namespace {
using namespace hyteg;

void buildStorage( const double* V, long nv, const long* T, long nt, SetupPrimitiveStorage& s )
{
   std::map< std::array< long, 3 >, PrimitiveID > faceIds;
   long                                          next = nv;
   static const int kFace[4][3] = { { 0, 1, 2 }, { 0, 1, 3 }, { 0, 2, 3 }, { 1, 2, 3 } };
   for ( long c = 0; c < nt; ++c )
   {
      auto cell = std::make_shared< Cell >();
      for ( int k = 0; k < 4; ++k )
      {
         const long v = T[4 * c + k];
         cell->verts.push_back( PrimitiveID{ v } );
         cell->coords[size_t( k )] = Point3D( V[3 * v], V[3 * v + 1], V[3 * v + 2] );
      }
      for ( const auto& f : kFace )
      {
         std::array< long, 3 > key = { T[4 * c + f[0]], T[4 * c + f[1]], T[4 * c + f[2]] };
         std::sort( key.begin(), key.end() );
         auto it = faceIds.find( key );
         if ( it == faceIds.end() )
         {
            it            = faceIds.emplace( key, PrimitiveID{ next++ } ).first;
            auto face     = std::make_shared< Face >();
            face->id      = it->second;
            for ( long v : key )
               face->verts.push_back( PrimitiveID{ v } );
            s.faces[face->id] = face;
         }
         cell->faces.push_back( it->second );
      }
      cell->id = PrimitiveID{ -( c + 1 ) };
      s.cells[cell->id] = cell;
   }
   // faces list their cells in cell order
   for ( long c = 0; c < nt; ++c )
   {
      const Cell& cell = *s.cells.at( PrimitiveID{ -( c + 1 ) } );
      for ( const auto& f : cell.faces )
         s.faces.at( f )->cells.push_back( cell.id );
   }
}
} // namespace

extern "C" {

int ref_shell_map_eval( const double* V, long nv, const long* T, long nt, int cell, const double* x, double* Fx,
                        double* DF )
{
   try
   {
      SetupPrimitiveStorage s;
      buildStorage( V, nv, T, nt, s );
      IcosahedralShellMap map( *s.getCell( PrimitiveID{ -( long( cell ) + 1 ) } ), s );
      Point3D  out;
      Matrix3r D;
      map.evalF( Point3D( x[0], x[1], x[2] ), out );
      map.evalDF( Point3D( x[0], x[1], x[2] ), D );
      for ( int i = 0; i < 3; ++i )
      {
         Fx[i] = out[size_t( i )];
         for ( int j = 0; j < 3; ++j )
            DF[3 * i + j] = D( i, j );
      }
      return 0;
   } catch ( const std::exception& )
   {
      return -1;
   }
}

int ref_blend_element_matrix( const double* V, long nv, const long* T, long nt, int cell, const double* X12, double alpha,
                              double* out16 )
{
   try
   {
      SetupPrimitiveStorage s;
      buildStorage( V, nv, T, nt, s );
      auto map = std::make_shared< IcosahedralShellMap >( *s.getCell( PrimitiveID{ -( long( cell ) + 1 ) } ), s );
      auto k   = [alpha]( const Point3D& y ) { return std::exp( alpha * ( 1.0 - y.norm() ) ); };
      forms::p1_div_k_grad_blending_q3 form( k, k );
      form.setGeometryMap( map );
      std::array< Point3D, 4 > X;
      for ( int j = 0; j < 4; ++j )
         X[size_t( j )] = Point3D( X12[3 * j], X12[3 * j + 1], X12[3 * j + 2] );
      Matrix< real_t, 4, 4 > A;
      form.integrateAll( X, A );
      for ( int i = 0; i < 4; ++i )
         for ( int j = 0; j < 4; ++j )
            out16[4 * i + j] = A( i, j );
      return 0;
   } catch ( const std::exception& )
   {
      return -1;
   }
}

// p1_div_k_grad_affine_q3::integrateAll on the tetrahedron X12 with the coefficient callback
// kind 0: the P1 interpolant of the nodal values k4 on that tetrahedron; kind 1:
// tanh(2 (x - 1/2)) + 2 (tests/hyteg/convergence/ElementwiseDivKGradCGConvergenceTest.cpp)
int ref_divkgrad_affine_element_matrix( const double* X12, int kind, const double* k4, double* out16 )
{
   if ( kind != 0 && kind != 1 )
      return -1;
   std::array< Point3D, 4 > X;
   for ( int j = 0; j < 4; ++j )
      X[size_t( j )] = Point3D( X12[3 * j], X12[3 * j + 1], X12[3 * j + 2] );
   // barycentric coordinates of y: solve [X1-X0 X2-X0 X3-X0] l = y - X0
   auto interp = [&]( const Point3D& y ) {
      double J[3][3], r[3];
      for ( int d = 0; d < 3; ++d )
      {
         for ( int c = 0; c < 3; ++c )
            J[d][c] = X[size_t( c + 1 )][size_t( d )] - X[0][size_t( d )];
         r[d] = y[size_t( d )] - X[0][size_t( d )];
      }
      const double det = J[0][0] * ( J[1][1] * J[2][2] - J[1][2] * J[2][1] ) -
                         J[0][1] * ( J[1][0] * J[2][2] - J[1][2] * J[2][0] ) +
                         J[0][2] * ( J[1][0] * J[2][1] - J[1][1] * J[2][0] );
      double l[3];
      for ( int c = 0; c < 3; ++c )
      {
         double M[3][3];
         for ( int a = 0; a < 3; ++a )
            for ( int b = 0; b < 3; ++b )
               M[a][b] = b == c ? r[a] : J[a][b];
         l[c] = ( M[0][0] * ( M[1][1] * M[2][2] - M[1][2] * M[2][1] ) - M[0][1] * ( M[1][0] * M[2][2] - M[1][2] * M[2][0] ) +
                  M[0][2] * ( M[1][0] * M[2][1] - M[1][1] * M[2][0] ) ) /
                 det;
      }
      return ( 1.0 - l[0] - l[1] - l[2] ) * k4[0] + l[0] * k4[1] + l[1] * k4[2] + l[2] * k4[3];
   };
   std::function< real_t( const Point3D& ) > k;
   if ( kind == 0 )
      k = interp;
   else
      k = []( const Point3D& y ) { return std::tanh( 2.0 * ( y[0] - 0.5 ) ) + 2.0; };
   forms::p1_div_k_grad_affine_q3 form( k, k );
   Matrix< real_t, 4, 4 >         A;
   form.integrateAll( X, A );
   for ( int i = 0; i < 4; ++i )
      for ( int j = 0; j < 4; ++j )
         out16[4 * i + j] = A( i, j );
   return 0;
}
}
