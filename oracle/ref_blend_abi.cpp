// C ABI (ours) over the reference's IcosahedralShellMap and p1_div_k_grad_blending_q3 form,
// compiled unchanged from the reference source tree against the shims in ref_shim_blend/.
// TEST INFRASTRUCTURE ONLY: it pins the oracle's restatement of the shell map and of the
// blended element matrix (tests/test_blend_oracle.py, tests/golden/make_blend_golden.py).
//
// The mesh is given as arrays (vertex coordinates, cell vertex lists); the storage shim is
// filled the way SetupPrimitiveStorage orders it (src/hyteg/primitivestorage/
// SetupPrimitiveStorage.cpp:244-300): a cell's faces are (v0 v1 v2), (v0 v1 v3), (v0 v2 v3),
// (v1 v2 v3), and a face lists its cells in cell order.
#include <algorithm>
#include <cmath>

#include "hyteg/geometry/IcosahedralShellMap.hpp"
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
}
