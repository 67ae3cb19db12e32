// C ABI (ours) over the reference's MeshInfo::meshSphericalShell
// (src/hyteg/mesh/MeshGenSphericalShell.cpp, SHELLMESH_CLASSIC), compiled unchanged from
// the reference source tree against the MeshInfo shim in ref_shim_mesh/.
// TEST INFRASTRUCTURE ONLY: it generates the golden shell meshes that pin the product's
// restated generator (tests/golden/make_shell_mesh_golden.py, tests/test_shell_mesh.py).
#include "hyteg/mesh/MeshInfo.hpp"

extern "C" {

// counts[0] = vertices, counts[1] = cells; with coords / tets non-null, also the vertices in
// id order (x, y, z) and the cells in the order of the reference's cell map (each cell's
// vertex ids in the order the generator gives them)
int ref_mesh_spherical_shell( int ntan, int nrad, double rmin, double rmax, long* counts, double* coords, long* tets )
{
   try
   {
      const hyteg::MeshInfo m = hyteg::MeshInfo::meshSphericalShell( hyteg::uint_t( ntan ), hyteg::uint_t( nrad ), rmin, rmax );
      counts[0] = long( m.getVertices().size() );
      counts[1] = long( m.getCells().size() );
      if ( coords )
         for ( const auto& v : m.getVertices() )
            for ( int d = 0; d < 3; ++d )
               coords[3 * long( v.first ) + d] = v.second.coords[std::size_t( d )];
      if ( tets )
      {
         long c = 0;
         for ( const auto& cell : m.getCells() )
         {
            for ( int k = 0; k < 4; ++k )
               tets[4 * c + k] = long( cell.first[std::size_t( k )] );
            ++c;
         }
      }
      return 0;
   } catch ( const std::exception& )
   {
      return -1;
   }
}
}
