// Host-side macro-mesh topology for the P1 multigrid hierarchy.
//
// Mirrors what the reference's SetupPrimitiveStorage builds from a MeshInfo
// (src/hyteg/primitivestorage/SetupPrimitiveStorage.cpp:63-366): macro-vertices
// in mesh order, macro-edges and macro-faces keyed by their sorted vertex ids
// (MeshInfo::addEdge/addFace, src/hyteg/mesh/MeshInfo.cpp:37-72), macro-cells in
// the given order with their given vertex order, and the boundary flags of
// setMeshBoundaryFlagsOnBoundary(1, 0, true) + BoundaryCondition::create0123BC
// (flag 1 -> DirichletBoundary, otherwise Inner).
//
// The device never sees these maps: build() flattens them into the small
// integer tables of DeviceTopology (per-cell class info and per-primitive cell
// embeddings) that the kernels use.
#pragma once

#include <array>
#include <cstdint>
#include <map>
#include <string>
#include <vector>

namespace hyb {

// DoFType bit flags (src/hyteg/types/types.hpp:35-44)
enum : uint8_t
{
   kInner     = 1,
   kDirichlet = 2,
   kNeumann   = 4,
   kFreeslip  = 8,
   kAll       = 15
};

// One embedding of a lower-dimensional macro-primitive into an adjacent cell:
// the cell and the cell-local indices (0..3) of the primitive's vertices in the
// primitive's own (sorted) vertex order.
struct Embedding
{
   int     cell;
   uint8_t k[3];
};

// Packed form used on the device: cell | k0<<24 | k1<<26 | k2<<28
inline int32_t packEmbedding( const Embedding& e )
{
   return int32_t( uint32_t( e.cell ) | ( uint32_t( e.k[0] ) << 24 ) | ( uint32_t( e.k[1] ) << 26 ) |
                   ( uint32_t( e.k[2] ) << 28 ) );
}

struct Topology
{
   std::vector< std::array< double, 3 > > V;
   std::vector< std::array< int, 4 > >    T;
   std::vector< std::array< int, 2 > >    E;
   std::vector< std::array< int, 3 > >    F;
   std::map< std::array< int, 2 >, int >  edgeId;
   std::map< std::array< int, 3 >, int >  faceId;
   std::vector< uint8_t >                 vBc, eBc, fBc;
   std::vector< std::vector< Embedding > > vEmb, eEmb, fEmb;

   // per cell and class mask (bit k set <=> barycentric coordinate k is zero):
   // the sub-primitive's kind (0 vertex .. 3 cell), id, BC, #adjacent cells,
   // and whether this cell owns the sub-primitive (its first adjacent cell)
   struct ClassInfo
   {
      int8_t  kind;
      int32_t id;
      uint8_t bc;
      int32_t ncells;
      bool    owned;
   };
   std::vector< std::array< ClassInfo, 16 > > cls;

   // colour labels per macro-vertex for multicolour SOR and the modulus
   std::vector< int > labels;
   int                colours = 0;

   void build( const std::vector< std::array< double, 3 > >& coords, const std::vector< std::array< int, 4 > >& tets );
   // Search labels l(v) in Z_m (m = 4, 5, ...) such that the colouring
   // c(p) = sum_k l(V_k) b_k(p) mod m separates every coupled pair of micro-vertices.
   void computeColouring( int maxColours = 16 );
   // check the colouring constraint on every cell (used by tests)
   bool colouringValid() const;

   int64_t numDofs( int level ) const;
};

// Mesh generators (restated from the reference's MeshInfo factories)
void meshCuboid( int nx, int ny, int nz, const double lo[3], const double hi[3], std::vector< std::array< double, 3 > >& V,
                 std::vector< std::array< int, 4 > >& T );
void meshSphericalShell( int ntan, int nrad, double rmin, double rmax, std::vector< std::array< double, 3 > >& V,
                         std::vector< std::array< int, 4 > >& T );
void readGmsh( const std::string& path, std::vector< std::array< double, 3 > >& V, std::vector< std::array< int, 4 > >& T );

} // namespace hyb
