// Shim (ours): the part of the reference's MeshInfo that MeshGenSphericalShell.cpp fills --
// vertices, edges, faces and cells in ordered maps keyed like the reference's containers
// (vertex id; sorted edge pair; face and cell vertex lists as given), the shell-mesh and
// hollow-flag enums, and the generator entry points.
#pragma once
#include <algorithm>
#include <array>
#include <map>
#include <vector>

#include "hyteg/types/PointND.hpp"

namespace walberla {
template < typename T >
inline uint_t uint_c( T x )
{
   return uint_t( x );
}
} // namespace walberla

namespace hyteg {
using walberla::real_t;
using walberla::uint_t;

class MeshInfo
{
 public:
   typedef uint_t IDType;
   typedef enum
   {
      SHELLMESH_ON_THE_FLY,
      SHELLMESH_CLASSIC
   } shellMeshType;
   typedef enum
   {
      flagInterior      = 0,
      flagInnerBoundary = 1,
      flagOuterBoundary = 2
   } hollowFlag;

   struct Vertex
   {
      Vertex() = default;
      Vertex( IDType i, const Point3D& c, uint_t f )
      : id( i )
      , coords( c )
      , flag( f )
      {}
      IDType  id   = 0;
      Point3D coords;
      uint_t  flag = 0;
   };
   struct Edge
   {
      Edge() = default;
      Edge( const std::array< IDType, 2 >& v, uint_t f )
      : verts( v )
      , flag( f )
      {}
      std::array< IDType, 2 > verts{};
      uint_t                  flag = 0;
   };
   struct Face
   {
      Face() = default;
      Face( const std::vector< IDType >& v, uint_t f )
      : verts( v )
      , flag( f )
      {}
      std::vector< IDType > verts;
      uint_t                flag = 0;
   };
   struct Cell
   {
      Cell() = default;
      Cell( const std::vector< IDType >& v, uint_t f )
      : verts( v )
      , flag( f )
      {}
      std::vector< IDType > verts;
      uint_t                flag = 0;
   };

   const std::map< IDType, Vertex >&                    getVertices() const { return vertices_; }
   const std::map< std::array< IDType, 2 >, Edge >&     getEdges() const { return edges_; }
   const std::map< std::vector< IDType >, Face >&       getFaces() const { return faces_; }
   const std::map< std::vector< IDType >, Cell >&       getCells() const { return cells_; }

   static MeshInfo meshSphericalShell( uint_t ntan, uint_t nrad, real_t rmin, real_t rmax,
                                       shellMeshType meshType = shellMeshType::SHELLMESH_CLASSIC );
   static MeshInfo meshSphericalShell( uint_t ntan, const std::vector< real_t >& layers,
                                       shellMeshType meshType = shellMeshType::SHELLMESH_CLASSIC );
   static MeshInfo meshThinSphericalShell( uint_t ntan, real_t radius );

   void computeSphericalShellVertices( uint_t ntan, const std::vector< real_t >& layers, MeshInfo::shellMeshType meshType );

   void addEdge( const Edge& e )
   {
      std::array< IDType, 2 > k = e.verts;
      std::sort( k.begin(), k.end() );
      edges_.emplace( k, e );
   }
   void addFace( const Face& f )
   {
      std::vector< IDType > k = f.verts;
      std::sort( k.begin(), k.end() );
      faces_.emplace( k, f );
   }
   void deduceEdgeFlagsFromVertices( uint_t ) {}
   void deduceFaceFlagsFromVertices( uint_t ) {}

 private:
   std::map< IDType, Vertex >                vertices_;
   std::map< std::array< IDType, 2 >, Edge > edges_;
   std::map< std::vector< IDType >, Face >   faces_;
   std::map< std::vector< IDType >, Cell >   cells_;
};
} // namespace hyteg
