// Shim (ours): the macro-primitive queries IcosahedralShellMap makes (coordinates, vertex
// and face neighbours of a cell, the cells of a face), over a mesh given as arrays.
#pragma once
#include <array>
#include <map>
#include <memory>
#include <vector>

#include "core/Abort.h"
#include "hyteg/types/PointND.hpp"

namespace hyteg {
class GeometryMap;

struct PrimitiveID
{
   long id = -1;
   bool operator==( const PrimitiveID& o ) const { return id == o.id; }
   bool operator!=( const PrimitiveID& o ) const { return id != o.id; }
   bool operator<( const PrimitiveID& o ) const { return id < o.id; }
};

struct Cell
{
   PrimitiveID                  id;
   std::array< Point3D, 4 >     coords;
   std::vector< PrimitiveID >   verts, faces;
   PrimitiveID                  getID() const { return id; }
   const std::array< Point3D, 4 >& getCoordinates() const { return coords; }
   void getNeighborVertices( std::vector< PrimitiveID >& v ) const { v = verts; }
   void getNeighborFaces( std::vector< PrimitiveID >& f ) const { f = faces; }
   uint_t getLocalVertexID( const PrimitiveID& v ) const
   {
      for ( uint_t k = 0; k < verts.size(); ++k )
         if ( verts[k] == v )
            return k;
      return 4;
   }
};

struct Face
{
   PrimitiveID                id;
   std::vector< PrimitiveID > verts, cells;
   PrimitiveID                getID() const { return id; }
   void getNeighborVertices( std::vector< PrimitiveID >& v ) const { v = verts; }
   void getNeighborCells( std::vector< PrimitiveID >& c ) const { c = cells; }
};

struct Edge
{
   PrimitiveID                id;
   std::vector< PrimitiveID > cells;
   PrimitiveID                getID() const { return id; }
   void getNeighborCells( std::vector< PrimitiveID >& c ) const { c = cells; }
};

class SetupPrimitiveStorage
{
 public:
   std::map< PrimitiveID, std::shared_ptr< Cell > > cells;
   std::map< PrimitiveID, std::shared_ptr< Face > > faces;
   std::map< PrimitiveID, std::shared_ptr< Edge > > edges;

   const Cell* getCell( const PrimitiveID& id ) const { return cells.at( id ).get(); }
   const Face* getFace( const PrimitiveID& id ) const { return faces.at( id ).get(); }
   const std::map< PrimitiveID, std::shared_ptr< Cell > >& getCells() const { return cells; }
   const std::map< PrimitiveID, std::shared_ptr< Face > >& getFaces() const { return faces; }
   const std::map< PrimitiveID, std::shared_ptr< Edge > >& getEdges() const { return edges; }
   void setGeometryMap( const PrimitiveID&, const std::shared_ptr< GeometryMap >& ) {}
};
} // namespace hyteg
