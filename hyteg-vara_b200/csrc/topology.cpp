// Host-side macro-mesh topology (see topology.hpp).
#include "topology.hpp"
#include <fstream>
#include <map>
#include <string>

#include <algorithm>
#include <cmath>
#include <numeric>
#include <queue>
#include <random>
#include <set>
#include <stdexcept>

namespace hyb {

namespace {
const int kFaceLocal[4][3] = { { 0, 1, 2 }, { 0, 1, 3 }, { 0, 2, 3 }, { 1, 2, 3 } };
}

void Topology::build( const std::vector< std::array< double, 3 > >& coords, const std::vector< std::array< int, 4 > >& tets )
{
   V = coords;
   T = tets;
   E.clear();
   F.clear();
   edgeId.clear();
   faceId.clear();
   for ( auto& t : T )
      for ( int k = 0; k < 4; ++k )
      {
         if ( t[k] < 0 || t[k] >= int( V.size() ) )
            throw std::invalid_argument( "tetrahedron references a vertex id outside the vertex list" );
         for ( int j = k + 1; j < 4; ++j )
            if ( t[j] == t[k] )
               throw std::invalid_argument( "tetrahedron with repeated vertex" );
      }
   // edges and faces keyed by sorted vertex ids, numbered in key order
   std::set< std::array< int, 2 > > es;
   std::set< std::array< int, 3 > > fs;
   for ( auto& t : T )
   {
      for ( int a = 0; a < 4; ++a )
         for ( int b = a + 1; b < 4; ++b )
            es.insert( { std::min( t[a], t[b] ), std::max( t[a], t[b] ) } );
      for ( auto& f : kFaceLocal )
      {
         std::array< int, 3 > key = { t[f[0]], t[f[1]], t[f[2]] };
         std::sort( key.begin(), key.end() );
         fs.insert( key );
      }
   }
   for ( auto& e : es )
   {
      edgeId[e] = int( E.size() );
      E.push_back( e );
   }
   for ( auto& f : fs )
   {
      faceId[f] = int( F.size() );
      F.push_back( f );
   }
   // embeddings of every lower-dimensional primitive into its adjacent cells,
   // cells visited in order, so the first embedding is the owning cell
   vEmb.assign( V.size(), {} );
   eEmb.assign( E.size(), {} );
   fEmb.assign( F.size(), {} );
   for ( int c = 0; c < int( T.size() ); ++c )
   {
      const auto& t     = T[c];
      auto        local = [&]( int v ) {
         for ( int k = 0; k < 4; ++k )
            if ( t[k] == v )
               return uint8_t( k );
         return uint8_t( 255 );
      };
      for ( int k = 0; k < 4; ++k )
         vEmb[t[k]].push_back( { c, { uint8_t( k ), 0, 0 } } );
      for ( int a = 0; a < 4; ++a )
         for ( int b = a + 1; b < 4; ++b )
         {
            std::array< int, 2 > key = { std::min( t[a], t[b] ), std::max( t[a], t[b] ) };
            eEmb[edgeId[key]].push_back( { c, { local( key[0] ), local( key[1] ), 0 } } );
         }
      for ( auto& f : kFaceLocal )
      {
         std::array< int, 3 > key = { t[f[0]], t[f[1]], t[f[2]] };
         std::sort( key.begin(), key.end() );
         fEmb[faceId[key]].push_back( { c, { local( key[0] ), local( key[1] ), local( key[2] ) } } );
      }
   }
   for ( auto& fe : fEmb )
      if ( fe.size() > 2 )
         throw std::invalid_argument( "non-manifold mesh: a face with more than two cells" );
   // boundary flags (SetupPrimitiveStorage::onBoundary, 3D branch: a face with one cell is on
   // the boundary, and so is every edge and vertex of such a face)
   vBc.assign( V.size(), kInner );
   eBc.assign( E.size(), kInner );
   fBc.assign( F.size(), kInner );
   for ( size_t f = 0; f < F.size(); ++f )
      if ( fEmb[f].size() == 1 )
      {
         fBc[f] = kDirichlet;
         const auto& k = F[f];
         eBc[edgeId[{ k[0], k[1] }]] = kDirichlet;
         eBc[edgeId[{ k[0], k[2] }]] = kDirichlet;
         eBc[edgeId[{ k[1], k[2] }]] = kDirichlet;
         for ( int v : k )
            vBc[v] = kDirichlet;
      }
   // class table
   cls.assign( T.size(), {} );
   for ( int c = 0; c < int( T.size() ); ++c )
   {
      const auto& t = T[c];
      for ( int mask = 0; mask < 16; ++mask )
      {
         ClassInfo ci{ -1, -1, 0, 0, false };
         std::vector< int > vs;
         for ( int k = 0; k < 4; ++k )
            if ( !( mask & ( 1 << k ) ) )
               vs.push_back( t[k] );
         std::sort( vs.begin(), vs.end() );
         switch ( vs.size() )
         {
         case 4:
            ci = { 3, c, kInner, 1, true };
            break;
         case 3: {
            const int f = faceId.at( { vs[0], vs[1], vs[2] } );
            ci          = { 2, f, fBc[f], int32_t( fEmb[f].size() ), fEmb[f][0].cell == c };
            break;
         }
         case 2: {
            const int e = edgeId.at( { vs[0], vs[1] } );
            ci          = { 1, e, eBc[e], int32_t( eEmb[e].size() ), eEmb[e][0].cell == c };
            break;
         }
         case 1:
            ci = { 0, vs[0], vBc[vs[0]], int32_t( vEmb[vs[0]].size() ), vEmb[vs[0]][0].cell == c };
            break;
         default:
            break;
         }
         cls[c][mask] = ci;
      }
   }
}

int64_t Topology::numDofs( int level ) const
{
   const int64_t N = int64_t( 1 ) << level;
   const int64_t nIntFace = N >= 3 ? ( N - 1 ) * ( N - 2 ) / 2 : 0;
   const int64_t nIntCell = N >= 4 ? ( N - 3 ) * ( N - 2 ) * ( N - 1 ) / 6 : 0;
   return int64_t( V.size() ) + int64_t( E.size() ) * std::max< int64_t >( N - 1, 0 ) + int64_t( F.size() ) * nIntFace +
          int64_t( T.size() ) * nIntCell;
}

namespace {
inline int mod( int a, int m ) { return ( ( a % m ) + m ) % m; }

// Constraint of one cell given (possibly partial) labels; -1 = unassigned.
bool cellOk( const std::array< int, 4 >& l, int m )
{
   for ( int a = 0; a < 4; ++a )
      for ( int b = a + 1; b < 4; ++b )
         if ( l[a] >= 0 && l[b] >= 0 && mod( l[a] - l[b], m ) == 0 )
            return false;
   // the octahedron diagonal (-1,1,-1) couples b0+b2 against b1+b3
   if ( l[0] >= 0 && l[1] >= 0 && l[2] >= 0 && l[3] >= 0 && mod( l[0] + l[2] - l[1] - l[3], m ) == 0 )
      return false;
   return true;
}
} // namespace

namespace {
int cellViolations( const std::array< int, 4 >& l, int m )
{
   int v = 0;
   for ( int a = 0; a < 4; ++a )
      for ( int b = a + 1; b < 4; ++b )
         if ( mod( l[a] - l[b], m ) == 0 )
            ++v;
   if ( mod( l[0] + l[2] - l[1] - l[3], m ) == 0 )
      ++v;
   return v;
}

// Min-conflicts local search for a labelling with m colours: repeatedly take a random
// violated cell, one of its vertices, and give it the label that violates the fewest
// constraints of its cells (a random label one time in 20). Deterministic for a seed.
bool labelsByLocalSearch( const std::vector< std::array< int, 4 > >& T, const std::vector< std::vector< int > >& vCells,
                          int m, long iterations, uint32_t seed, std::vector< int >& lab )
{
   std::mt19937 rng( seed );
   const int    nc = int( T.size() ), nv = int( vCells.size() );
   lab.assign( nv, 0 );
   for ( auto& x : lab )
      x = int( rng() % uint32_t( m ) );
   std::vector< int > pos( nc, -1 ), bad, cands;
   auto viol = [&]( int c ) { return cellViolations( { lab[T[c][0]], lab[T[c][1]], lab[T[c][2]], lab[T[c][3]] }, m ); };
   auto update = [&]( int c ) {
      const bool v = viol( c ) > 0;
      if ( v && pos[c] < 0 )
      {
         pos[c] = int( bad.size() );
         bad.push_back( c );
      }
      else if ( !v && pos[c] >= 0 )
      {
         const int last = bad.back();
         bad[pos[c]]    = last;
         pos[last]      = pos[c];
         bad.pop_back();
         pos[c] = -1;
      }
   };
   for ( int c = 0; c < nc; ++c )
      update( c );
   for ( long it = 0; it < iterations && !bad.empty(); ++it )
   {
      const int c    = bad[rng() % bad.size()];
      const int v    = T[c][rng() % 4];
      int       best = 1 << 30;
      cands.clear();
      for ( int x = 0; x < m; ++x )
      {
         lab[v]   = x;
         int cost = 0;
         for ( int cc : vCells[v] )
            cost += viol( cc );
         if ( cost < best )
         {
            best = cost;
            cands.assign( 1, x );
         }
         else if ( cost == best )
            cands.push_back( x );
      }
      lab[v] = ( rng() % 20 == 0 ) ? int( rng() % uint32_t( m ) ) : cands[rng() % cands.size()];
      for ( int cc : vCells[v] )
         update( cc );
   }
   return bad.empty();
}
} // namespace

void Topology::computeColouring( int maxColours )
{
   const int nv = int( V.size() );
   std::vector< std::vector< int > > vCells( nv );
   for ( int c = 0; c < int( T.size() ); ++c )
      for ( int k = 0; k < 4; ++k )
         vCells[T[c][k]].push_back( c );
   // BFS order over the vertex graph keeps constraints local during backtracking
   std::vector< std::vector< int > > adj( nv );
   for ( auto& e : E )
   {
      adj[e[0]].push_back( e[1] );
      adj[e[1]].push_back( e[0] );
   }
   std::vector< int > order;
   std::vector< char > seen( nv, 0 );
   for ( int s = 0; s < nv; ++s )
   {
      if ( seen[s] )
         continue;
      std::queue< int > q;
      q.push( s );
      seen[s] = 1;
      while ( !q.empty() )
      {
         int v = q.front();
         q.pop();
         order.push_back( v );
         for ( int w : adj[v] )
            if ( !seen[w] )
            {
               seen[w] = 1;
               q.push( w );
            }
      }
   }
   for ( int m = 4; m <= maxColours; ++m )
   {
      std::vector< int > lab( nv, -1 );
      std::vector< int > next( nv, 0 );
      long               budget = 4000000;
      int                pos    = 0;
      bool               ok     = false;
      while ( budget-- > 0 )
      {
         if ( pos == nv )
         {
            ok = true;
            break;
         }
         if ( pos < 0 )
            break;
         const int v = order[pos];
         bool placed = false;
         while ( next[pos] < m )
         {
            lab[v] = next[pos]++;
            bool good = true;
            for ( int c : vCells[v] )
            {
               std::array< int, 4 > l = { lab[T[c][0]], lab[T[c][1]], lab[T[c][2]], lab[T[c][3]] };
               if ( !cellOk( l, m ) )
               {
                  good = false;
                  break;
               }
            }
            if ( good )
            {
               placed = true;
               break;
            }
         }
         if ( placed )
         {
            ++pos;
            if ( pos < nv )
               next[pos] = 0;
         }
         else
         {
            lab[v] = -1;
            next[pos] = 0;
            --pos;
         }
      }
      if ( ok )
      {
         labels  = lab;
         colours = m;
         break;
      }
   }
   if ( colours == 0 )
      throw std::runtime_error( "no valid multicolour labelling found" );
   // The backtracking gives up on a count once its budget is spent, which on the
   // icosahedral shells leaves 10 colours where 8 exist. On small meshes that needed 8 or
   // more, a local search tries two and then one colour fewer (fixed seeds and iteration
   // budgets, so the labelling is reproducible); every interface colour is one pass per
   // SOR sweep.
   if ( colours >= 8 && nv <= 4000 )
      for ( int m : { colours - 2, colours - 1 } )
      {
         std::vector< int > lab;
         bool               found = false;
         for ( uint32_t seed = 1; seed <= 4 && !found; ++seed )
            found = labelsByLocalSearch( T, vCells, m, 300000, seed, lab );
         if ( found )
         {
            labels  = lab;
            colours = m;
            break;
         }
      }
}

bool Topology::colouringValid() const
{
   if ( colours < 2 || labels.size() != V.size() )
      return false;
   for ( auto& t : T )
      if ( !cellOk( { labels[t[0]], labels[t[1]], labels[t[2]], labels[t[3]] }, colours ) )
         return false;
   return true;
}

// MeshInfo::meshCuboid (src/hyteg/mesh/MeshGenCuboid.cpp:34-160): vertices with x fastest,
// six tetrahedra per cube from the hexahedron node table, cells in the lexicographic order
// of their vertex-id lists (the std::map order in which SetupPrimitiveStorage numbers them).
void meshCuboid( int nx, int ny, int nz, const double lo[3], const double hi[3], std::vector< std::array< double, 3 > >& V,
                 std::vector< std::array< int, 4 > >& T )
{
   if ( nx < 1 || ny < 1 || nz < 1 )
      throw std::invalid_argument( "meshCuboid: need at least one cube per direction" );
   const double hx = ( hi[0] - lo[0] ) / nx, hy = ( hi[1] - lo[1] ) / ny, hz = ( hi[2] - lo[2] ) / nz;
   V.clear();
   T.clear();
   for ( int iz = 0; iz <= nz; ++iz )
      for ( int iy = 0; iy <= ny; ++iy )
         for ( int ix = 0; ix <= nx; ++ix )
            V.push_back( { lo[0] + ix * hx, lo[1] + iy * hy, lo[2] + iz * hz } );
   const int tNode[6][4] = { { 4, 5, 7, 3 }, { 0, 3, 1, 4 }, { 4, 1, 5, 3 }, { 5, 6, 7, 2 }, { 1, 3, 2, 5 }, { 7, 2, 3, 5 } };
   const int off[8][3]   = { { 0, 0, 0 }, { 1, 0, 0 }, { 1, 1, 0 }, { 0, 1, 0 }, { 0, 0, 1 }, { 1, 0, 1 }, { 1, 1, 1 }, { 0, 1, 1 } };
   auto      vid         = [&]( int i, int j, int k ) { return k * ( nx + 1 ) * ( ny + 1 ) + j * ( nx + 1 ) + i; };
   std::set< std::array< int, 4 > > cells;
   for ( int iz = 0; iz < nz; ++iz )
      for ( int iy = 0; iy < ny; ++iy )
         for ( int ix = 0; ix < nx; ++ix )
            for ( auto& tn : tNode )
            {
               std::array< int, 4 > c;
               for ( int m = 0; m < 4; ++m )
                  c[m] = vid( ix + off[tn[m]][0], iy + off[tn[m]][1], iz + off[tn[m]][2] );
               cells.insert( c );
            }
   T.assign( cells.begin(), cells.end() );
}

// MeshInfo::fromGmshFile (src/hyteg/mesh/MeshGenFromGmshFile.cpp:36-190): Gmsh 2.2 ASCII.
// Vertices in ascending file id (made 0-based), tetrahedra (element type 4) in the
// lexicographic order of their vertex-index lists (the reference keeps them in a std::map
// keyed by that list); points (15), edges (1) and triangles (2) are read and skipped (their
// boundary tags are superseded by setMeshBoundaryFlagsOnBoundary). Any other element type
// is an error, as in the reference.
void readGmsh( const std::string& path, std::vector< std::array< double, 3 > >& V, std::vector< std::array< int, 4 > >& T )
{
   std::ifstream f( path );
   if ( !f )
      throw std::invalid_argument( "readGmsh: cannot open " + path );
   std::string tok;
   auto        expect = [&]( const char* want ) {
      if ( !( f >> tok ) || tok != want )
         throw std::invalid_argument( std::string( "readGmsh: expected " ) + want + " in " + path );
   };
   expect( "$MeshFormat" );
   if ( !( f >> tok ) || tok != "2.2" )
      throw std::invalid_argument( "readGmsh: only the Gmsh 2.2 ASCII format is supported" );
   int fileType = 0, dataSize = 0;
   f >> fileType >> dataSize;
   if ( fileType != 0 )
      throw std::invalid_argument( "readGmsh: binary Gmsh files are not supported" );
   expect( "$EndMeshFormat" );
   expect( "$Nodes" );
   long nNodes = 0;
   f >> nNodes;
   if ( !f || nNodes < 4 )
      throw std::invalid_argument( "readGmsh: bad node count" );
   std::map< long, std::array< double, 3 > > nodes;
   for ( long i = 0; i < nNodes; ++i )
   {
      long                    id;
      std::array< double, 3 > x;
      if ( !( f >> id >> x[0] >> x[1] >> x[2] ) )
         throw std::invalid_argument( "readGmsh: truncated $Nodes" );
      nodes[id] = x;
   }
   expect( "$EndNodes" );
   std::map< long, int > index;
   V.clear();
   for ( const auto& kv : nodes )
   {
      index[kv.first] = int( V.size() );
      V.push_back( kv.second );
   }
   expect( "$Elements" );
   long nElem = 0;
   f >> nElem;
   std::set< std::array< int, 4 > > cells;
   for ( long e = 0; e < nElem; ++e )
   {
      long id;
      int  type, ntags;
      if ( !( f >> id >> type >> ntags ) || ntags < 0 )
         throw std::invalid_argument( "readGmsh: truncated $Elements" );
      for ( int t = 0; t < ntags; ++t )
      {
         long tag;
         f >> tag;
      }
      const int nv = type == 15 ? 1 : type == 1 ? 2 : type == 2 ? 3 : type == 4 ? 4 : -1;
      if ( nv < 0 )
         throw std::invalid_argument( "readGmsh: unsupported element type " + std::to_string( type ) );
      std::array< int, 4 > c{};
      for ( int k = 0; k < nv; ++k )
      {
         long v;
         if ( !( f >> v ) )
            throw std::invalid_argument( "readGmsh: truncated element" );
         auto it = index.find( v );
         if ( it == index.end() )
            throw std::invalid_argument( "readGmsh: element refers to an unknown node" );
         if ( type == 4 )
            c[k] = it->second;
      }
      if ( type == 4 )
         cells.insert( c );
   }
   expect( "$EndElements" );
   if ( cells.empty() )
      throw std::invalid_argument( "readGmsh: no tetrahedra in " + path );
   T.assign( cells.begin(), cells.end() );
}

// Thick spherical shell (the mesh family of MeshInfo::meshSphericalShell,
// src/hyteg/mesh/MeshGenSphericalShell.cpp:579-690): the 20 faces of the icosahedron are
// each cut into (ntan - 1)^2 triangles, projected onto the unit sphere, and the sphere is
// repeated on nrad radii evenly spaced in [rmin, rmax]; every prism between two radii is
// split into three tetrahedra. This gives the reference's cell count,
// 60 (ntan - 1)^2 (nrad - 1), and vertex count, (10 (ntan - 1)^2 + 2) nrad, with affine
// macro-cells, but the triangulation of the sphere is this function's own (uniform
// barycentric subdivision of the icosahedron faces), not the reference's diamond meshing.
// Shared sphere points are computed once, from a canonical key, so coincident vertices
// are bitwise equal. Prism split: with the triangle's vertices in ascending id order
// (0, 1, 2) and b/t its bottom/top copies, the tetrahedra (b0 b1 b2 t2), (b0 b1 t1 t2),
// (b0 t0 t1 t2) cut every quadrilateral side from its lower-id bottom vertex to its
// higher-id top vertex, so neighbouring prisms agree on the shared diagonal.
void meshSphericalShell( int ntan, int nrad, double rmin, double rmax, std::vector< std::array< double, 3 > >& V,
                         std::vector< std::array< int, 4 > >& T )
{
   if ( ntan < 2 || nrad < 2 )
      throw std::invalid_argument( "meshSphericalShell: need ntan >= 2 and nrad >= 2" );
   if ( !( rmin > 0 ) || !( rmin < rmax ) )
      throw std::invalid_argument( "meshSphericalShell: need 0 < rmin < rmax" );
   const int    n   = ntan - 1;
   const double phi = ( 1.0 + std::sqrt( 5.0 ) ) / 2.0;
   // icosahedron: cyclic permutations of (0, +-1, +-phi)
   std::vector< std::array< double, 3 > > ico;
   for ( int a : { -1, 1 } )
      for ( int b : { -1, 1 } )
      {
         ico.push_back( { 0.0, double( a ), b * phi } );
         ico.push_back( { double( a ), b * phi, 0.0 } );
         ico.push_back( { b * phi, 0.0, double( a ) } );
      }
   auto dist2 = [&]( int i, int j ) {
      double d = 0;
      for ( int k = 0; k < 3; ++k )
         d += ( ico[i][k] - ico[j][k] ) * ( ico[i][k] - ico[j][k] );
      return d;
   };
   // faces: triples of mutually adjacent vertices (edge length 2)
   std::vector< std::array< int, 3 > > faces;
   for ( int i = 0; i < 12; ++i )
      for ( int j = i + 1; j < 12; ++j )
         for ( int k = j + 1; k < 12; ++k )
            if ( std::fabs( dist2( i, j ) - 4 ) < 1e-9 && std::fabs( dist2( i, k ) - 4 ) < 1e-9 &&
                 std::fabs( dist2( j, k ) - 4 ) < 1e-9 )
               faces.push_back( { i, j, k } );
   if ( faces.size() != 20 )
      throw std::logic_error( "meshSphericalShell: icosahedron construction failed" );
   // sphere points by canonical key: (kind, a, b, c) with kind 0 vertex (a), 1 edge point
   // (a < b, c steps from a), 2 face point (face a, i = b, j = c)
   std::map< std::array< int, 4 >, int >  key2id;
   std::vector< std::array< double, 3 > > S;
   auto point = [&]( const std::array< int, 4 >& key, const std::array< double, 3 >& x ) {
      auto it = key2id.find( key );
      if ( it != key2id.end() )
         return it->second;
      const double r = std::sqrt( x[0] * x[0] + x[1] * x[1] + x[2] * x[2] );
      S.push_back( { x[0] / r, x[1] / r, x[2] / r } );
      key2id[key] = int( S.size() ) - 1;
      return int( S.size() ) - 1;
   };
   auto mix = [&]( int a, double wa, int b, double wb, int c, double wc ) {
      std::array< double, 3 > x;
      for ( int k = 0; k < 3; ++k )
         x[k] = ( ico[a][k] * wa + ico[b][k] * wb + ico[c][k] * wc ) / n;
      return x;
   };
   std::vector< std::array< int, 3 > > tris;
   for ( int f = 0; f < 20; ++f )
   {
      const int a = faces[f][0], b = faces[f][1], c = faces[f][2]; // ascending
      auto      P = [&]( int i, int j ) {
         const int wa = n - i - j, wb = i, wc = j;
         if ( wb == 0 && wc == 0 )
            return point( { 0, a, 0, 0 }, ico[a] );
         if ( wa == 0 && wc == 0 )
            return point( { 0, b, 0, 0 }, ico[b] );
         if ( wa == 0 && wb == 0 )
            return point( { 0, c, 0, 0 }, ico[c] );
         if ( wc == 0 )
            return point( { 1, a, b, wb }, mix( a, wa, b, wb, c, 0 ) );
         if ( wb == 0 )
            return point( { 1, a, c, wc }, mix( a, wa, c, wc, b, 0 ) );
         if ( wa == 0 )
            return point( { 1, b, c, wc }, mix( b, wb, c, wc, a, 0 ) );
         return point( { 2, f, i, j }, mix( a, wa, b, wb, c, wc ) );
      };
      for ( int j = 0; j < n; ++j )
         for ( int i = 0; i + j < n; ++i )
         {
            tris.push_back( { P( i, j ), P( i + 1, j ), P( i, j + 1 ) } );
            if ( i + j + 1 < n )
               tris.push_back( { P( i + 1, j ), P( i + 1, j + 1 ), P( i, j + 1 ) } );
         }
   }
   const int nS = int( S.size() );
   V.clear();
   T.clear();
   for ( int l = 0; l < nrad; ++l )
   {
      const double r = rmin + ( rmax - rmin ) * l / ( nrad - 1 );
      for ( const auto& x : S )
         V.push_back( { r * x[0], r * x[1], r * x[2] } );
   }
   for ( auto t : tris )
   {
      std::sort( t.begin(), t.end() );
      for ( int l = 0; l + 1 < nrad; ++l )
      {
         const int b0 = l * nS + t[0], b1 = l * nS + t[1], b2 = l * nS + t[2];
         const int t0 = b0 + nS, t1 = b1 + nS, t2 = b2 + nS;
         T.push_back( { b0, b1, b2, t2 } );
         T.push_back( { b0, b1, t1, t2 } );
         T.push_back( { b0, t0, t1, t2 } );
      }
   }
}

} // namespace hyb
