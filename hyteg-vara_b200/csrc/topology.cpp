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

// Thick spherical shell: MeshInfo::meshSphericalShell( ntan, nrad, rmin, rmax ) with the
// reference's default meshing SHELLMESH_CLASSIC (src/hyteg/mesh/MeshGenSphericalShell.cpp:
// 577-900), restated. The unit sphere is the icosahedron seen as ten "diamonds" (pairs of
// triangles sharing an edge, five around each pole), each refined by repeated arc midpoints
// into an ntan x ntan grid of nodes (ntan - 1 a power of two); the nodes are scaled to nrad
// equidistant radii. Vertex ids: the north pole of every radius, then the south poles, then
// radius by radius the other nodes diamond by diamond. Every grid square between two radii
// is a prism-like local cell of 8 vertices split into 6 tetrahedra by fixed tables (one for
// each hemisphere). Cells come out in the order of the reference's cell map: sorted by their
// vertex-id lists. The tables (icosahedral nodes, diamond corners, local-cell offsets, the
// two tetrahedron splits) must be the reference's for the meshes to be the same.
void meshSphericalShell( int ntan, int nrad, double rmin, double rmax, std::vector< std::array< double, 3 > >& V,
                         std::vector< std::array< int, 4 > >& T )
{
   if ( ntan < 2 || nrad < 2 )
      throw std::invalid_argument( "meshSphericalShell: need ntan >= 2 and nrad >= 2" );
   if ( !( rmin > 0 ) || !( rmin < rmax ) )
      throw std::invalid_argument( "meshSphericalShell: need 0 < rmin < rmax" );
   const int n1 = ntan - 1;
   if ( ( n1 & ( n1 - 1 ) ) != 0 )
      throw std::invalid_argument( "meshSphericalShell: ntan - 1 must be a power of two" );
   std::vector< double > radius( static_cast< size_t >( nrad ), 0.0 );
   for ( int l = 0; l < nrad; ++l )
      radius[size_t( l )] = rmin + ( ( rmax - rmin ) / double( nrad - 1 ) ) * double( l );

   // the twelve icosahedral nodes: poles 0 and 11, an upper ring 1..5 and a lower ring 6..10
   // of pentagons, each ring counter-clockwise
   double       ico[12][3];
   const double fifthPi = 0.4 * std::asin( 1.0 );
   const double w       = 2.0 * std::acos( 1.0 / ( 2.0 * std::sin( fifthPi ) ) );
   const double cw = std::cos( w ), sw = std::sin( w );
   ico[0][0] = 0.0, ico[0][1] = 0.0, ico[0][2] = 1.0;
   ico[11][0] = 0.0, ico[11][1] = 0.0, ico[11][2] = -1.0;
   for ( int k = 1; k <= 5; ++k )
   {
      const double up = 2.0 * ( double( k ) - 0.5 ) * fifthPi, lo = 2.0 * ( double( k ) - 1 ) * fifthPi;
      ico[k][0] = sw * std::cos( up ), ico[k][1] = sw * std::sin( up ), ico[k][2] = cw;
      ico[k + 5][0] = sw * std::cos( lo ), ico[k + 5][1] = sw * std::sin( lo ), ico[k + 5][2] = -cw;
   }
   // diamond corners: pole, then counter-clockwise (left, bottom, right on the north side)
   static const int diamond[10][4] = { { 0, 5, 6, 1 },   { 0, 1, 7, 2 },  { 0, 2, 8, 3 },  { 0, 3, 9, 4 },
                                       { 0, 4, 10, 5 },  { 11, 7, 1, 6 }, { 11, 8, 2, 7 }, { 11, 9, 3, 8 },
                                       { 11, 10, 4, 9 }, { 11, 6, 5, 10 } };
   // unit-sphere node (i1, i2) of diamond d: arc midpoints, level by level
   std::vector< double > node( size_t( ntan ) * ntan * 10 * 3, 0.0 );
   auto nd = [&]( int i1, int i2, int d ) { return &node[( ( size_t( i1 ) * ntan + i2 ) * 10 + d ) * 3]; };
   auto midpoint = [&]( double* out, const double* p, const double* q ) {
      const double x = p[0] + q[0], y = p[1] + q[1], z = p[2] + q[2];
      const double s = std::sqrt( x * x + y * y + z * z );
      out[0] = x / s, out[1] = y / s, out[2] = z / s;
   };
   for ( int d = 0; d < 10; ++d )
   {
      const int left = d < 5 ? 1 : 3, right = d < 5 ? 3 : 1; // mirrored on the south side
      std::copy( ico[diamond[d][0]], ico[diamond[d][0]] + 3, nd( 0, 0, d ) );
      std::copy( ico[diamond[d][left]], ico[diamond[d][left]] + 3, nd( n1, 0, d ) );
      std::copy( ico[diamond[d][2]], ico[diamond[d][2]] + 3, nd( n1, n1, d ) );
      std::copy( ico[diamond[d][right]], ico[diamond[d][right]] + 3, nd( 0, n1, d ) );
      for ( int m = 1; m < n1; m *= 2 )
      {
         const int l = n1 / m, h = l / 2;
         for ( int a = 0; a <= m; ++a ) // along i2 on the lines i1 = a l
            for ( int b = 0; b < m; ++b )
               midpoint( nd( a * l, b * l + h, d ), nd( a * l, b * l, d ), nd( a * l, b * l + l, d ) );
         for ( int a = 0; a <= m; ++a ) // along i1 on the lines i2 = a l
            for ( int b = 0; b < m; ++b )
               midpoint( nd( b * l + h, a * l, d ), nd( b * l, a * l, d ), nd( b * l + l, a * l, d ) );
         for ( int a = 0; a < m; ++a ) // the diagonals (i1 - h, i2 + h) -- (i1 + h, i2 - h)
            for ( int b = 0; b < m; ++b )
               midpoint( nd( a * l + h, b * l + h, d ), nd( a * l, b * l + l, d ), nd( a * l + l, b * l, d ) );
      }
   }
   // vertex id of grid node (s1, s2) of diamond d on radius r; nodes on a diamond's left
   // edges are stored with the neighbouring diamond that owns them
   const int perLayer = 10 * n1 * n1;
   auto      vertexId = [&]( int s1, int s2, int d, int r ) {
      if ( s1 == 0 && s2 == 0 )
         return d < 5 ? r : nrad + r;
      if ( s2 == 0 )
      {
         s2 = s1;
         s1 = 0;
         d  = d < 5 ? ( d + 4 ) % 5 : ( d + 4 ) % 5 + 5;
      }
      else if ( s1 == n1 )
      {
         s1 = n1 - s2;
         s2 = n1;
         d  = d < 5 ? ( d + 4 ) % 5 + 5 : d % 5;
      }
      return 2 * nrad + r * perLayer + d * n1 * n1 + ( s2 - 1 ) * n1 + s1;
   };
   V.assign( size_t( ( perLayer + 2 ) * nrad ), { 0.0, 0.0, 0.0 } );
   for ( int id = 0; id < ( perLayer + 2 ) * nrad; ++id )
   {
      int s1 = 0, s2 = 0, d = 0, r = 0;
      if ( id < nrad )
         r = id;
      else if ( id < 2 * nrad )
         d = 5, r = id - nrad;
      else
      {
         int k = id - 2 * nrad;
         r     = k / perLayer;
         k -= r * perLayer;
         d = k / ( n1 * n1 );
         k -= d * n1 * n1;
         s2 = k / n1 + 1;
         s1 = k - ( s2 - 1 ) * n1;
      }
      const double* u = nd( s1, s2, d );
      V[size_t( id )] = { u[0] * radius[size_t( r )], u[1] * radius[size_t( r )], u[2] * radius[size_t( r )] };
   }
   // local cell of grid square (s1, s2) between radii r and r + 1: corner k at offsets
   // (ds1, ds2, dr) (ds1 and ds2 swapped on the south side), split into six tetrahedra
   static const int corner[8][3] = { { 0, 0, 1 }, { 1, 0, 1 }, { 1, 1, 1 }, { 0, 1, 1 },
                                     { 0, 0, 0 }, { 1, 0, 0 }, { 1, 1, 0 }, { 0, 1, 0 } };
   static const int north[6][4]  = { { 0, 1, 3, 7 }, { 4, 7, 5, 0 }, { 0, 5, 1, 7 },
                                     { 1, 2, 3, 6 }, { 5, 7, 6, 1 }, { 3, 6, 7, 1 } };
   static const int south[6][4]  = { { 4, 7, 5, 1 }, { 0, 1, 3, 4 }, { 4, 3, 7, 1 },
                                     { 7, 6, 5, 2 }, { 3, 1, 2, 7 }, { 5, 2, 1, 7 } };
   std::vector< std::array< int, 4 > > cells;
   for ( int r = 0; r + 1 < nrad; ++r )
      for ( int d = 0; d < 10; ++d )
         for ( int s2 = 0; s2 < n1; ++s2 )
            for ( int s1 = 0; s1 < n1; ++s1 )
            {
               int v[8];
               for ( int k = 0; k < 8; ++k )
               {
                  const int a = d <= 4 ? corner[k][0] : corner[k][1], b = d <= 4 ? corner[k][1] : corner[k][0];
                  v[k] = vertexId( s1 + a, s2 + b, d, r + corner[k][2] );
               }
               for ( int t = 0; t < 6; ++t )
               {
                  const int( &tab )[4] = d <= 4 ? north[t] : south[t];
                  cells.push_back( { v[tab[0]], v[tab[1]], v[tab[2]], v[tab[3]] } );
               }
            }
   std::sort( cells.begin(), cells.end() );
   T = cells;
}

} // namespace hyb
