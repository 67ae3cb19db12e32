// CPU oracle for the HyTeG P1 matrix-free geometric-multigrid path.
//
// TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline / reference arm load this library as the checker or the timed CPU
// baseline. The product path never links, loads or calls it.
//
// Design: one value per unique micro-vertex (global DoF vector in the canonical
// order documented in hyteg_oracle.h). Macro-cell closure points are mapped to
// DoFs through exact integer barycentric keys, so no face/edge permutation
// table is involved. Operators are evaluated row by row as the sum, over the
// macro-cells containing the DoF, of that cell's partial row -- exactly how the
// reference assembles its macro-face/edge/vertex stencils
// (src/hyteg/p1functionspace/P1Elements.hpp:464-526 calculateStencilInMacroCellForm_new,
//  P1Operator.hpp:1045-1175 apply_edge / apply_face3D).
#include "hyteg_oracle.h"
#ifdef _OPENMP
#include <omp.h>
#endif

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <set>
#include <stdexcept>
#include <vector>

namespace {

using i64 = int64_t;

// ---------------------------------------------------------------------------
// Index space (src/hyteg/Levelinfo.hpp:35-105, indexing/MacroCellIndexing.hpp:37-54)
// ---------------------------------------------------------------------------
inline i64 tetSize( i64 w ) { return ( w + 2 ) * ( w + 1 ) * w / 6; }
// linearMacroCellIndex( width, x, y, z )
inline i64 cellIdx( i64 width, i64 x, i64 y, i64 z )
{
   const i64 wms = width - z;
   return tetSize( width ) - tetSize( wms ) + y * ( wms + 1 ) - ( ( y + 1 ) * y ) / 2 + x;
}

// The 15 stencil offsets in the repository-wide order.
const int kOff[15][3] = { { 0, 0, 0 },  { 1, 0, 0 },  { -1, 0, 0 }, { 0, 1, 0 },  { 0, -1, 0 },
                          { 0, 0, 1 },  { 0, 0, -1 }, { -1, 1, 0 }, { 1, -1, 0 }, { -1, 0, 1 },
                          { 1, 0, -1 }, { 0, -1, 1 }, { 0, 1, -1 }, { -1, 1, -1 }, { 1, -1, 1 } };

int offsetId( int x, int y, int z )
{
   for ( int o = 0; o < 15; ++o )
      if ( kOff[o][0] == x && kOff[o][1] == y && kOff[o][2] == z )
         return o;
   return -1;
}

// Micro-cell types and their micro-vertices
// (src/hyteg/volumedofspace/CellDoFIndexing.hpp:38-46, 155-198).
const int kMicro[6][4][3] = {
    { { 0, 0, 0 }, { 1, 0, 0 }, { 0, 1, 0 }, { 0, 0, 1 } }, // WHITE_UP
    { { 1, 0, 0 }, { 1, 1, 0 }, { 0, 1, 0 }, { 1, 0, 1 } }, // BLUE_UP
    { { 1, 0, 0 }, { 0, 1, 0 }, { 1, 0, 1 }, { 0, 0, 1 } }, // GREEN_UP
    { { 1, 1, 0 }, { 1, 1, 1 }, { 0, 1, 1 }, { 1, 0, 1 } }, // WHITE_DOWN
    { { 1, 0, 1 }, { 0, 1, 1 }, { 0, 0, 1 }, { 0, 1, 0 } }, // BLUE_DOWN
    { { 0, 1, 0 }, { 1, 1, 0 }, { 1, 0, 1 }, { 0, 1, 1 } }, // GREEN_DOWN
};
// Micro-cells per row of each type: WHITE_UP N, WHITE_DOWN N-2, others N-1
// (CellDoFIndexing.hpp numCellsPerRowByType).
inline i64 microWidth( int type, i64 N ) { return type == 0 ? N : ( type == 3 ? N - 2 : N - 1 ); }

// The 24 micro-tets incident to a micro-vertex: (type, role k) -> vertex offsets
// relative to the vertex (vertex j of the tet at offset kMicro[t][j]-kMicro[t][k]).
struct Incident
{
   int t, k;
   int rel[4][3];
};
std::vector< Incident > makeIncident()
{
   std::vector< Incident > v;
   for ( int t = 0; t < 6; ++t )
      for ( int k = 0; k < 4; ++k )
      {
         Incident in{ t, k, {} };
         for ( int j = 0; j < 4; ++j )
            for ( int d = 0; d < 3; ++d )
               in.rel[j][d] = kMicro[t][j][d] - kMicro[t][k][d];
         v.push_back( in );
      }
   return v;
}
const std::vector< Incident > kIncident = makeIncident();

// Barycentric micro-coordinate change of an offset: db0 = -(x+y+z), db1 = x, db2 = y, db3 = z.
// A point has "class mask" bit k set iff its barycentric coordinate b_k is zero; a micro-tet
// incident to it lies in the closure iff db_k >= 0 for all its vertices and all k in the mask.
inline int pointMask( i64 N, i64 x, i64 y, i64 z )
{
   int m = 0;
   if ( N - x - y - z == 0 ) m |= 1;
   if ( x == 0 ) m |= 2;
   if ( y == 0 ) m |= 4;
   if ( z == 0 ) m |= 8;
   return m;
}
inline bool relAllowed( int mask, const int* r )
{
   if ( ( mask & 1 ) && -( r[0] + r[1] + r[2] ) < 0 ) return false;
   if ( ( mask & 2 ) && r[0] < 0 ) return false;
   if ( ( mask & 4 ) && r[1] < 0 ) return false;
   if ( ( mask & 8 ) && r[2] < 0 ) return false;
   return true;
}
inline bool inClosure( i64 N, i64 x, i64 y, i64 z ) { return x >= 0 && y >= 0 && z >= 0 && x + y + z <= N; }

// P1 element stiffness  K_ij = |T| grad(phi_i).grad(phi_j)  for a tetrahedron.
// (What src/hyteg/forms/form_fenics_generated/p1_tet_diffusion.h tabulate_tensor computes.)
void p1Stiffness( const std::array< std::array< double, 3 >, 4 >& X, double K[4][4], double* absDetOut = nullptr )
{
   double J[3][3];
   for ( int r = 0; r < 3; ++r )
      for ( int c = 0; c < 3; ++c )
         J[r][c] = X[c + 1][r] - X[0][r]; // columns = edge vectors
   const double det = J[0][0] * ( J[1][1] * J[2][2] - J[1][2] * J[2][1] ) -
                      J[0][1] * ( J[1][0] * J[2][2] - J[1][2] * J[2][0] ) +
                      J[0][2] * ( J[1][0] * J[2][1] - J[1][1] * J[2][0] );
   // inverse transpose rows = gradients of barycentric coords 1..3
   double inv[3][3];
   inv[0][0] = ( J[1][1] * J[2][2] - J[1][2] * J[2][1] ) / det;
   inv[0][1] = ( J[0][2] * J[2][1] - J[0][1] * J[2][2] ) / det;
   inv[0][2] = ( J[0][1] * J[1][2] - J[0][2] * J[1][1] ) / det;
   inv[1][0] = ( J[1][2] * J[2][0] - J[1][0] * J[2][2] ) / det;
   inv[1][1] = ( J[0][0] * J[2][2] - J[0][2] * J[2][0] ) / det;
   inv[1][2] = ( J[0][2] * J[1][0] - J[0][0] * J[1][2] ) / det;
   inv[2][0] = ( J[1][0] * J[2][1] - J[1][1] * J[2][0] ) / det;
   inv[2][1] = ( J[0][1] * J[2][0] - J[0][0] * J[2][1] ) / det;
   inv[2][2] = ( J[0][0] * J[1][1] - J[0][1] * J[1][0] ) / det;
   double g[4][3];
   for ( int i = 0; i < 3; ++i )
      for ( int d = 0; d < 3; ++d )
         g[i + 1][d] = inv[i][d]; // row i of J^-1 is grad(lambda_{i+1})
   for ( int d = 0; d < 3; ++d )
      g[0][d] = -g[1][d] - g[2][d] - g[3][d];
   const double vol = std::fabs( det ) / 6.0;
   for ( int i = 0; i < 4; ++i )
      for ( int j = 0; j < 4; ++j )
         K[i][j] = vol * ( g[i][0] * g[j][0] + g[i][1] * g[j][1] + g[i][2] * g[j][2] );
   if ( absDetOut )
      *absDetOut = std::fabs( det );
}

// The 5-point degree-3 rule of p1_div_k_grad_affine_q3::integrateAll, tetrahedron
// (src/hyteg/forms/form_hyteg_generated/p1/p1_div_k_grad_affine_q3.cpp:179-381): the centroid
// with weight -2/15 and the four points with barycentric coordinates (1/2, 1/6, 1/6, 1/6)
// (the 1/2 on vertex a) with weight 3/40, on the reference tetrahedron of volume 1/6; the
// element matrix is |det J| sum_q w_q k(x_q) grad(phi_i).grad(phi_j).
// Barycentric coordinates of point q (q = 0 centroid, q = a + 1 the point weighted on a).
inline double divKGradBary( int q, int j ) { return q == 0 ? 0.25 : ( j == q - 1 ? 0.5 : 1.0 / 6.0 ); }
inline double divKGradWeight( int q ) { return q == 0 ? -2.0 / 15.0 : 3.0 / 40.0; }
// 6 sum_q w_q kq[q] (the factor on the stiffness K_ij = |T| grad.grad, |det J| = 6 |T|)
inline double divKGradScale( const double kq[5] )
{
   double s = 0;
   for ( int q = 0; q < 5; ++q )
      s += divKGradWeight( q ) * kq[q];
   return 6.0 * s;
}

// ---------------------------------------------------------------------------
// Topology
// ---------------------------------------------------------------------------
struct Level
{
   int                                 L;
   i64                                 N, S, nDof;
   i64                                 offE, offF, offC, nIntFace, nIntCell;
   std::vector< std::vector< int32_t > > cellMap; // [cell][closure idx] -> DoF
   std::vector< uint8_t >              kind, bc;
   std::vector< int32_t >              owner;
   // entries for non-cell-interior DoFs [0, offC): (cell, x, y, z)
   std::vector< i64 >                  entOff;
   std::vector< std::array< int32_t, 4 > > ent;
};

// IcosahedralShellMap of one macro-cell (src/hyteg/geometry/IcosahedralShellMap.hpp:286-303):
// the ref/ray vertex pair on one radial ray, the two remaining vertices, the pair's radii.
struct ShellMap
{
   std::array< double, 3 > ref, ray, thr, fou;
   double                  radRef = 0, radRay = 0;
};

struct Op
{
   bool variable = false;
   // blending (p1_div_k_grad_blending_q3 on the IcosahedralShellMap): per-cell maps and the
   // coefficient k(x) = exp( alpha (1 - |x|) ) of the mapped point
   bool                    blend = false;
   double                  alpha = 0;
   std::vector< ShellMap > maps;
   // constant: stencil[level][cell][mask][15]
   std::vector< std::vector< std::array< std::array< double, 15 >, 16 > > > st;
   // variable: nodal k per level, element matrices K[level][cell][type][4][4]
   std::vector< std::vector< double > > k;
   // variable, coefficient given as a function (the reference form's callback): per level and
   // cell, 6 sum_q w_q k(x_q) of every micro-tet at index type * closure size + closure index
   // of its vertex 0 (empty: the nodal coefficient k above is used)
   std::vector< std::vector< std::vector< double > > > kq6;
   std::vector< std::vector< std::array< std::array< std::array< double, 4 >, 4 >, 6 > > > K;
};

struct Oracle
{
   std::vector< std::array< double, 3 > > V;
   std::vector< std::array< int, 4 > >    T;
   std::vector< std::array< int, 2 > >    E;
   std::vector< std::array< int, 3 > >    F;
   std::map< std::array< int, 2 >, int >  eId;
   std::map< std::array< int, 3 >, int >  fId;
   std::vector< uint8_t >                 vBc, eBc, fBc;
   std::vector< std::vector< int > >      fEdges, fVerts, eVerts; // closures
   int                                    maxLevel;
   std::vector< Level >                   lv;
   std::vector< Op >                      ops;
   std::vector< double >                  cheb; // Chebyshev smoother: omega_0 .. omega_{order-1}
};

void buildTopology( Oracle& o )
{
   // edges/faces from cells (MeshInfo::addEdge/addFace keep sorted keys; mesh/MeshInfo.cpp:37-72)
   std::set< std::array< int, 2 > > es;
   std::set< std::array< int, 3 > > fs;
   for ( auto& t : o.T )
   {
      for ( int a = 0; a < 4; ++a )
         for ( int b = a + 1; b < 4; ++b )
            es.insert( { std::min( t[a], t[b] ), std::max( t[a], t[b] ) } );
      const int fl[4][3] = { { 0, 1, 2 }, { 0, 1, 3 }, { 0, 2, 3 }, { 1, 2, 3 } };
      for ( auto& f : fl )
      {
         std::array< int, 3 > k = { t[f[0]], t[f[1]], t[f[2]] };
         std::sort( k.begin(), k.end() );
         fs.insert( k );
      }
   }
   for ( auto& e : es )
   {
      o.eId[e] = int( o.E.size() );
      o.E.push_back( e );
   }
   for ( auto& f : fs )
   {
      o.fId[f] = int( o.F.size() );
      o.F.push_back( f );
   }
   // boundary: faces with one neighbour cell, and every edge/vertex of such a face
   // (SetupPrimitiveStorage::setMeshBoundaryFlagsOnBoundary(1,0,true) + create0123BC:
   //  flag 1 -> DirichletBoundary, 0 -> Inner)
   std::vector< int > fCells( o.F.size(), 0 );
   for ( auto& t : o.T )
   {
      const int fl[4][3] = { { 0, 1, 2 }, { 0, 1, 3 }, { 0, 2, 3 }, { 1, 2, 3 } };
      for ( auto& f : fl )
      {
         std::array< int, 3 > k = { t[f[0]], t[f[1]], t[f[2]] };
         std::sort( k.begin(), k.end() );
         fCells[o.fId[k]]++;
      }
   }
   o.vBc.assign( o.V.size(), ORC_INNER );
   o.eBc.assign( o.E.size(), ORC_INNER );
   o.fBc.assign( o.F.size(), ORC_INNER );
   o.fEdges.resize( o.F.size() );
   o.fVerts.resize( o.F.size() );
   o.eVerts.resize( o.E.size() );
   for ( size_t e = 0; e < o.E.size(); ++e )
      o.eVerts[e] = { o.E[e][0], o.E[e][1] };
   for ( size_t f = 0; f < o.F.size(); ++f )
   {
      auto& k       = o.F[f];
      o.fVerts[f]   = { k[0], k[1], k[2] };
      o.fEdges[f]   = { o.eId[{ k[0], k[1] }], o.eId[{ k[0], k[2] }], o.eId[{ k[1], k[2] }] };
      if ( fCells[f] == 1 )
      {
         o.fBc[f] = ORC_DIRICHLET;
         for ( int e : o.fEdges[f] )
            o.eBc[e] = ORC_DIRICHLET;
         for ( int v : o.fVerts[f] )
            o.vBc[v] = ORC_DIRICHLET;
      }
   }
}

void buildLevel( Oracle& o, int L )
{
   Level lv;
   lv.L           = L;
   lv.N           = i64( 1 ) << L;
   const i64 N    = lv.N;
   lv.S           = tetSize( N + 1 );
   const i64 nV   = i64( o.V.size() ), nE = i64( o.E.size() ), nF = i64( o.F.size() ), nC = i64( o.T.size() );
   lv.nIntFace    = N >= 3 ? ( N - 1 ) * ( N - 2 ) / 2 : 0;
   lv.nIntCell    = N >= 4 ? tetSize( N - 3 ) : 0;
   lv.offE        = nV;
   lv.offF        = lv.offE + nE * std::max< i64 >( N - 1, 0 );
   lv.offC        = lv.offF + nF * lv.nIntFace;
   lv.nDof        = lv.offC + nC * lv.nIntCell;
   lv.kind.resize( lv.nDof );
   lv.bc.resize( lv.nDof );
   lv.owner.resize( lv.nDof );
   for ( i64 v = 0; v < nV; ++v )
   {
      lv.kind[v]  = 0;
      lv.bc[v]    = o.vBc[v];
      lv.owner[v] = int32_t( v );
   }
   for ( i64 e = 0; e < nE; ++e )
      for ( i64 i = 0; i < N - 1; ++i )
      {
         i64 d       = lv.offE + e * ( N - 1 ) + i;
         lv.kind[d]  = 1;
         lv.bc[d]    = o.eBc[e];
         lv.owner[d] = int32_t( e );
      }
   for ( i64 f = 0; f < nF; ++f )
      for ( i64 i = 0; i < lv.nIntFace; ++i )
      {
         i64 d       = lv.offF + f * lv.nIntFace + i;
         lv.kind[d]  = 2;
         lv.bc[d]    = o.fBc[f];
         lv.owner[d] = int32_t( f );
      }
   for ( i64 c = 0; c < nC; ++c )
      for ( i64 i = 0; i < lv.nIntCell; ++i )
      {
         i64 d       = lv.offC + c * lv.nIntCell + i;
         lv.kind[d]  = 3;
         lv.bc[d]    = ORC_INNER;
         lv.owner[d] = int32_t( c );
      }
   // closure point -> DoF by exact barycentric key
   lv.cellMap.assign( nC, std::vector< int32_t >( lv.S ) );
   std::vector< std::vector< std::array< int32_t, 4 > > > entries( lv.offC );
   for ( i64 c = 0; c < nC; ++c )
   {
      auto& t = o.T[c];
      for ( i64 z = 0; z <= N; ++z )
         for ( i64 y = 0; y <= N - z; ++y )
            for ( i64 x = 0; x <= N - y - z; ++x )
            {
               const i64 b[4] = { N - x - y - z, x, y, z };
               std::vector< std::pair< int, i64 > > nz;
               for ( int k = 0; k < 4; ++k )
                  if ( b[k] > 0 )
                     nz.push_back( { t[k], b[k] } );
               std::sort( nz.begin(), nz.end() );
               i64 d = -1;
               if ( nz.size() == 1 )
                  d = nz[0].first;
               else if ( nz.size() == 2 )
               {
                  const int e = o.eId.at( { nz[0].first, nz[1].first } );
                  d           = lv.offE + e * ( N - 1 ) + ( nz[1].second - 1 );
               }
               else if ( nz.size() == 3 )
               {
                  const int f = o.fId.at( { nz[0].first, nz[1].first, nz[2].first } );
                  const i64 i = nz[1].second, j = nz[2].second;
                  d = lv.offF + f * lv.nIntFace + ( j - 1 ) * ( N - 1 ) - ( j - 1 ) * j / 2 + ( i - 1 );
               }
               else
               {
                  d = lv.offC + c * lv.nIntCell + cellIdx( N - 3, x - 1, y - 1, z - 1 );
               }
               lv.cellMap[c][cellIdx( N + 1, x, y, z )] = int32_t( d );
               if ( d < lv.offC )
                  entries[d].push_back( { int32_t( c ), int32_t( x ), int32_t( y ), int32_t( z ) } );
            }
   }
   lv.entOff.assign( lv.offC + 1, 0 );
   for ( i64 d = 0; d < lv.offC; ++d )
      lv.entOff[d + 1] = lv.entOff[d] + i64( entries[d].size() );
   lv.ent.reserve( lv.entOff[lv.offC] );
   for ( i64 d = 0; d < lv.offC; ++d )
      for ( auto& e : entries[d] )
         lv.ent.push_back( e );
   o.lv.push_back( std::move( lv ) );
}

std::array< double, 3 > microCoord( const Oracle& o, int c, i64 N, i64 x, i64 y, i64 z )
{
   // vertexdof::macrocell::coordinateFromIndex (src/hyteg/p1functionspace/VertexDoFMacroCell.hpp:68-75)
   const auto& t = o.T[c];
   std::array< double, 3 > p;
   for ( int d = 0; d < 3; ++d )
   {
      const double v0 = o.V[t[0]][d];
      p[d] = v0 + ( o.V[t[1]][d] - v0 ) / double( N ) * double( x ) + ( o.V[t[2]][d] - v0 ) / double( N ) * double( y ) +
             ( o.V[t[3]][d] - v0 ) / double( N ) * double( z );
   }
   return p;
}

// P1 element mass matrix M_ij = |T| (1 + delta_ij) / 20 (the exact integral that
// P1ElementwiseMassOperator's form computes)
void p1Mass( const std::array< std::array< double, 3 >, 4 >& X, double M[4][4] )
{
   double K[4][4], absDet = 0;
   p1Stiffness( X, K, &absDet );
   const double vol = absDet / 6.0;
   for ( int i = 0; i < 4; ++i )
      for ( int j = 0; j < 4; ++j )
         M[i][j] = vol * ( i == j ? 2.0 : 1.0 ) / 20.0;
}

// Element matrices of the six micro-tet shapes of a cell at level L (stiffness, or mass).
void cellElementMatrices( const Oracle& o, int c, i64 N, std::array< std::array< std::array< double, 4 >, 4 >, 6 >& K,
                          bool mass = false )
{
   for ( int t = 0; t < 6; ++t )
   {
      std::array< std::array< double, 3 >, 4 > X;
      for ( int j = 0; j < 4; ++j )
         X[j] = microCoord( o, c, N, kMicro[t][j][0], kMicro[t][j][1], kMicro[t][j][2] );
      double Km[4][4];
      if ( mass )
         p1Mass( X, Km );
      else
         p1Stiffness( X, Km );
      for ( int i = 0; i < 4; ++i )
         for ( int j = 0; j < 4; ++j )
            K[t][i][j] = Km[i][j];
   }
}

// ---------------------------------------------------------------------------
// Blending: IcosahedralShellMap and the p1_div_k_grad_blending_q3 element matrix
// ---------------------------------------------------------------------------
using V3 = std::array< double, 3 >;
inline V3     sub3( const V3& a, const V3& b ) { return { a[0] - b[0], a[1] - b[1], a[2] - b[2] }; }
inline double dot3( const V3& a, const V3& b ) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
inline V3     cross3( const V3& a, const V3& b )
{
   return { a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0] };
}

// classifyTet + classifyVertices + findNonSkewTetInPrism
// (src/hyteg/geometry/IcosahedralShellMap.hpp:299-344, 346-451, 454-492): the cell's vertices
// are inner or outer by radius (within 0.1 % of the radial extent of the outer one); one outer
// vertex = outwards, three = inwards, two = skew. The first vertex pair (in local order) whose
// cross product vanishes relative to their radii (1e-14) lies on one ray. Outwards: ref = the
// outer of the pair; inwards: ref = the inner one; thr = the last remaining local vertex, for
// the other. A skew cell takes the map of the other cell at its first face (local order 012,
// 013, 023, 123) that does not hold both pair vertices and has a second cell.
bool classifyShell( const Oracle& o, const std::map< std::array< int, 3 >, std::vector< int > >& faceCells, int c,
                    ShellMap& m, int depth )
{
   if ( depth > 16 )
      return false;
   const auto& t = o.T[size_t( c )];
   double      rad[4], inner = 1e300, outer = 0;
   for ( int k = 0; k < 4; ++k )
   {
      rad[k] = std::sqrt( dot3( o.V[t[k]], o.V[t[k]] ) );
      inner  = std::min( inner, rad[k] );
      outer  = std::max( outer, rad[k] );
   }
   const double eps    = ( outer - inner ) * 0.001;
   int          nOuter = 0;
   for ( int k = 0; k < 4; ++k )
      nOuter += ( outer - rad[k] ) < eps ? 1 : 0;
   if ( nOuter < 1 || nOuter > 3 )
      return false;
   int  iRef = -1, iRay = -1;
   for ( int k = 0; k < 4 && iRef < 0; ++k )
      for ( int j = k + 1; j < 4 && iRef < 0; ++j )
      {
         const V3 cr = cross3( o.V[t[k]], o.V[t[j]] );
         bool     ok = true;
         for ( int d = 0; d < 3; ++d )
            ok = ok && std::abs( cr[d] ) / ( rad[k] * rad[j] ) <= 1e-14;
         if ( ok )
         {
            iRef = k;
            iRay = j;
         }
      }
   if ( iRef < 0 )
      return false;
   if ( nOuter == 2 )
   {
      static const int kFace[4][3] = { { 0, 1, 2 }, { 0, 1, 3 }, { 0, 2, 3 }, { 1, 2, 3 } };
      for ( const auto& f : kFace )
      {
         bool hasRef = false, hasRay = false;
         for ( int a : f )
         {
            hasRef = hasRef || a == iRef;
            hasRay = hasRay || a == iRay;
         }
         if ( hasRef && hasRay )
            continue;
         std::array< int, 3 > key = { t[f[0]], t[f[1]], t[f[2]] };
         std::sort( key.begin(), key.end() );
         for ( int other : faceCells.at( key ) )
            if ( other != c )
               return classifyShell( o, faceCells, other, m, depth + 1 );
      }
      return false;
   }
   int iThr = -1, iFor = -1;
   for ( int k = 0; k < 4; ++k )
      if ( k != iRef && k != iRay )
         iThr = k;
   for ( int k = 0; k < 4; ++k )
      if ( k != iRef && k != iRay && k != iThr )
         iFor = k;
   if ( ( nOuter == 1 && rad[iRef] < rad[iRay] ) || ( nOuter == 3 && rad[iRef] > rad[iRay] ) )
      std::swap( iRef, iRay );
   m.ref    = o.V[t[iRef]];
   m.ray    = o.V[t[iRay]];
   m.thr    = o.V[t[iThr]];
   m.fou    = o.V[t[iFor]];
   m.radRef = std::sqrt( dot3( m.ref, m.ref ) );
   m.radRay = std::sqrt( dot3( m.ray, m.ray ) );
   return true;
}

// evalF (IcosahedralShellMap.hpp:99-136): the barycentric coordinate b of x with respect to
// the ref vertex in the tet (ref, ray, thr, for) sets the new radius
// radRay + |b| (radRef - radRay); x is scaled radially to it.
V3 shellF( const ShellMap& m, const V3& x )
{
   const V3     nrm  = cross3( sub3( m.thr, m.ray ), sub3( m.fou, m.ray ) );
   const double volT = dot3( sub3( m.ref, m.ray ), nrm ), volX = dot3( sub3( x, m.ray ), nrm );
   const double bary = std::abs( volX / volT );
   const double oldR = std::sqrt( dot3( x, x ) ), newR = m.radRay + bary * ( m.radRef - m.radRay );
   return { x[0] * newR / oldR, x[1] * newR / oldR, x[2] * newR / oldR };
}

// evalDF (IcosahedralShellMap.hpp:173-223), derived from F(x) = x R(x) / |x| with
// R = radRay + (radRef - radRay) volX / volT and grad volX = (thr - ray) x (for - ray):
// DF = R/|x| (I - x x^T / |x|^2) + x (radRef - radRay) n^T / (volT |x|). Returns det DF.
double shellDF( const ShellMap& m, const V3& x, double D[3][3] )
{
   const V3     nrm  = cross3( sub3( m.thr, m.ray ), sub3( m.fou, m.ray ) );
   const double volT = dot3( sub3( m.ref, m.ray ), nrm ), volX = dot3( sub3( x, m.ray ), nrm );
   const double s    = ( m.radRef - m.radRay ) / volT;
   const double R    = m.radRay + s * volX;
   const double r2 = dot3( x, x ), r = std::sqrt( r2 );
   for ( int i = 0; i < 3; ++i )
      for ( int j = 0; j < 3; ++j )
         D[i][j] = R / r * ( ( i == j ? 1.0 : 0.0 ) - x[i] * x[j] / r2 ) + x[i] * s * nrm[j] / r;
   return D[0][0] * ( D[1][1] * D[2][2] - D[1][2] * D[2][1] ) - D[0][1] * ( D[1][0] * D[2][2] - D[1][2] * D[2][0] ) +
          D[0][2] * ( D[1][0] * D[2][1] - D[1][1] * D[2][0] );
}

// p1_div_k_grad_blending_q3::integrateAll, tetrahedron
// (src/hyteg/forms/form_hyteg_generated/p1/p1_div_k_grad_blending_q3.cpp:412-1059):
// A_ij = sum_q w_q k(F(xi_q)) |det J_aff| |det DF(xi_q)| (G_q g_i) . (G_q g_j), G_q = (DF J_aff)^-T,
// g the reference gradients, the 5-point degree-3 rule (centroid, weight -2/15; the four
// points with barycentric (1/2, 1/6, 1/6, 1/6), weight 3/40), xi_q the quadrature point in
// computational coordinates; k(y) = exp( alpha (1 - |y|) ).
void blendElementMatrix( const ShellMap& m, const V3 X[4], double alpha, double A[4][4] )
{
   const V3     e1 = sub3( X[1], X[0] ), e2 = sub3( X[2], X[0] ), e3 = sub3( X[3], X[0] );
   const double detA = dot3( e1, cross3( e2, e3 ) );
   // columns of J_aff^-T: the reference gradients of vertices 1..3 mapped to computational space
   const V3 c1 = cross3( e2, e3 ), c2 = cross3( e3, e1 ), c3 = cross3( e1, e2 );
   V3       ga[4];
   for ( int d = 0; d < 3; ++d )
   {
      ga[1][d] = c1[d] / detA;
      ga[2][d] = c2[d] / detA;
      ga[3][d] = c3[d] / detA;
      ga[0][d] = -( ga[1][d] + ga[2][d] + ga[3][d] );
   }
   for ( int i = 0; i < 4; ++i )
      for ( int j = 0; j < 4; ++j )
         A[i][j] = 0;
   for ( int q = 0; q < 5; ++q )
   {
      double lam[4];
      for ( int j = 0; j < 4; ++j )
         lam[j] = q == 0 ? 0.25 : ( j == q - 1 ? 0.5 : 1.0 / 6.0 );
      V3 xi = { 0, 0, 0 };
      for ( int j = 0; j < 4; ++j )
         for ( int d = 0; d < 3; ++d )
            xi[d] += lam[j] * X[j][d];
      double       D[3][3];
      const double detD = shellDF( m, xi, D );
      const V3     Fx   = shellF( m, xi );
      const double k    = std::exp( alpha * ( 1.0 - std::sqrt( dot3( Fx, Fx ) ) ) );
      // D^-T = cof(D) / det D
      double C[3][3];
      for ( int i = 0; i < 3; ++i )
         for ( int j = 0; j < 3; ++j )
         {
            const int i1 = ( i + 1 ) % 3, i2 = ( i + 2 ) % 3, j1 = ( j + 1 ) % 3, j2 = ( j + 2 ) % 3;
            C[i][j] = ( D[i1][j1] * D[i2][j2] - D[i1][j2] * D[i2][j1] ) / detD;
         }
      V3 g[4];
      for ( int a = 0; a < 4; ++a )
         for ( int i = 0; i < 3; ++i )
            g[a][i] = C[i][0] * ga[a][0] + C[i][1] * ga[a][1] + C[i][2] * ga[a][2];
      const double w = ( q == 0 ? -2.0 / 15.0 : 3.0 / 40.0 ) * k * std::abs( detA ) * std::abs( detD );
      for ( int i = 0; i < 4; ++i )
         for ( int j = 0; j < 4; ++j )
            A[i][j] += w * dot3( g[i], g[j] );
   }
}

// ---------------------------------------------------------------------------
// Row evaluation: the partial row of DoF at closure point p of cell c.
// val(d) supplies the value of DoF d (current or snapshot, see smooth_sor).
// ---------------------------------------------------------------------------
template < typename T, typename Val >
inline void partialRow( const Oracle& o, const Op& op, const Level& lv, int c, i64 x, i64 y, i64 z, Val&& val, T& diag,
                        T& off )
{
   const i64 N    = lv.N;
   const int mask = pointMask( N, x, y, z );
   const auto& map = lv.cellMap[c];
   if ( !op.variable && !op.blend )
   {
      const auto& st = op.st[lv.L][c][mask];
      diag += T( st[0] );
      for ( int q = 1; q < 15; ++q )
      {
         const i64 xx = x + kOff[q][0], yy = y + kOff[q][1], zz = z + kOff[q][2];
         if ( !inClosure( N, xx, yy, zz ) )
            continue;
         off += T( st[q] ) * val( map[cellIdx( N + 1, xx, yy, zz )] );
      }
   }
   else if ( op.blend )
   {
      for ( const auto& in : kIncident )
      {
         bool ok = true;
         for ( int j = 0; j < 4 && ok; ++j )
            ok = relAllowed( mask, in.rel[j] );
         if ( !ok )
            continue;
         V3 X[4];
         for ( int j = 0; j < 4; ++j )
            X[j] = microCoord( o, c, N, x + in.rel[j][0], y + in.rel[j][1], z + in.rel[j][2] );
         double A[4][4];
         blendElementMatrix( op.maps[size_t( c )], X, op.alpha, A );
         for ( int j = 0; j < 4; ++j )
         {
            if ( j == in.k )
               diag += T( A[in.k][j] );
            else
               off += T( A[in.k][j] ) * val( map[cellIdx( N + 1, x + in.rel[j][0], y + in.rel[j][1], z + in.rel[j][2] )] );
         }
      }
   }
   else
   {
      const auto& K  = op.K[lv.L][c];
      const auto& kv = op.k[lv.L];
      for ( const auto& in : kIncident )
      {
         bool ok = true;
         for ( int j = 0; j < 4 && ok; ++j )
            ok = relAllowed( mask, in.rel[j] );
         if ( !ok )
            continue;
         i64 dof[4];
         for ( int j = 0; j < 4; ++j )
            dof[j] = map[cellIdx( N + 1, x + in.rel[j][0], y + in.rel[j][1], z + in.rel[j][2] )];
         // 5-point degree-3 rule of p1_div_k_grad_affine_q3::integrateAll
         // (src/hyteg/forms/form_hyteg_generated/p1/p1_div_k_grad_affine_q3.cpp:179+) with the
         // coefficient callback = P1 interpolant of the nodal k: centroid weight -2/15, four
         // points (1/2,1/6,1/6,1/6) with weight 3/40, all times |det J| = 6|T|.
         double scale; // K holds |T| grad.grad = |detJ|/6 grad.grad
         if ( !op.kq6.empty() )
            scale = op.kq6[lv.L][c][size_t( in.t ) * size_t( lv.S ) +
                                    size_t( cellIdx( N + 1, x + in.rel[0][0], y + in.rel[0][1], z + in.rel[0][2] ) )];
         else
         {
            double kq[5];
            for ( int q = 0; q < 5; ++q )
            {
               double s = 0;
               for ( int j = 0; j < 4; ++j )
                  s += divKGradBary( q, j ) * kv[dof[j]];
               kq[q] = s;
            }
            scale = divKGradScale( kq );
         }
         for ( int j = 0; j < 4; ++j )
         {
            const double a = scale * K[in.t][in.k][j];
            if ( j == in.k )
               diag += T( a );
            else
               off += T( a ) * val( dof[j] );
         }
      }
   }
}

template < typename T, typename Val >
inline void fullRow( const Oracle& o, const Op& op, const Level& lv, i64 d, Val&& val, T& diag, T& off )
{
   if ( d >= lv.offC )
   {
      const i64 c = ( d - lv.offC ) / lv.nIntCell;
      // invert the interior tet index by scanning (used only for per-DoF access paths)
      i64 r = ( d - lv.offC ) % lv.nIntCell;
      const i64 W = lv.N - 3;
      for ( i64 z = 0; z < W; ++z )
      {
         const i64 sl = ( W - z ) * ( W - z + 1 ) / 2;
         if ( r >= sl )
         {
            r -= sl;
            continue;
         }
         for ( i64 y = 0; y < W - z; ++y )
         {
            const i64 rl = W - z - y;
            if ( r >= rl )
            {
               r -= rl;
               continue;
            }
            partialRow( o, op, lv, int( c ), r + 1, y + 1, z + 1, val, diag, off );
            return;
         }
      }
      return;
   }
   for ( i64 e = lv.entOff[d]; e < lv.entOff[d + 1]; ++e )
   {
      const auto& en = lv.ent[e];
      partialRow( o, op, lv, en[0], en[1], en[2], en[3], val, diag, off );
   }
}

inline bool flagged( uint8_t bc, int flag ) { return ( bc & flag ) != 0; }

// apply (P1Operator.hpp:196-324; P1ElementwiseOperator.cpp:64-221)
template < typename T >
void applyT( const Oracle& o, const Op& op, const Level& lv, const T* src, T* dst, int flag, bool add )
{
   auto val = [src]( i64 d ) { return src[d]; };
#pragma omp parallel for schedule( dynamic, 64 )
   for ( i64 d = 0; d < lv.offC; ++d )
   {
      if ( !flagged( lv.bc[d], flag ) )
         continue;
      T diag = 0, off = 0;
      fullRow( o, op, lv, d, val, diag, off );
      const T r = diag * src[d] + off;
      dst[d]    = add ? dst[d] + r : r;
   }
   const i64 N = lv.N;
#pragma omp parallel for schedule( dynamic, 1 )
   for ( i64 c = 0; c < i64( o.T.size() ); ++c )
      for ( i64 z = 1; z <= N; ++z )
         for ( i64 y = 1; y <= N - z; ++y )
            for ( i64 x = 1; x <= N - y - z - 1; ++x )
            {
               const i64 d = lv.cellMap[c][cellIdx( N + 1, x, y, z )];
               T diag = 0, off = 0;
               partialRow( o, op, lv, int( c ), x, y, z, val, diag, off );
               const T r = diag * src[d] + off;
               dst[d]    = add ? dst[d] + r : r;
            }
}

template < typename T >
inline void sorUpdate( T& x, T b, T diag, T off, T relax )
{
   x = ( T( 1 ) - relax ) * x + relax * ( b - off ) / diag;
}

// smooth_sor (P1Operator.hpp:352-422): six-way ghost update, then forward sweeps
// V -> E -> F -> C. Within a macro-face/edge/vertex the sweep is lexicographic and
// reads current values only for DoFs of that primitive's closure; DoFs of other
// primitives are read from the ghost layers filled before the sweep (VertexDoFPackInfo.hpp:
// edge->face only refreshes the face's own boundary, not its ghost layers), i.e.
// from the start-of-sweep snapshot. Macro-cells read their full (refreshed) closure.
//
// smooth_sor_backwards (P1Operator.hpp:385-400, backwards = true): the stages run
// C -> F -> E -> V with a ghost update (cell->face, face->edge, edge->vertex) before each
// of the last three, so a stage reads its own closure current and everything else from
// the state at the start of that stage; inside each primitive the lexicographic order is
// reversed (sor_3D_macrocell_P1_backwards.cpp:52-57, sor_3D_macroface_P1_backwards.cpp).
// stages: bit 0 vertices, 1 edges, 2 faces, 3 cells (15 = the whole sweep; a single stage
// isolates one primitive type's sweep for comparison with that type's generated kernel).
template < typename T >
void sorRefT( const Oracle& o, const Op& op, const Level& lv, T* x, const T* b, T relax, int flag, bool backwards,
              int stages = 15 )
{
   const i64 N = lv.N;
   std::vector< T > xs( x, x + lv.nDof );
   const T* snap = xs.data();
   auto refresh = [&]() { std::copy( x, x + lv.nDof, xs.begin() ); };
   // vertices (VertexDoFMacroVertex.hpp:208-229)
   auto vertices = [&]() {
      for ( i64 k = 0; k < i64( o.V.size() ); ++k )
      {
         const i64 v = backwards ? i64( o.V.size() ) - 1 - k : k;
         if ( !flagged( lv.bc[v], flag ) )
            continue;
         auto val = [&]( i64 d ) { return d == v ? x[d] : snap[d]; };
         T diag = 0, off = 0;
         fullRow( o, op, lv, v, val, diag, off );
         sorUpdate( x[v], b[v], diag, off, relax );
      }
   };
   // edges (P1Operator.hpp:1353-1423), each independent given the snapshot
   auto edges = [&]() {
      if ( N < 2 )
         return;
#pragma omp parallel for schedule( dynamic, 1 )
      for ( i64 e = 0; e < i64( o.E.size() ); ++e )
      {
         if ( !flagged( o.eBc[e], flag ) )
            continue;
         const int va = o.E[e][0], vb = o.E[e][1];
         auto val = [&]( i64 d ) {
            const bool mine = ( lv.kind[d] == 1 && lv.owner[d] == e ) || ( lv.kind[d] == 0 && ( d == va || d == vb ) );
            return mine ? x[d] : snap[d];
         };
         for ( i64 k = 0; k < N - 1; ++k )
         {
            const i64 d = lv.offE + e * ( N - 1 ) + ( backwards ? N - 2 - k : k );
            T diag = 0, off = 0;
            fullRow( o, op, lv, d, val, diag, off );
            sorUpdate( x[d], b[d], diag, off, relax );
         }
      }
   };
   // faces (P1ConstantOperator.cpp:372-534)
   auto faces = [&]() {
      if ( N < 3 )
         return;
#pragma omp parallel for schedule( dynamic, 1 )
      for ( i64 f = 0; f < i64( o.F.size() ); ++f )
      {
         if ( !flagged( o.fBc[f], flag ) )
            continue;
         const auto& fe = o.fEdges[f];
         const auto& fv = o.fVerts[f];
         auto val = [&]( i64 d ) {
            bool mine = false;
            switch ( lv.kind[d] )
            {
            case 2: mine = lv.owner[d] == f; break;
            case 1: mine = lv.owner[d] == fe[0] || lv.owner[d] == fe[1] || lv.owner[d] == fe[2]; break;
            case 0: mine = d == fv[0] || d == fv[1] || d == fv[2]; break;
            default: mine = false;
            }
            return mine ? x[d] : snap[d];
         };
         for ( i64 k = 0; k < lv.nIntFace; ++k )
         {
            const i64 d = lv.offF + f * lv.nIntFace + ( backwards ? lv.nIntFace - 1 - k : k );
            T diag = 0, off = 0;
            fullRow( o, op, lv, d, val, diag, off );
            sorUpdate( x[d], b[d], diag, off, relax );
         }
      }
   };
   // cells (sor_3D_macrocell_P1.cpp:31-77): lexicographic, x fastest; backwards from the
   // last interior point
   auto cells = [&]() {
      auto cur = [x]( i64 d ) { return x[d]; };
#pragma omp parallel for schedule( dynamic, 1 )
      for ( i64 c = 0; c < i64( o.T.size() ); ++c )
         for ( i64 zk = 1; zk <= N; ++zk )
         {
            const i64 z = backwards ? N + 1 - zk : zk;
            for ( i64 yk = 1; yk <= N - z; ++yk )
            {
               const i64 y = backwards ? N - z + 1 - yk : yk;
               for ( i64 xk = 1; xk <= N - y - z - 1; ++xk )
               {
                  const i64 xx = backwards ? N - y - z - xk : xk;
                  const i64 d  = lv.cellMap[c][cellIdx( N + 1, xx, y, z )];
                  T diag = 0, off = 0;
                  partialRow( o, op, lv, int( c ), xx, y, z, cur, diag, off );
                  sorUpdate( x[d], b[d], diag, off, relax );
               }
            }
         }
   };
   if ( !backwards )
   {
      if ( stages & 1 )
         vertices();
      if ( stages & 2 )
         edges();
      if ( stages & 4 )
         faces();
      if ( stages & 8 )
         cells();
   }
   else
   {
      if ( stages & 8 )
         cells();
      refresh();
      if ( stages & 4 )
         faces();
      refresh();
      if ( stages & 2 )
         edges();
      refresh();
      if ( stages & 1 )
         vertices();
   }
}

int dofColour( const Oracle& o, const Level& lv, i64 d, const int* labels, int m )
{
   int32_t c;
   i64     x, y, z;
   if ( d >= lv.offC )
   {
      c = int32_t( ( d - lv.offC ) / lv.nIntCell );
      // find by scanning the cell closure map (per-DoF path; small sizes only)
      const auto& map = lv.cellMap[c];
      const i64 N = lv.N;
      for ( z = 0; z <= N; ++z )
         for ( y = 0; y <= N - z; ++y )
            for ( x = 0; x <= N - y - z; ++x )
               if ( map[cellIdx( N + 1, x, y, z )] == d )
                  goto found;
      return -1;
   }
   else
   {
      const auto& en = lv.ent[lv.entOff[d]];
      c = en[0];
      x = en[1];
      y = en[2];
      z = en[3];
   }
found:
   const auto& t = o.T[c];
   const i64 b[4] = { lv.N - x - y - z, x, y, z };
   i64 s = 0;
   for ( int k = 0; k < 4; ++k )
      s += i64( labels[t[k]] ) * b[k];
   return int( ( ( s % m ) + m ) % m );
}

template < typename T >
void surfaceColourPass( const Oracle& o, const Op& op, const Level& lv, T* x, const T* b, T relax, int flag,
                        const int* labels, int m, int col )
{
   auto cur = [x]( i64 d ) { return x[d]; };
#pragma omp parallel for schedule( dynamic, 64 )
   for ( i64 d = 0; d < lv.offC; ++d )
   {
      if ( !flagged( lv.bc[d], flag ) )
         continue;
      if ( dofColour( o, lv, d, labels, m ) != col )
         continue;
      T diag = 0, off = 0;
      fullRow( o, op, lv, d, cur, diag, off );
      sorUpdate( x[d], b[d], diag, off, relax );
   }
}

template < typename T >
void interiorColourPass( const Oracle& o, const Op& op, const Level& lv, T* x, const T* b, T relax, int col )
{
   const i64 N = lv.N;
   auto cur = [x]( i64 d ) { return x[d]; };
#pragma omp parallel for schedule( dynamic, 1 )
   for ( i64 c = 0; c < i64( o.T.size() ); ++c )
      for ( i64 z = 1; z <= N; ++z )
         for ( i64 y = 1; y <= N - z; ++y )
            for ( i64 xx = 1; xx <= N - y - z - 1; ++xx )
            {
               if ( ( xx + 2 * y + 3 * z ) % 4 != col )
                  continue;
               const i64 d = lv.cellMap[c][cellIdx( N + 1, xx, y, z )];
               T diag = 0, off = 0;
               partialRow( o, op, lv, int( c ), xx, y, z, cur, diag, off );
               sorUpdate( x[d], b[d], diag, off, relax );
            }
}

// Multicolour SOR, the ordering the GPU path uses. First the DoFs on macro-faces,
// -edges and -vertices, by global colour colour(p) = sum_k label(V_k) b_k mod m over the
// barycentric micro-coordinates (c = 0..m-1); then the macro-cell interiors by the local
// colour (x + 2y + 3z) mod 4 (c = 0..3). Within one pass no two DoFs are coupled, so the
// update order inside a pass is irrelevant.
//
// Backwards (the multicolour counterpart of smooth_sor_backwards): the same passes in
// the reverse order, interior colours 3..0 first, then the surface colours m-1..0, so a
// forward sweep followed by a backward one is a symmetric SOR step.
template < typename T >
void sorColoredT( const Oracle& o, const Op& op, const Level& lv, T* x, const T* b, T relax, int flag, const int* labels,
                  int m, bool backwards )
{
   if ( backwards )
   {
      for ( int col = 3; col >= 0; --col )
         interiorColourPass( o, op, lv, x, b, relax, col );
      for ( int col = m - 1; col >= 0; --col )
         surfaceColourPass( o, op, lv, x, b, relax, flag, labels, m, col );
      return;
   }
   for ( int col = 0; col < m; ++col )
      surfaceColourPass( o, op, lv, x, b, relax, flag, labels, m, col );
   for ( int col = 0; col < 4; ++col )
      interiorColourPass( o, op, lv, x, b, relax, col );
}

// Weighted Jacobi (P1Operator.hpp smooth_jac / WeightedJacobiSmoother):
// x <- x + relax * D^-1 (b - A x)
template < typename T >
void jacobiT( const Oracle& o, const Op& op, const Level& lv, T* x, const T* b, T relax, int flag )
{
   std::vector< T > xo( x, x + lv.nDof );
   const T* xs = xo.data();
   auto val = [xs]( i64 d ) { return xs[d]; };
#pragma omp parallel for schedule( dynamic, 256 )
   for ( i64 d = 0; d < lv.nDof; ++d )
   {
      if ( !flagged( lv.bc[d], flag ) )
         continue;
      T diag = 0, off = 0;
      fullRow( o, op, lv, d, val, diag, off );
      x[d] = xs[d] + relax * ( b[d] - off - diag * xs[d] ) / diag;
   }
}

// first (cell, x, y, z) occurrence of every DoF of a level
struct Where
{
   std::vector< std::array< int32_t, 4 > > w;
};
Where whereOf( const Oracle& o, const Level& lv )
{
   Where W;
   W.w.assign( lv.nDof, { -1, 0, 0, 0 } );
   const i64 N = lv.N;
   for ( i64 c = 0; c < i64( o.T.size() ); ++c )
      for ( i64 z = 0; z <= N; ++z )
         for ( i64 y = 0; y <= N - z; ++y )
            for ( i64 x = 0; x <= N - y - z; ++x )
            {
               const i64 d = lv.cellMap[c][cellIdx( N + 1, x, y, z )];
               if ( W.w[d][0] < 0 )
                  W.w[d] = { int32_t( c ), int32_t( x ), int32_t( y ), int32_t( z ) };
            }
   return W;
}

// Linear interpolation of a fine micro-vertex from the coarse level: coincident
// coarse vertex (weight 1) or the midpoint of a coarse micro-edge (1/2, 1/2).
// (P1toP1LinearProlongation.cpp:194-410 with the generated push kernel.)
template < typename T >
T interpolateFine( const Oracle& o, const Level& cl, int c, i64 X, i64 Y, i64 Z, const T* coarse )
{
   const i64 Nc = cl.N;
   const auto& map = cl.cellMap[c];
   const int px = int( X & 1 ), py = int( Y & 1 ), pz = int( Z & 1 );
   if ( !px && !py && !pz )
      return coarse[map[cellIdx( Nc + 1, X / 2, Y / 2, Z / 2 )]];
   int ox = 0, oy = 0, oz = 0;
   const int pat = px | ( py << 1 ) | ( pz << 2 );
   switch ( pat )
   {
   case 1: ox = 1; break;
   case 2: oy = 1; break;
   case 4: oz = 1; break;
   case 3: ox = -1; oy = 1; break;
   case 5: ox = -1; oz = 1; break;
   case 6: oy = -1; oz = 1; break;
   case 7: ox = -1; oy = 1; oz = -1; break;
   }
   const i64 a = map[cellIdx( Nc + 1, ( X - ox ) / 2, ( Y - oy ) / 2, ( Z - oz ) / 2 )];
   const i64 b = map[cellIdx( Nc + 1, ( X + ox ) / 2, ( Y + oy ) / 2, ( Z + oz ) / 2 )];
   return T( 0.5 ) * ( coarse[a] + coarse[b] );
}

template < typename T >
void prolongateT( const Oracle& o, int coarseLevel, const T* coarse, T* fine, int flag, bool add )
{
   const Level& cl = o.lv[coarseLevel];
   const Level& fl = o.lv[coarseLevel + 1];
   Where W = whereOf( o, fl );
#pragma omp parallel for schedule( static )
   for ( i64 d = 0; d < fl.nDof; ++d )
   {
      if ( !flagged( fl.bc[d], flag ) )
         continue;
      const auto& w = W.w[d];
      const T v = interpolateFine( o, cl, w[0], w[1], w[2], w[3], coarse );
      fine[d]   = add ? fine[d] + v : v;
   }
}

// Full-weighting restriction = transpose of the linear prolongation
// (P1toP1LinearRestriction.cpp:168-345 with the generated pull kernel, whose
//  1/#neighbour-cells factors make each fine point count exactly once).
template < typename T >
void restrictT( const Oracle& o, int fineLevel, const T* fine, T* coarse, int flag )
{
   const Level& fl = o.lv[fineLevel];
   const Level& cl = o.lv[fineLevel - 1];
   Where W = whereOf( o, cl );
   const i64 Nf = fl.N;
#pragma omp parallel for schedule( dynamic, 64 )
   for ( i64 d = 0; d < cl.nDof; ++d )
   {
      if ( !flagged( cl.bc[d], flag ) )
         continue;
      // all cells containing the coarse DoF
      std::vector< std::array< int32_t, 4 > > occ;
      if ( d < cl.offC )
         for ( i64 e = cl.entOff[d]; e < cl.entOff[d + 1]; ++e )
            occ.push_back( cl.ent[e] );
      else
         occ.push_back( W.w[d] );
      if ( occ.size() == 1 )
      {
         // a single cell: the fine neighbours inside it are distinct
         const auto& en  = occ[0];
         const i64   X   = 2 * en[1], Y = 2 * en[2], Z = 2 * en[3];
         const auto& map = fl.cellMap[en[0]];
         T           h   = 0;
         for ( int q = 1; q < 15; ++q )
         {
            const i64 xx = X + kOff[q][0], yy = Y + kOff[q][1], zz = Z + kOff[q][2];
            if ( inClosure( Nf, xx, yy, zz ) )
               h += fine[map[cellIdx( Nf + 1, xx, yy, zz )]];
         }
         coarse[d] = fine[map[cellIdx( Nf + 1, X, Y, Z )]] + T( 0.5 ) * h;
         continue;
      }
      std::set< i64 > nbr;
      i64 centre = -1;
      for ( auto& en : occ )
      {
         const i64 X = 2 * en[1], Y = 2 * en[2], Z = 2 * en[3];
         const auto& map = fl.cellMap[en[0]];
         centre = map[cellIdx( Nf + 1, X, Y, Z )];
         for ( int q = 1; q < 15; ++q )
         {
            const i64 xx = X + kOff[q][0], yy = Y + kOff[q][1], zz = Z + kOff[q][2];
            if ( inClosure( Nf, xx, yy, zz ) )
               nbr.insert( map[cellIdx( Nf + 1, xx, yy, zz )] );
         }
      }
      T s = fine[centre];
      T h = 0;
      for ( i64 q : nbr )
         h += fine[q];
      coarse[d] = s + T( 0.5 ) * h;
   }
}

template < typename T >
double dotT( const Level& lv, const T* a, const T* b, int flag )
{
   double s = 0;
#pragma omp parallel for reduction( + : s ) schedule( static )
   for ( i64 d = 0; d < lv.nDof; ++d )
      if ( flagged( lv.bc[d], flag ) )
         s += double( a[d] ) * double( b[d] );
   return s;
}

// CGSolver::solve (src/hyteg/solvers/CGSolver.hpp:66-135, init :237+), identity preconditioner,
// absolute stopping test sqrt(r.r) < tol, flag Inner|Neumann|Freeslip.
template < typename T >
int cgT( const Oracle& o, const Op& op, const Level& lv, T* x, const T* b, double tol, int maxIter )
{
   const int flag = ORC_INNER | ORC_NEUMANN | ORC_FREESLIP;
   const i64 n    = lv.nDof;
   std::vector< T > p( n, 0 ), ap( n, 0 ), r( n, 0 );
   applyT( o, op, lv, x, p.data(), flag, false );
   for ( i64 d = 0; d < n; ++d )
      if ( flagged( lv.bc[d], flag ) )
         r[d] = b[d] - p[d];
   for ( i64 d = 0; d < n; ++d )
      if ( flagged( lv.bc[d], flag ) )
         p[d] = r[d];
   double prsold = dotT( lv, r.data(), r.data(), flag );
   if ( std::sqrt( prsold ) < tol )
      return 0;
   int it = 0;
   for ( ; it < maxIter; ++it )
   {
      applyT( o, op, lv, p.data(), ap.data(), flag, false );
      const double pAp   = dotT( lv, p.data(), ap.data(), flag );
      const T      alpha = T( prsold / pAp );
      for ( i64 d = 0; d < n; ++d )
         if ( flagged( lv.bc[d], flag ) )
         {
            x[d] += alpha * p[d];
            r[d] -= alpha * ap[d];
         }
      const double rsnew = dotT( lv, r.data(), r.data(), flag );
      if ( std::sqrt( rsnew ) < tol )
         break;
      const T beta = T( rsnew / prsold );
      for ( i64 d = 0; d < n; ++d )
         if ( flagged( lv.bc[d], flag ) )
            p[d] = r[d] + beta * p[d];
      prsold = rsnew;
   }
   return it;
}

Oracle* H( void* h ) { return static_cast< Oracle* >( h ); }

// ---------------------------------------------------------------------------
// GMG (GeometricMultigridSolver.hpp:136-235)
// ---------------------------------------------------------------------------
// diag(A) of every DoF (the full row's diagonal: macro-primitive DoFs sum their cells)
template < typename T >
void invDiagT( const Oracle& o, const Op& op, const Level& lv, T* out )
{
   auto zero = []( i64 ) { return T( 0 ); };
   for ( i64 d = 0; d < lv.offC; ++d )
   {
      T diag = 0, off = 0;
      fullRow( o, op, lv, d, zero, diag, off );
      out[d] = T( 1 ) / diag;
   }
   const i64 N = lv.N;
   for ( i64 c = 0; c < i64( o.T.size() ); ++c )
      for ( i64 z = 1; z <= N; ++z )
         for ( i64 y = 1; y <= N - z; ++y )
            for ( i64 x = 1; x <= N - y - z - 1; ++x )
            {
               T diag = 0, off = 0;
               partialRow( o, op, lv, int( c ), x, y, z, zero, diag, off );
               out[lv.cellMap[c][cellIdx( N + 1, x, y, z )]] = T( 1 ) / diag;
            }
}

// ChebyshevSmoother::solve (src/hyteg/solvers/ChebyshevSmoother.hpp:49-96) on flag
// Inner|Neumann: t = D^-1 (b - A x), x += w_0 t, then for k >= 1 t = D^-1 A t, x += w_k t.
template < typename T >
void chebyshevT( const Oracle& o, const Op& op, const Level& lv, T* x, const T* b, const std::vector< double >& w )
{
   const int flag = ORC_INNER | ORC_NEUMANN;
   std::vector< T > inv( lv.nDof ), t( lv.nDof, T( 0 ) ), t2( lv.nDof, T( 0 ) );
   invDiagT( o, op, lv, inv.data() );
   applyT( o, op, lv, x, t.data(), flag, false );
   for ( i64 d = 0; d < lv.nDof; ++d )
      if ( flagged( lv.bc[d], flag ) )
      {
         t[d] = inv[d] * ( b[d] - t[d] );
         x[d] += T( w[0] ) * t[d];
      }
   for ( size_t k = 1; k < w.size(); ++k )
   {
      applyT( o, op, lv, t.data(), t2.data(), flag, false );
      for ( i64 d = 0; d < lv.nDof; ++d )
         if ( flagged( lv.bc[d], flag ) )
         {
            t[d] = inv[d] * t2[d];
            x[d] += T( w[k] ) * t[d];
         }
   }
}

// Power-basis coefficients w_0 .. w_{k-1} of the Chebyshev smoother of order k for the
// eigenvalue interval [lo, hi] of D^-1 A: the residual polynomial is
// r(l) = T_k((th - l) / de) / T_k(th / de), th = (hi + lo) / 2, de = (hi - lo) / 2, T_k the
// Chebyshev polynomial of the first kind (the polynomial smoother of Adams, Brezina, Hu and
// Tuminaro, J. Comput. Phys. 188 (2003)), and x += p(D^-1 A) D^-1 r with
// 1 - l p(l) = r(l). The polynomials are expanded with the three-term recurrence.
void chebyshevCoefficients( int order, double lo, double hi, std::vector< double >& w )
{
   const double th = 0.5 * ( hi + lo ), de = 0.5 * ( hi - lo );
   // s(l) = a + c l
   const double a = th / de, c = -1.0 / de;
   std::vector< double > tm( order + 1, 0.0 ), tc( order + 1, 0.0 ), tn( order + 1, 0.0 );
   tm[0] = 1.0;          // T_0
   tc[0] = a, tc[1] = c; // T_1
   if ( order == 1 )
      tn = tc;
   for ( int n = 1; n < order; ++n )
   {
      std::fill( tn.begin(), tn.end(), 0.0 );
      for ( int i = 0; i <= n; ++i )
      {
         tn[i] += 2 * a * tc[i];
         tn[i + 1] += 2 * c * tc[i];
      }
      for ( int i = 0; i <= n; ++i )
         tn[i] -= tm[i];
      tm = tc;
      tc = tn;
   }
   const double t0 = tn[0]; // T_k(th / de) = r's value at 0 before scaling
   w.assign( order, 0.0 );
   for ( int i = 1; i <= order; ++i )
      w[i - 1] = -tn[i] / t0;
}

template < typename T >
struct Hier
{
   std::vector< std::vector< T > > x, b, tmp;
};

struct GmgCfg
{
   int         op, minL, maxL, pre, post, smoother, m;
   double      relax, coarseTol;
   const int*  labels;
   int         cycleType; // 0 = V-cycle, 1 = W-cycle (GeometricMultigridSolver.hpp:201-204)
};

template < typename T >
void smoothT( const Oracle& o, const GmgCfg& g, int level, T* x, const T* b )
{
   const Op& op = o.ops[g.op];
   const Level& lv = o.lv[level];
   const int flag = ORC_INNER | ORC_NEUMANN;
   switch ( g.smoother )
   {
   case 0: sorRefT( o, op, lv, x, b, T( g.relax ), flag, false ); break;
   case 1: sorColoredT( o, op, lv, x, b, T( g.relax ), flag, g.labels, g.m, false ); break;
   case 2: jacobiT( o, op, lv, x, b, T( g.relax ), flag ); break;
   // SymmetricSORSmoother::solve (SymmetricSORSmoother.hpp:38-57): forward, then backwards
   case 3:
      sorRefT( o, op, lv, x, b, T( g.relax ), flag, false );
      sorRefT( o, op, lv, x, b, T( g.relax ), flag, true );
      break;
   case 5: chebyshevT( o, op, lv, x, b, o.cheb ); break;
   default:
      sorColoredT( o, op, lv, x, b, T( g.relax ), flag, g.labels, g.m, false );
      sorColoredT( o, op, lv, x, b, T( g.relax ), flag, g.labels, g.m, true );
   }
}

template < typename T >
void vcycleT( const Oracle& o, const GmgCfg& g, Hier< T >& h, int level )
{
   const int flag = ORC_INNER | ORC_NEUMANN;
   const Op& op   = o.ops[g.op];
   if ( level == g.minL )
   {
      // coarse grid solve in FP64 (the mixed-precision variant keeps it in FP64 too)
      const Level& lv = o.lv[level];
      std::vector< double > xd( h.x[level].begin(), h.x[level].end() ), bd( h.b[level].begin(), h.b[level].end() );
      cgT< double >( o, op, lv, xd.data(), bd.data(), g.coarseTol, 100000 );
      for ( i64 d = 0; d < lv.nDof; ++d )
         h.x[level][d] = T( xd[d] );
      return;
   }
   const Level& lv = o.lv[level];
   for ( int i = 0; i < g.pre; ++i )
      smoothT( o, g, level, h.x[level].data(), h.b[level].data() );
   applyT( o, op, lv, h.x[level].data(), h.tmp[level].data(), flag, false );
   for ( i64 d = 0; d < lv.nDof; ++d )
      if ( flagged( lv.bc[d], flag ) )
         h.tmp[level][d] = h.b[level][d] - h.tmp[level][d];
   restrictT( o, level, h.tmp[level].data(), h.tmp[level - 1].data(), flag );
   const Level& cl = o.lv[level - 1];
   for ( i64 d = 0; d < cl.nDof; ++d )
      if ( flagged( cl.bc[d], flag ) )
         h.b[level - 1][d] = h.tmp[level - 1][d];
   std::fill( h.x[level - 1].begin(), h.x[level - 1].end(), T( 0 ) ); // x.interpolate(0, level-1) on All
   vcycleT( o, g, h, level - 1 );
   if ( g.cycleType == 1 )
      vcycleT( o, g, h, level - 1 );
   prolongateT( o, level - 1, h.x[level - 1].data(), h.x[level].data(), flag, true );
   for ( int i = 0; i < g.post; ++i )
      smoothT( o, g, level, h.x[level].data(), h.b[level].data() );
}

template < typename T >
void allocHier( const Oracle& o, Hier< T >& h, int maxL )
{
   h.x.resize( maxL + 1 );
   h.b.resize( maxL + 1 );
   h.tmp.resize( maxL + 1 );
   for ( int l = 0; l <= maxL; ++l )
   {
      h.x[l].assign( o.lv[l].nDof, T( 0 ) );
      h.b[l].assign( o.lv[l].nDof, T( 0 ) );
      h.tmp[l].assign( o.lv[l].nDof, T( 0 ) );
   }
}

double relResidual( const Oracle& o, const Op& op, int level, const double* x, const double* b, std::vector< double >& r )
{
   const int flag  = ORC_INNER | ORC_NEUMANN;
   const Level& lv = o.lv[level];
   applyT( o, op, lv, x, r.data(), flag, false );
   for ( i64 d = 0; d < lv.nDof; ++d )
      r[d] = flagged( lv.bc[d], flag ) ? b[d] - r[d] : 0.0;
   const double nb = std::sqrt( dotT( lv, b, b, flag ) );
   return std::sqrt( dotT( lv, r.data(), r.data(), flag ) ) / ( nb > 0 ? nb : 1.0 );
}

} // namespace

// ---------------------------------------------------------------------------
// C API
// ---------------------------------------------------------------------------
extern "C" {

void* orc_create( const double* coords, int64_t nv, const int64_t* tets, int64_t nt, int maxLevel )
{
   auto* o = new Oracle;
   o->V.resize( nv );
   for ( int64_t i = 0; i < nv; ++i )
      o->V[i] = { coords[3 * i], coords[3 * i + 1], coords[3 * i + 2] };
   o->T.resize( nt );
   for ( int64_t i = 0; i < nt; ++i )
      o->T[i] = { int( tets[4 * i] ), int( tets[4 * i + 1] ), int( tets[4 * i + 2] ), int( tets[4 * i + 3] ) };
   o->maxLevel = maxLevel;
   buildTopology( *o );
   for ( int l = 0; l <= maxLevel; ++l )
      buildLevel( *o, l );
   orc_op_laplace( o ); // op 0
   return o;
}

void orc_destroy( void* h ) { delete H( h ); }

int64_t orc_num_dofs( void* h, int level ) { return H( h )->lv[level].nDof; }

int64_t orc_num_prims( void* h, int kind )
{
   auto* o = H( h );
   switch ( kind )
   {
   case 0: return int64_t( o->V.size() );
   case 1: return int64_t( o->E.size() );
   case 2: return int64_t( o->F.size() );
   default: return int64_t( o->T.size() );
   }
}

void orc_dof_coords( void* h, int level, double* xyz )
{
   auto* o = H( h );
   const Level& lv = o->lv[level];
   const i64 N = lv.N;
   for ( i64 c = 0; c < i64( o->T.size() ); ++c )
      for ( i64 z = 0; z <= N; ++z )
         for ( i64 y = 0; y <= N - z; ++y )
            for ( i64 x = 0; x <= N - y - z; ++x )
            {
               const i64 d = lv.cellMap[c][cellIdx( N + 1, x, y, z )];
               auto p = microCoord( *o, int( c ), N, x, y, z );
               xyz[3 * d] = p[0];
               xyz[3 * d + 1] = p[1];
               xyz[3 * d + 2] = p[2];
            }
}

void orc_dof_info( void* h, int level, uint8_t* kind, uint8_t* bc )
{
   const Level& lv = H( h )->lv[level];
   std::memcpy( kind, lv.kind.data(), lv.nDof );
   std::memcpy( bc, lv.bc.data(), lv.nDof );
}

void orc_cell_closure_map( void* h, int level, int cell, int32_t* out )
{
   const auto& m = H( h )->lv[level].cellMap[cell];
   std::memcpy( out, m.data(), m.size() * sizeof( int32_t ) );
}

namespace {
// operator with a constant element matrix per micro-tet shape (stiffness or mass): the
// stencils of every cell and class mask
int constantOperator( Oracle* o, bool mass )
{
   Op op;
   op.variable = false;
   op.st.resize( o->maxLevel + 1 );
   for ( int L = 0; L <= o->maxLevel; ++L )
   {
      const i64 N = i64( 1 ) << L;
      op.st[L].resize( o->T.size() );
      for ( size_t c = 0; c < o->T.size(); ++c )
      {
         std::array< std::array< std::array< double, 4 >, 4 >, 6 > K;
         cellElementMatrices( *o, int( c ), N, K, mass );
         for ( int mask = 0; mask < 16; ++mask )
         {
            auto& st = op.st[L][c][mask];
            st.fill( 0.0 );
            // sum of row "k" of every incident micro-tet inside the closure
            // (P1Elements.hpp:215-302 getNeighboringElements, :464-526)
            for ( const auto& in : kIncident )
            {
               bool ok = true;
               for ( int j = 0; j < 4 && ok; ++j )
                  ok = relAllowed( mask, in.rel[j] );
               if ( !ok )
                  continue;
               for ( int j = 0; j < 4; ++j )
                  st[offsetId( in.rel[j][0], in.rel[j][1], in.rel[j][2] )] += K[in.t][in.k][j];
            }
         }
      }
   }
   o->ops.push_back( std::move( op ) );
   return int( o->ops.size() - 1 );
}
} // namespace

int orc_op_laplace( void* h ) { return constantOperator( H( h ), false ); }

int orc_op_mass( void* h ) { return constantOperator( H( h ), true ); }

// P1ElementwiseOperator< p1_div_k_grad_affine_q3 > with the coefficient as the form's callback,
// evaluated at the 5 quadrature points of every micro-tet on every level, as the reference
// assembles it (P1ElementwiseOperator.cpp:64-221 calling integrateAll per micro-tet):
//   kind 1: tanh(2 (x - 1/2)) + 2 (ElementwiseDivKGradCGConvergenceTest);
//   kind 2: exp( radial (1 - |x|) + sigma sqrt(2/M) sum_m cos( w_m . x + phase_m ) ), the random-
//           Fourier-feature field of the benchmarks (w: M x 3, phase: M).
int orc_op_divkgrad_callback( void* h, int kind, const double* w, const double* phase, int modes, double sigma,
                              double radial )
{
   auto* o = H( h );
   if ( kind != 1 && kind != 2 )
      return -1;
   auto kfun = [&]( const double* x ) {
      if ( kind == 1 )
         return std::tanh( 2.0 * ( x[0] - 0.5 ) ) + 2.0;
      double g = 0;
      for ( int m = 0; m < modes; ++m )
         g += std::cos( w[3 * m] * x[0] + w[3 * m + 1] * x[1] + w[3 * m + 2] * x[2] + phase[m] );
      const double r = std::sqrt( x[0] * x[0] + x[1] * x[1] + x[2] * x[2] );
      return std::exp( radial * ( 1.0 - r ) + sigma * std::sqrt( 2.0 / modes ) * g );
   };
   Op op;
   op.variable = true;
   op.k.resize( o->maxLevel + 1 );
   op.K.resize( o->maxLevel + 1 );
   op.kq6.resize( o->maxLevel + 1 );
   for ( int L = 0; L <= o->maxLevel; ++L )
   {
      const i64 N = i64( 1 ) << L, S = o->lv[L].S;
      op.k[L].assign( o->lv[L].nDof, 0.0 );
      op.K[L].resize( o->T.size() );
      op.kq6[L].resize( o->T.size() );
#pragma omp parallel for schedule( dynamic )
      for ( size_t c = 0; c < o->T.size(); ++c )
      {
         cellElementMatrices( *o, int( c ), N, op.K[L][c] );
         auto& kc = op.kq6[L][c];
         kc.assign( size_t( 6 * S ), 0.0 );
         for ( int t = 0; t < 6; ++t )
            for ( i64 az = 0; az <= N; ++az )
               for ( i64 ay = 0; ay + az <= N; ++ay )
                  for ( i64 ax = 0; ax + ay + az <= N; ++ax )
                  {
                     bool inside = true;
                     for ( int j = 0; j < 4 && inside; ++j )
                        inside = inClosure( N, ax + kMicro[t][j][0], ay + kMicro[t][j][1], az + kMicro[t][j][2] );
                     if ( !inside )
                        continue;
                     std::array< double, 3 > X[4];
                     for ( int j = 0; j < 4; ++j )
                        X[j] = microCoord( *o, int( c ), N, ax + kMicro[t][j][0], ay + kMicro[t][j][1],
                                           az + kMicro[t][j][2] );
                     double kq[5];
                     for ( int q = 0; q < 5; ++q )
                     {
                        double x[3] = { 0, 0, 0 };
                        for ( int j = 0; j < 4; ++j )
                           for ( int d = 0; d < 3; ++d )
                              x[d] += divKGradBary( q, j ) * X[j][d];
                        kq[q] = kfun( x );
                     }
                     kc[size_t( t ) * size_t( S ) + size_t( cellIdx( N + 1, ax + kMicro[t][0][0], ay + kMicro[t][0][1],
                                                                     az + kMicro[t][0][2] ) )] = divKGradScale( kq );
                  }
      }
   }
   o->ops.push_back( std::move( op ) );
   return int( o->ops.size() - 1 );
}

int orc_op_divkgrad( void* h, const double* const* nodalK )
{
   auto* o = H( h );
   Op op;
   op.variable = true;
   op.k.resize( o->maxLevel + 1 );
   op.K.resize( o->maxLevel + 1 );
   for ( int L = 0; L <= o->maxLevel; ++L )
   {
      op.k[L].assign( nodalK[L], nodalK[L] + o->lv[L].nDof );
      op.K[L].resize( o->T.size() );
      for ( size_t c = 0; c < o->T.size(); ++c )
         cellElementMatrices( *o, int( c ), i64( 1 ) << L, op.K[L][c] );
   }
   o->ops.push_back( std::move( op ) );
   return int( o->ops.size() - 1 );
}

namespace {
std::map< std::array< int, 3 >, std::vector< int > > faceCellLists( const Oracle& o )
{
   std::map< std::array< int, 3 >, std::vector< int > > fc;
   static const int kFace[4][3] = { { 0, 1, 2 }, { 0, 1, 3 }, { 0, 2, 3 }, { 1, 2, 3 } };
   for ( size_t c = 0; c < o.T.size(); ++c )
      for ( const auto& f : kFace )
      {
         std::array< int, 3 > key = { o.T[c][f[0]], o.T[c][f[1]], o.T[c][f[2]] };
         std::sort( key.begin(), key.end() );
         fc[key].push_back( int( c ) );
      }
   return fc;
}
bool shellMaps( const Oracle& o, std::vector< ShellMap >& maps )
{
   const auto fc = faceCellLists( o );
   maps.resize( o.T.size() );
   for ( size_t c = 0; c < o.T.size(); ++c )
      if ( !classifyShell( o, fc, int( c ), maps[c], 0 ) )
         return false;
   return true;
}
} // namespace

int orc_op_blend_div_k_grad( void* h, double alpha )
{
   auto* o = H( h );
   Op    op;
   op.blend = true;
   op.alpha = alpha;
   if ( !shellMaps( *o, op.maps ) )
      return -1;
   o->ops.push_back( std::move( op ) );
   return int( o->ops.size() - 1 );
}

int orc_shell_map_eval( void* h, int cell, const double* x, double* Fx, double* DF )
{
   std::vector< ShellMap > maps;
   if ( !shellMaps( *H( h ), maps ) )
      return -1;
   const V3 p  = { x[0], x[1], x[2] };
   const V3 f  = shellF( maps[size_t( cell )], p );
   double   D[3][3];
   shellDF( maps[size_t( cell )], p, D );
   for ( int i = 0; i < 3; ++i )
   {
      Fx[i] = f[i];
      for ( int j = 0; j < 3; ++j )
         DF[3 * i + j] = D[i][j];
   }
   return 0;
}

int orc_blend_element_matrix( void* h, int cell, const double* X12, double alpha, double* out16 )
{
   std::vector< ShellMap > maps;
   if ( !shellMaps( *H( h ), maps ) )
      return -1;
   V3 X[4];
   for ( int j = 0; j < 4; ++j )
      X[j] = { X12[3 * j], X12[3 * j + 1], X12[3 * j + 2] };
   double A[4][4];
   blendElementMatrix( maps[size_t( cell )], X, alpha, A );
   for ( int i = 0; i < 4; ++i )
      for ( int j = 0; j < 4; ++j )
         out16[4 * i + j] = A[i][j];
   return 0;
}

int orc_set_threads( int n )
{
#ifdef _OPENMP
   if ( n > 0 )
      omp_set_num_threads( n );
   return omp_get_max_threads();
#else
   (void) n;
   return 1;
#endif
}

int orc_divkgrad_element_matrix( const double* X12, int kind, const double* k4, double* out16 )
{
   std::array< std::array< double, 3 >, 4 > X;
   for ( int j = 0; j < 4; ++j )
      X[j] = { X12[3 * j], X12[3 * j + 1], X12[3 * j + 2] };
   double kq[5];
   for ( int q = 0; q < 5; ++q )
   {
      double x[3] = { 0, 0, 0 }, kl = 0;
      for ( int j = 0; j < 4; ++j )
      {
         for ( int d = 0; d < 3; ++d )
            x[d] += divKGradBary( q, j ) * X[j][d];
         kl += divKGradBary( q, j ) * k4[j];
      }
      if ( kind == 0 )
         kq[q] = kl; // the P1 interpolant of the nodal values k4
      else if ( kind == 1 )
         kq[q] = std::tanh( 2.0 * ( x[0] - 0.5 ) ) + 2.0; // ElementwiseDivKGradCGConvergenceTest's k
      else
         return -1;
   }
   double K[4][4];
   p1Stiffness( X, K );
   const double sc = divKGradScale( kq );
   for ( int i = 0; i < 4; ++i )
      for ( int j = 0; j < 4; ++j )
         out16[4 * i + j] = sc * K[i][j];
   return 0;
}

void orc_cell_stencil( void* h, int op, int level, int cell, int mask, double* out15 )
{
   const auto& st = H( h )->ops[op].st[level][cell][mask];
   for ( int q = 0; q < 15; ++q )
      out15[q] = st[q];
}

void orc_apply( void* h, int op, int level, const double* src, double* dst, int flag, int add )
{
   auto* o = H( h );
   applyT( *o, o->ops[op], o->lv[level], src, dst, flag, add != 0 );
}

void orc_sor_ref( void* h, int op, int level, double* x, const double* b, double relax, int flag, int backwards )
{
   auto* o = H( h );
   sorRefT( *o, o->ops[op], o->lv[level], x, b, relax, flag, backwards != 0 );
}

void orc_apply_rows( void* h, int op, int level, const double* src, const int64_t* dofs, int64_t n, double* out )
{
   auto*        o  = H( h );
   const Op&    O  = o->ops[op];
   const Level& lv = o->lv[level];
#pragma omp parallel for schedule( dynamic, 16 )
   for ( int64_t i = 0; i < n; ++i )
   {
      const i64 d    = dofs[i];
      double    diag = 0, off = 0;
      fullRow( *o, O, lv, d, [src]( i64 k ) { return src[k]; }, diag, off );
      out[i] = diag * src[d] + off;
   }
}

void orc_sor_ref_stages( void* h, int op, int level, double* x, const double* b, double relax, int flag, int backwards,
                         int stages )
{
   auto* o = H( h );
   sorRefT( *o, o->ops[op], o->lv[level], x, b, relax, flag, backwards != 0, stages );
}

void orc_sor_colored( void* h, int op, int level, double* x, const double* b, double relax, int flag, const int* labels,
                      int m, int backwards )
{
   auto* o = H( h );
   sorColoredT( *o, o->ops[op], o->lv[level], x, b, relax, flag, labels, m, backwards != 0 );
}

void orc_jacobi( void* h, int op, int level, double* x, const double* b, double relax, int flag )
{
   auto* o = H( h );
   jacobiT( *o, o->ops[op], o->lv[level], x, b, relax, flag );
}

void orc_prolongate( void* h, int coarseLevel, const double* coarse, double* fine, int flag, int add )
{
   prolongateT( *H( h ), coarseLevel, coarse, fine, flag, add != 0 );
}

void orc_restrict( void* h, int fineLevel, const double* fine, double* coarse, int flag )
{
   restrictT( *H( h ), fineLevel, fine, coarse, flag );
}

void orc_chebyshev_coefficients( int order, double lower, double upper, double* out )
{
   std::vector< double > w;
   chebyshevCoefficients( order, lower, upper, w );
   std::copy( w.begin(), w.end(), out );
}

void orc_set_chebyshev( void* h, int order, double lower, double upper )
{
   chebyshevCoefficients( order, lower, upper, H( h )->cheb );
}

void orc_inv_diag( void* h, int op, int level, double* out )
{
   auto* o = H( h );
   invDiagT( *o, o->ops[op], o->lv[level], out );
}

void orc_smooth_chebyshev( void* h, int op, int level, double* x, const double* b )
{
   auto* o = H( h );
   chebyshevT( *o, o->ops[op], o->lv[level], x, b, o->cheb );
}

// estimateSpectralRadiusWithPowerIteration (src/hyteg/numerictools/SpectrumEstimation.hpp:57-81)
// on D^-1 A (chebyshev::estimateRadius), flag All; x is the start vector and is overwritten
double orc_spectral_radius( void* h, int op, int level, int iterations, double* x )
{
   auto*        o  = H( h );
   const Op&    A  = o->ops[op];
   const Level& lv = o->lv[level];
   std::vector< double > inv( lv.nDof ), ax( lv.nDof );
   invDiagT( *o, A, lv, inv.data() );
   auto opApply = [&]( const double* src, double* dst ) {
      applyT( *o, A, lv, src, dst, ORC_ALL, false );
      for ( i64 d = 0; d < lv.nDof; ++d )
         dst[d] *= inv[d];
   };
   double norm = std::sqrt( dotT( lv, x, x, ORC_ALL ) );
   for ( i64 d = 0; d < lv.nDof; ++d )
      x[d] /= norm;
   opApply( x, ax.data() );
   double radius = 0;
   for ( int it = 1; it <= iterations; ++it )
   {
      norm = std::sqrt( dotT( lv, ax.data(), ax.data(), ORC_ALL ) );
      for ( i64 d = 0; d < lv.nDof; ++d )
         x[d] = ax[d] / norm;
      opApply( x, ax.data() );
      radius = dotT( lv, x, ax.data(), ORC_ALL );
   }
   return radius;
}

double orc_dot( void* h, int level, const double* a, const double* b, int flag )
{
   return dotT( H( h )->lv[level], a, b, flag );
}

int orc_cg( void* h, int op, int level, double* x, const double* b, double tol, int maxIter )
{
   auto* o = H( h );
   return cgT( *o, o->ops[op], o->lv[level], x, b, tol, maxIter );
}

int orc_gmg_solve( void* h, int op, int minLevel, int maxLevel, double* x, const double* b, int pre, int post,
                   double relax, int smoother, const int* labels, int m, double coarseTol, int maxCycles, double relTol,
                   int precision, double* history, int cycleType )
{
   auto* o = H( h );
   GmgCfg g{ op, minLevel, maxLevel, pre, post, smoother, m, relax, coarseTol, labels, cycleType };
   const Op& A = o->ops[op];
   const Level& lv = o->lv[maxLevel];
   const int flag  = ORC_INNER | ORC_NEUMANN;
   std::vector< double > r( lv.nDof );
   double rel = relResidual( *o, A, maxLevel, x, b, r );
   if ( history )
      history[0] = rel;
   int cyc = 0;
   if ( precision == 64 )
   {
      Hier< double > hd;
      allocHier( *o, hd, maxLevel );
      hd.x[maxLevel].assign( x, x + lv.nDof );
      hd.b[maxLevel].assign( b, b + lv.nDof );
      while ( cyc < maxCycles && rel > relTol )
      {
         vcycleT( *o, g, hd, maxLevel );
         hd.b[maxLevel].assign( b, b + lv.nDof ); // coarse levels of b are scratch; finest is restored
         ++cyc;
         rel = relResidual( *o, A, maxLevel, hd.x[maxLevel].data(), b, r );
         if ( history )
            history[cyc] = rel;
      }
      std::copy( hd.x[maxLevel].begin(), hd.x[maxLevel].end(), x );
   }
   else
   {
      // FP32 V-cycle on the residual equation inside FP64 iterative refinement
      // (tests/hyteg/mixedPrecision/mixedPrecisionIterativeRefinement.cpp:162-171).
      Hier< float > hf;
      allocHier( *o, hf, maxLevel );
      while ( cyc < maxCycles && rel > relTol )
      {
         for ( i64 d = 0; d < lv.nDof; ++d )
         {
            hf.b[maxLevel][d] = float( r[d] );
            hf.x[maxLevel][d] = 0.0f;
         }
         vcycleT( *o, g, hf, maxLevel );
         for ( i64 d = 0; d < lv.nDof; ++d )
            if ( flagged( lv.bc[d], flag ) )
               x[d] += double( hf.x[maxLevel][d] );
         ++cyc;
         rel = relResidual( *o, A, maxLevel, x, b, r );
         if ( history )
            history[cyc] = rel;
      }
   }
   return cyc;
}

} // extern "C"
