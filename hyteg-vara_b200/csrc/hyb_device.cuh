// Device-side data layout and per-point arithmetic of the P1 multigrid path.
//
// Layout in HBM. A function on level L stores, for every macro-cell, the values
// of its whole closure (interior, faces, edges, vertices: (N+1)(N+2)(N+3)/6
// points, N = 2^L) in the reference's tetrahedral linear order
// (src/hyteg/indexing/MacroCellIndexing.hpp:37-54, x fastest, then y, then z);
// each cell slab is padded to a multiple of 32 values. A micro-vertex shared by
// several cells has one replica per cell; every kernel that writes it writes all
// replicas, so all replicas always agree. The reference's ghost-layer copies
// (VertexDoFPackInfo) therefore never run: a "ghost update" is the replica write
// fused into the kernel that produced the value.
//
// Point classes. A closure point's class mask has bit k set iff its barycentric
// micro-coordinate b_k is zero (b = (N-x-y-z, x, y, z)). Mask 0 is the cell
// interior; one bit = a macro-face, two = a macro-edge, three = a macro-vertex.
// Per cell and mask the class table gives the owning primitive and its BC.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace hyb {

struct ClassDev
{
   int32_t id;    // primitive id within its kind
   uint8_t kind;  // 0 vertex, 1 edge, 2 face, 3 cell
   uint8_t bc;    // DoFType bits
   uint8_t owned; // this cell holds the canonical replica
   uint8_t k0, k1, k2; // cell-local indices of the primitive's vertices (sorted-id order)
   uint8_t pad;
   double  invN;  // 1 / #cells adjacent to the primitive (exact in FP64 restriction weights)
};
static_assert( sizeof( ClassDev ) == 24, "ClassDev layout" );

struct TopoDev
{
   int             nC, nF, nE, nV;
   const ClassDev* cls;     // [nC][16]
   const int32_t*  fEmb;    // [nF][2] packed embeddings, -1 if absent
   const int32_t*  eEmbOff; // [nE+1]
   const int32_t*  eEmb;
   const int32_t*  vEmbOff; // [nV+1]
   const int32_t*  vEmb;
   const uint8_t*  fBc;
   const uint8_t*  eBc;
   const uint8_t*  vBc;
   const int8_t*   labels;  // [nC][4] colour labels of the cell's vertices
   int             m;       // number of colours
};

struct LevelDev
{
   int     L, N, W, S, stride; // W = N+1 points per macro-edge, S = closure size
   int     nIntFace, nIntCell;
   int     nBdry;              // nV + nE (N-1) + nF nIntFace
   int     nSeg;               // interior row segments (32 points each)
   const int32_t* seg;         // packed z | y<<10 | x0<<20
   const int32_t* xyz;         // closure index -> x | y<<10 | z<<20
   // Cell-interior points, the same for every cell of the level. A block is a run of
   // interior points at consecutive storage positions whose 15 neighbours sit at the same
   // offsets (a residue group x = 4g + r of one row, r fixed); blk[16 b + q] is the
   // position of stencil neighbour q of point g of block b, minus g. pts lists every
   // interior point as g | b << 8 in storage order; ptsC lists the points of interior SOR
   // colour c in [ptsOff[c], ptsOff[c + 1]), also in storage order.
   int            nPts;
   int            ptsOff[5];
   const int32_t* blk;
   const int32_t* blkXYZ; // per block: x | y << 10 | z << 20 of its g = 0 point (x steps by 4)
   const int32_t* pts;
   const int32_t* ptsC;
   // Prolongation from the next coarser level, per block b of the point table: the block's
   // points x = x0 + 4g share a parity pattern, so each interpolates the coarse points
   // A(g) and B(g) with x' = xA + 2g (xB + 2g) on fixed coarse rows. pro[2b] = {a0, a1, xA,
   // b0}, pro[2b + 1] = {b1, xB, single, 0}: coarse index of A = (g odd ? a1 : a0) +
   // ((xA + 2g) >> 2), of B likewise; single = 1 when the fine point is a coarse point.
   const int4*    pro;
   // Interior quads for the constant-coefficient apply: entry g | row << 8 stands for the
   // points x = 4g .. 4g + 3 of interior row `row` (rowYZ[row] = y | z << 16), in storage
   // order; a quad holds at least one interior point.
   int            nQuads;
   const int32_t* quads;
   const int32_t* rowYZ;
   // Hyperplanes of the reference-order (lexicographic) SOR: the cell-interior points
   // x | y << 10 | z << 20 grouped by t = x + 2y + 3z (hyperplane t at [lexCellOff[t],
   // lexCellOff[t + 1])), and the face-interior points i | j << 16 grouped by t = i + 2j. Every
   // stencil coupling changes t in the direction of the lexicographic order (x fastest, then
   // y, then z; in a face i, then j), so updating the hyperplanes in increasing t equals the
   // lexicographic sweep, and the points of one hyperplane are independent.
   int            nLexCellT, nLexFaceT;
   int            nLexCell, lexCellMax; // interior points; most points on one hyperplane
   const int32_t* lexCell;
   const int32_t* lexCellOff;
   const int32_t* lexFace;
   const int32_t* lexFaceOff;
   // for the point at lexCell[k]: the positions, within their own hyperplanes, of the seven
   // interior neighbours a sweep updates before it, as 7 int16 in one int4 (m = 0..6 for
   // offset sorRefEarlier(bw, m); -1 where the neighbour lies on the closure), forward
   // entries at [k], backward entries at [nLexCell + k]; only where the ring of the cell
   // wavefront fits
   const int4*    lexCellNbr;
   const int32_t* lexOfPts; // hyperplane-list position of each point of `pts`
   const int32_t* lexSidx;  // storage index of the point at lexCell[k]
};

// 15 stencil offsets, order shared with the oracle and the C ABI
__host__ __device__ constexpr int offX( int q )
{
   return q == 1 ? 1 : q == 2 ? -1 : q == 7 ? -1 : q == 8 ? 1 : q == 9 ? -1 : q == 10 ? 1 : q == 13 ? -1 : q == 14 ? 1 : 0;
}
__host__ __device__ constexpr int offY( int q )
{
   return q == 3 ? 1 : q == 4 ? -1 : q == 7 ? 1 : q == 8 ? -1 : q == 11 ? -1 : q == 12 ? 1 : q == 13 ? 1 : q == 14 ? -1 : 0;
}
__host__ __device__ constexpr int offZ( int q )
{
   return q == 5 ? 1 : q == 6 ? -1 : q == 9 ? 1 : q == 10 ? -1 : q == 11 ? 1 : q == 12 ? -1 : q == 13 ? -1 : q == 14 ? 1 : 0;
}

// hyperplane step t(q) = offX + 2 offY + 3 offZ of each offset (never 0, |t| <= 3), and the
// seven offsets of each sweep direction whose neighbours a lexicographic sweep updates
// before the point: t(q) < 0 forwards, t(q) > 0 backwards
__host__ __device__ constexpr int offT( int q ) { return offX( q ) + 2 * offY( q ) + 3 * offZ( q ); }
__host__ __device__ constexpr int sorRefEarlier( int backwards, int m )
{
   return backwards ? ( m == 0 ? 1 : m == 1 ? 3 : m == 2 ? 5 : m == 3 ? 7 : m == 4 ? 9 : m == 5 ? 11 : 14 )
                    : ( m == 0 ? 2 : m == 1 ? 4 : m == 2 ? 6 : m == 3 ? 8 : m == 4 ? 10 : m == 5 ? 12 : 13 );
}

// valid offsets (bit q) of a point of class mask (offset stays inside the closure)
__constant__ const uint16_t kValidOffsets[16] = { 0x7fff, 0x3fd5, 0x5d7b, 0x1d51, 0x36ef, 0x36c5, 0x146b, 0x1441,
                                                  0x4bbf, 0x0b95, 0x493b, 0x0911, 0x02af, 0x0285, 0x002b, 0x0001 };
// incident micro-tets (bit i of the 24 below) lying inside the closure, per class mask
__constant__ const uint32_t kValidTets[16] = { 0xffffff, 0xe324ae, 0x9e4a4d, 0x82000c, 0x458d9b, 0x41048a,
                                               0x040809, 0x000008, 0x381377, 0x200026, 0x180245, 0x000004,
                                               0x000113, 0x000002, 0x000001, 0x000000 };

// The 24 micro-tets incident to a micro-vertex: micro-cell type t (WHITE_UP, BLUE_UP,
// GREEN_UP, WHITE_DOWN, BLUE_DOWN, GREEN_DOWN of src/hyteg/volumedofspace/CellDoFIndexing.hpp:
// 155-198), the vertex's role k in it, and the stencil offset of each of its 4 vertices.
struct IncidentTet
{
   int t, k, q[4];
};
__host__ __device__ constexpr IncidentTet incidentTet( int i )
{
   constexpr int tab[24][6] = { { 0, 0, 0, 1, 3, 5 },   { 0, 1, 2, 0, 7, 9 },    { 0, 2, 4, 8, 0, 11 },  { 0, 3, 6, 10, 12, 0 },
                                { 1, 0, 0, 3, 7, 5 },   { 1, 1, 4, 0, 2, 11 },   { 1, 2, 8, 1, 0, 14 },  { 1, 3, 6, 12, 13, 0 },
                                { 2, 0, 0, 7, 5, 9 },   { 2, 1, 8, 0, 14, 11 },  { 2, 2, 6, 13, 0, 2 },  { 2, 3, 10, 12, 1, 0 },
                                { 3, 0, 0, 5, 9, 11 },  { 3, 1, 6, 0, 2, 4 },    { 3, 2, 10, 1, 0, 8 },  { 3, 3, 12, 3, 7, 0 },
                                { 4, 0, 0, 7, 2, 13 },  { 4, 1, 8, 0, 4, 6 },    { 4, 2, 1, 3, 0, 12 },  { 4, 3, 14, 5, 11, 0 },
                                { 5, 0, 0, 1, 14, 5 },  { 5, 1, 2, 0, 11, 9 },   { 5, 2, 13, 12, 0, 7 }, { 5, 3, 6, 10, 8, 0 } };
   return IncidentTet{ tab[i][0], tab[i][1], { tab[i][2], tab[i][3], tab[i][4], tab[i][5] } };
}
// the three vertices of incident tet i other than the row's point (offsets in the tet's
// vertex order): with the row's point as vertex 0, the row of the element matrix is row 0
struct IncidentOthers
{
   int   q[3];    // stencil offset indices
   float d[3][3]; // their lattice offsets (x, y, z) from the row's point
};
__host__ __device__ constexpr IncidentOthers incidentOthers( int i )
{
   const IncidentTet it = incidentTet( i );
   IncidentOthers    o{ { 0, 0, 0 }, { { 0, 0, 0 }, { 0, 0, 0 }, { 0, 0, 0 } } };
   int               n = 0;
   for ( int j = 0; j < 4; ++j )
      if ( j != it.k )
      {
         o.q[n]    = it.q[j];
         o.d[n][0] = float( offX( it.q[j] ) );
         o.d[n][1] = float( offY( it.q[j] ) );
         o.d[n][2] = float( offZ( it.q[j] ) );
         ++n;
      }
   return o;
}
__constant__ const IncidentOthers kIncidentOthers[24] = {
   incidentOthers( 0 ),  incidentOthers( 1 ),  incidentOthers( 2 ),  incidentOthers( 3 ),  incidentOthers( 4 ),
   incidentOthers( 5 ),  incidentOthers( 6 ),  incidentOthers( 7 ),  incidentOthers( 8 ),  incidentOthers( 9 ),
   incidentOthers( 10 ), incidentOthers( 11 ), incidentOthers( 12 ), incidentOthers( 13 ), incidentOthers( 14 ),
   incidentOthers( 15 ), incidentOthers( 16 ), incidentOthers( 17 ), incidentOthers( 18 ), incidentOthers( 19 ),
   incidentOthers( 20 ), incidentOthers( 21 ), incidentOthers( 22 ), incidentOthers( 23 ) };

// the incident-tet table in constant memory, for loops that index it at run time (a
// warp's lanes read the same entry: a broadcast)
__constant__ const IncidentTet kIncidentTets[24] = {
   incidentTet( 0 ),  incidentTet( 1 ),  incidentTet( 2 ),  incidentTet( 3 ),  incidentTet( 4 ),  incidentTet( 5 ),
   incidentTet( 6 ),  incidentTet( 7 ),  incidentTet( 8 ),  incidentTet( 9 ),  incidentTet( 10 ), incidentTet( 11 ),
   incidentTet( 12 ), incidentTet( 13 ), incidentTet( 14 ), incidentTet( 15 ), incidentTet( 16 ), incidentTet( 17 ),
   incidentTet( 18 ), incidentTet( 19 ), incidentTet( 20 ), incidentTet( 21 ), incidentTet( 22 ), incidentTet( 23 ) };


__host__ __device__ __forceinline__ int tetSize( int w ) { return ( w + 2 ) * ( w + 1 ) * w / 6; }
// first index of row (y, z) in a closure of width W
__host__ __device__ __forceinline__ int rowStart( int W, int y, int z )
{
   const int wms = W - z;
   return tetSize( W ) - tetSize( wms ) + y * ( wms + 1 ) - ( ( y + 1 ) * y ) / 2;
}
// tet-linear index (vertexdof::macrocell::index): the canonical numbering of a tetrahedral
// point set, used for the canonical DoF order of cell interiors
__host__ __device__ __forceinline__ int cidx( int W, int x, int y, int z ) { return rowStart( W, y, z ) + x; }

// Storage layout of a closure slab: rows (y, z) in tet-linear order at their tet-linear
// start, but inside a row of length n the points are grouped by x mod 4 -- all x = 0 mod 4
// first, then 1, 2, 3 -- so that one interior SOR colour ((x + 2y + 3z) mod 4 is fixed in a
// row) is one contiguous run of every row.
__host__ __device__ __forceinline__ int resOff( int r, int n )
{
   const int m = n & 3;
   return r * ( n >> 2 ) + ( r < m ? r : m );
}
__host__ __device__ __forceinline__ int resCarry( int v ) { return v < 0 ? -1 : ( v > 3 ? 1 : 0 ); }
// storage position of closure point (x, y, z)
__host__ __device__ __forceinline__ int sidx( int W, int x, int y, int z )
{
   return rowStart( W, y, z ) + resOff( x & 3, W - y - z ) + ( x >> 2 );
}

__host__ __device__ __forceinline__ int classMask( int N, int x, int y, int z )
{
   return ( N - x - y - z == 0 ? 1 : 0 ) | ( x == 0 ? 2 : 0 ) | ( y == 0 ? 4 : 0 ) | ( z == 0 ? 8 : 0 );
}

// The seven rows a 15-point stencil at row (y, z) touches: start (tet-linear recurrences)
// and length. Order: (y,z), (y+1,z), (y-1,z), (y,z+1), (y,z-1), (y-1,z+1), (y+1,z-1).
// Rows outside the closure (y = 0 or z = 0) get meaningless values and must not be read.
struct StencilRows
{
   int start[7], len[7];
};
__host__ __device__ __forceinline__ StencilRows stencilRows( int W, int y, int z )
{
   StencilRows R;
   const int   n   = W - z - y;
   const int   rs  = rowStart( W, y, z );
   const int   slz = ( W - z ) * ( W - z + 1 ) / 2;     // points in slice z
   const int   slm = ( W - z + 1 ) * ( W - z + 2 ) / 2; // points in slice z-1
   R.start[0] = rs;
   R.len[0]   = n;
   R.start[1] = rs + n;
   R.len[1]   = n - 1;
   R.start[2] = rs - ( n + 1 );
   R.len[2]   = n + 1;
   R.start[3] = rs + slz - y;
   R.len[3]   = n - 1;
   R.start[4] = rs - ( slm - y );
   R.len[4]   = n + 1;
   R.start[5] = R.start[2] + slz - ( y - 1 );
   R.len[5]   = n;
   R.start[6] = R.start[1] - slm + ( y + 1 );
   R.len[6]   = n;
   return R;
}
// stencil offset q -> its row in StencilRows
__host__ __device__ __forceinline__ int offRow( int q )
{
   constexpr int t[15] = { 0, 0, 0, 1, 2, 3, 4, 1, 2, 3, 4, 5, 6, 6, 5 };
   return t[q];
}

// Positions of the 15 neighbours of interior point x = 4g + r of row (y, z), relative to
// g: neighbour q sits at d[q] + g. (The host builds the point tables from sidx and checks
// them against this; the kernels read the tables.)
struct NbrOff
{
   int d[15];
};
__host__ __device__ __forceinline__ NbrOff residueNbr( int W, int y, int z, int r )
{
   const StencilRows R = stencilRows( W, y, z );
   NbrOff            o;
#pragma unroll
   for ( int q = 0; q < 15; ++q )
   {
      const int v = r + offX( q );
      const int k = offRow( q );
      o.d[q]      = R.start[k] + resOff( v & 3, R.len[k] ) + resCarry( v );
   }
   return o;
}

// Unpack a primitive embedding and place primitive-local barycentric weights
// (weights of the primitive's vertices in sorted-id order) into the cell.
__device__ __forceinline__ void embeddingCoords( int32_t packed, int kind, int N, int i, int j, int& cell, int& x, int& y,
                                                 int& z )
{
   cell         = packed & 0xFFFFFF;
   const int k0 = ( packed >> 24 ) & 3, k1 = ( packed >> 26 ) & 3, k2 = ( packed >> 28 ) & 3;
   int       b[4] = { 0, 0, 0, 0 };
   if ( kind == 0 )
      b[k0] = N;
   else if ( kind == 1 )
   {
      b[k0] = N - i;
      b[k1] = i;
   }
   else
   {
      b[k0] = N - i - j;
      b[k1] = i;
      b[k2] = j;
   }
   x = b[1];
   y = b[2];
   z = b[3];
}

__device__ __forceinline__ int colourOf( const TopoDev& tp, int cell, int N, int x, int y, int z )
{
   const int8_t* l = tp.labels + 4 * cell;
   const int     s = int( l[0] ) * ( N - x - y - z ) + int( l[1] ) * x + int( l[2] ) * y + int( l[3] ) * z;
   return ( ( s % tp.m ) + tp.m ) % tp.m;
}

// Operator data of one level, in the compute type T.
template < typename T >
struct OpDev
{
   const T* st;  // constant coefficient: [nC][16][15] partial stencils per class
   const T* K;   // variable coefficient: [nC][6][4][4] micro-tet matrices (1/4 folded in)
   const T* kap; // variable coefficient: nodal k, function layout
   // variable coefficient integrated at quadrature points (the reference form's callback):
   // per cell 6 slabs (one per micro-tet type) holding, at the slab position of a micro-tet's
   // vertex 0, 24 sum_q w_q k(x_q) -- the factor on its matrix K (which has the 1/4 folded
   // in) that replaces the sum of the 4 nodal values; null: nodal k (kap)
   const T* kq;
   int      stride;
   // blending operator (curved shell): element matrices integrated on the fly per row
   const double*  bcell;  // [nC][4][3] macro-cell vertex coordinates (computational domain)
   const double*  bmap;   // [nC][8] shell map of the cell: ray vertex, n = (thr - ray) x (for - ray),
                          // radRay, s = (radRef - radRay) / ((ref - ray) . n)
   double         balpha; // coefficient k(y) = exp( balpha (1 - |y|) )
   int            bN;     // micro-edges per macro-edge (2^level)
};

// Partial row of the operator at closure point (x,y,z) of `cell`: the contributions
// of the micro-tets of this cell only. u = the cell's slab. VAR (throughout the kernels):
// 0 constant stencils, 1 variable coefficient from nodal values (OpDev::kap), 2 variable
// coefficient integrated at quadrature points (OpDev::kq).
template < typename T, int VAR >
__device__ __forceinline__ void partialRow( const OpDev< T >& op, const T* u, int cell, int W, int x, int y,
                                            int z, T& diag, T& off )
{
   const int         N     = W - 1;
   const int         mask  = classMask( N, x, y, z );
   const uint32_t    valid = kValidOffsets[mask];
   const StencilRows R     = stencilRows( W, y, z );
   // positions of the neighbours inside the closure (the others are never read)
   int pos[15];
#pragma unroll
   for ( int q = 0; q < 15; ++q )
   {
      const int xq = x + offX( q ), k = offRow( q );
      pos[q]       = ( valid & ( 1u << q ) ) ? R.start[k] + resOff( xq & 3, R.len[k] ) + ( xq >> 2 ) : 0;
   }
   if constexpr ( !VAR )
   {
      const T* st = op.st + ( size_t( cell ) * 16 + mask ) * 15;
      diag += st[0];
#pragma unroll
      for ( int q = 1; q < 15; ++q )
         if ( valid & ( 1u << q ) )
            off += st[q] * u[pos[q]];
   }
   else
   {
      const T*       kv    = op.kap + size_t( cell ) * op.stride;
      const T*       kqc   = VAR == 2 ? op.kq + size_t( cell ) * 6 * op.stride : nullptr;
      const T*       K     = op.K + size_t( cell ) * 96;
      const uint32_t validT = kValidTets[mask];
#pragma unroll
      for ( int i = 0; i < 24; ++i )
      {
         const IncidentTet it = incidentTet( i );
         if ( !( validT & ( 1u << i ) ) )
            continue;
         T ks;
         if constexpr ( VAR == 2 )
            ks = kqc[size_t( it.t ) * op.stride + pos[it.q[0]]];
         else
            ks = kv[pos[it.q[0]]] + kv[pos[it.q[1]]] + kv[pos[it.q[2]]] + kv[pos[it.q[3]]];
         const T* Kr = K + it.t * 16 + it.k * 4;
#pragma unroll
         for ( int j = 0; j < 4; ++j )
         {
            if ( j == it.k )
               diag += ks * Kr[j];
            else
               off += ks * Kr[j] * u[pos[it.q[j]]];
         }
      }
   }
}

} // namespace hyb
